"""ctypes mirrors of the structures in include/rodgpu.h and the helpers that
need no library of their own.  Importing this module loads nothing: the
functions that fill a configuration or generate a scene take the library that
provides the exported C function (librodgpu.so, librodhost.so, or any other
library built from the same host sources).
"""
import ctypes

_d = ctypes.c_double
_i = ctypes.c_int32

MODEL = {"none": 0, "nsc": 1, "harmonic": 2, "hertz-mindlin": 3}
FRICTION = {"smooth": 0, "cundall": 1, "karnopp": 2}
WARM = {"cache": 0, "none": 1, "mlp": 2}
STATUS = ["ok", "bad argument", "CUDA error", "capacity exceeded", "non-finite state",
          "PSOR not converged", "no CUDA device", "device wait timed out", "call out of order"]


class RgConfig(ctypes.Structure):
    """Mirror of struct rg_config (include/rodgpu.h)."""
    _fields_ = [
        ("n_bodies", _i), ("model", _i), ("dt", _d), ("gravity", _d * 3),
        ("lin_damp", _d), ("ang_damp", _d), ("w_max", _d),
        ("pbc_enabled", _i), ("pbc_min", _d * 3), ("pbc_max", _d * 3),
        ("soft_delta", _d), ("soft_k_scaler", _d), ("soft_damping", _d), ("soft_mu", _d),
        ("soft_mu_static", _d), ("soft_nu", _d), ("soft_kt", _d), ("soft_vel_deadband", _d),
        ("soft_enable_friction", _i), ("soft_friction_mode", _i),
        ("hm_youngs_modulus", _d), ("hm_poisson_ratio", _d), ("hm_restitution", _d),
        ("hm_friction", _d), ("hm_friction_static", _d), ("hm_friction_transition_vel", _d),
        ("hm_rolling_friction", _d), ("hm_enable_tangential", _i), ("hm_enable_rolling", _i),
        ("nsc_mu", _d), ("nsc_beta", _d), ("nsc_cfm", _d), ("nsc_omega", _d), ("nsc_slop", _d),
        ("nsc_tol", _d), ("nsc_velocity_iters", _i), ("nsc_position_stabilization", _i),
        ("nsc_position_iters", _i), ("nsc_position_psor_iters", _i), ("nsc_warm_start", _i),
        ("psor_order", _i), ("skin", _d), ("max_neighbors", _i), ("team_blocks", _i),
        ("nsc_mlp_scope", _i), ("nsc_mlp_min_sweeps", _i), ("near_skin_pct", _i),
        ("spin_limit", _i), ("test_absent_blocks", _i), ("cylinder_enabled", _i), ("cylinder_radius", _d),
        ("cylinder_axis", _d * 3),
    ]


class RgStepStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64), ("contacts", ctypes.c_int64), ("collisions", ctypes.c_int64),
        ("psor_sweeps", ctypes.c_int64), ("psor_sweeps_last", ctypes.c_int64),
        ("list_rebuilds", ctypes.c_int64), ("colors", ctypes.c_int64),
        ("history_size", ctypes.c_int64), ("residual", _d), ("jn_sum", _d), ("jt_sum", _d),
        ("potential_energy", _d), ("kinetic_energy", _d), ("max_residual", _d),
        ("not_converged", ctypes.c_int64), ("device_ms", _d), ("psor_row_sweeps", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64), ("contact_steps", ctypes.c_int64),
        ("near_rebuilds", ctypes.c_int64), ("reserved", ctypes.c_int64 * 1),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


def ptr(a, ctype=_d):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def apply_config(c, **kw):
    for k, v in kw.items():
        if k == "model" and isinstance(v, str):
            v = MODEL[v]
        if k == "soft_friction_mode" and isinstance(v, str):
            v = FRICTION[v]
        if k == "nsc_warm_start" and isinstance(v, str):
            v = WARM[v]
        if k in ("gravity", "pbc_min", "pbc_max", "cylinder_axis"):
            arr = getattr(c, k)
            for j in range(3):
                arr[j] = float(v[j])
            continue
        setattr(c, k, v)
    return c


def config_from(L, **kw):
    """rg_config_default() as exported by library L, with keyword overrides."""
    c = RgConfig()
    L.rg_config_default.argtypes = [ctypes.POINTER(RgConfig)]
    L.rg_config_default.restype = None
    L.rg_config_default(ctypes.byref(c))
    return apply_config(c, **kw)


def bind_scene_lib(L):
    """Declares the scene-generator entry points (host/scene_gen.cpp) and
    rg_config_default (host/config_default.cpp) on library L."""
    dp = ctypes.POINTER(_d)
    L.rg_capsule_mass.argtypes = [ctypes.c_int, dp, dp, dp, dp, dp]
    L.rg_capsule_mass.restype = None
    L.rg_scene_rsa.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_uint64, ctypes.c_int, dp, dp]
    L.rg_scene_rsa.restype = ctypes.c_int
    L.rg_scene_velocities.argtypes = [ctypes.c_int, _d, _d, ctypes.c_uint64, dp, dp]
    L.rg_scene_velocities.restype = None
    L.rg_config_default.argtypes = [ctypes.POINTER(RgConfig)]
    L.rg_config_default.restype = None
    return L
