"""ctypes binding of librodgpu.so, the B200 contact hot path.

This is the thin Python edge over the C ABI declared in include/rodgpu.h.
It holds no physics: every step, detection and force evaluation runs in the
CUDA library, which must be loadable (there is no CPU fallback; a missing or
unloadable library raises at import of the first System).

Arrays are numpy float64 in the ABI's layouts: x (N,3), q (N,4) as
(w,x,y,z), v (N,3), w (N,3).
"""
import ctypes
import os

import numpy as np

from .abi import (FRICTION, MODEL, STATUS, WARM, RgConfig, RgStepStats, apply_config,  # noqa: F401
                  bind_scene_lib, config_from, ptr)

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "librodgpu.so")
HOST_PATH = os.path.join(PKG, "librodhost.so")

_d = ctypes.c_double
_i = ctypes.c_int32

_lib = None
_host = None

# Every entry point of include/rodgpu.h, in declaration order.
ABI_SYMBOLS = [
    "rg_abi_version", "rg_config_default", "rg_status_string", "rg_last_error", "rg_create",
    "rg_destroy", "rg_get_config", "rg_set_bodies", "rg_set_state", "rg_get_state", "rg_step",
    "rg_detect", "rg_get_impulses", "rg_set_network_export", "rg_get_contact_network",
    "rg_compute_forces", "rg_get_history", "rg_set_profiling",
    "rg_get_profile", "rg_get_phase_times", "rg_scene_rsa_device", "rg_detect_noalloc",
    "rg_mlp_param_count", "rg_mlp_set_params", "rg_mlp_get_params", "rg_mlp_record",
    "rg_mlp_records", "rg_mlp_train", "rg_mlp_infer", "rg_batch_create", "rg_batch_destroy",
    "rg_batch_set_bodies", "rg_batch_set_state", "rg_batch_get_state", "rg_batch_step",
    "rg_batch_set_mlp", "rg_mlp_grad", "rg_batch_size", "rg_batch_member", "rg_batch_last_error",
    "rg_batch_set_schedule", "rg_batch_get_schedule", "rg_batch_autotune",
    "rg_batch_set_state_all", "rg_batch_get_state_all", "rg_batch_get_costs", "rg_batch_get_team_times",
]


def lib():
    """Loads librodgpu.so (raises if it is missing: no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"librodgpu.so not built ({LIB_PATH}); run rod-dynamics-3d_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        dp = ctypes.POINTER(_d)
        L.rg_config_default.argtypes = [ctypes.POINTER(RgConfig)]
        L.rg_config_default.restype = None
        L.rg_status_string.restype = ctypes.c_char_p
        L.rg_last_error.argtypes = [P]
        L.rg_last_error.restype = ctypes.c_char_p
        L.rg_create.argtypes = [ctypes.POINTER(RgConfig), ctypes.POINTER(P)]
        L.rg_destroy.argtypes = [P]
        L.rg_set_bodies.argtypes = [P, dp, dp, dp, dp, dp]
        L.rg_set_state.argtypes = [P, dp, dp, dp, dp, dp, dp]
        L.rg_get_state.argtypes = [P, dp, dp, dp, dp, dp, dp]
        L.rg_step.argtypes = [P, ctypes.c_int, ctypes.POINTER(RgStepStats)]
        L.rg_detect.argtypes = [P, _d, ctypes.POINTER(_i), dp, dp, ctypes.c_size_t,
                                ctypes.POINTER(ctypes.c_size_t)]
        L.rg_get_impulses.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.POINTER(_i),
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.rg_compute_forces.argtypes = [P, dp, dp, dp]
        L.rg_scene_rsa_device.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_uint64, ctypes.c_int, dp, dp,
                                          ctypes.POINTER(ctypes.c_int)]
        L.rg_set_network_export.argtypes = [P, ctypes.c_int]
        L.rg_get_contact_network.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_size_t)]
        L.rg_get_history.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.rg_set_profiling.argtypes = [P, ctypes.c_int]
        L.rg_get_profile.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int64)]
        L.rg_get_phase_times.argtypes = [P, dp, ctypes.c_int]
        L.rg_detect_noalloc.argtypes = [P, P, P, P, P, ctypes.c_int, ctypes.c_int, dp, dp, _d, P, P,
                                        ctypes.c_int, P, P]
        L.rg_mlp_param_count.restype = ctypes.c_size_t
        fp = ctypes.POINTER(ctypes.c_float)
        L.rg_mlp_set_params.argtypes = [P, fp, ctypes.c_size_t]
        L.rg_mlp_get_params.argtypes = [P, fp, ctypes.c_size_t]
        L.rg_mlp_record.argtypes = [P, ctypes.c_int, ctypes.c_size_t]
        L.rg_mlp_records.argtypes = [P, fp, fp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.rg_mlp_train.argtypes = [P, fp, fp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_uint64, fp]
        L.rg_mlp_infer.argtypes = [P, fp, fp, ctypes.c_size_t]
        L.rg_mlp_grad.argtypes = [P, fp, fp, ctypes.c_size_t, fp, fp]
        L.rg_batch_create.argtypes = [ctypes.POINTER(RgConfig), ctypes.c_int, ctypes.POINTER(P)]
        L.rg_batch_destroy.argtypes = [P]
        L.rg_batch_set_bodies.argtypes = [P, ctypes.c_int, dp, dp, dp, dp, dp]
        L.rg_batch_set_state.argtypes = [P, ctypes.c_int, dp, dp, dp, dp]
        L.rg_batch_get_state.argtypes = [P, ctypes.c_int, dp, dp, dp, dp]
        L.rg_batch_step.argtypes = [P, ctypes.c_int, ctypes.POINTER(RgStepStats)]
        L.rg_batch_set_mlp.argtypes = [P, fp, ctypes.c_size_t]
        L.rg_batch_size.argtypes = [P]
        L.rg_batch_member.argtypes = [P, ctypes.c_int]
        L.rg_batch_member.restype = P
        L.rg_batch_last_error.argtypes = [P]
        L.rg_batch_last_error.restype = ctypes.c_char_p
        L.rg_batch_set_schedule.argtypes = [P, ctypes.c_int, ctypes.c_int]
        L.rg_batch_get_schedule.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]
        L.rg_batch_autotune.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), dp]
        L.rg_batch_set_state_all.argtypes = [P, dp, dp, dp, dp]
        L.rg_batch_get_costs.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int)]
        L.rg_batch_get_team_times.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.rg_batch_get_state_all.argtypes = [P, dp, dp, dp, dp]
        _lib = L
    return _lib


def host():
    """Loads librodhost.so (scene generator, mass properties, config
    defaults; no device code)."""
    global _host
    if _host is None:
        _host = bind_scene_lib(ctypes.CDLL(HOST_PATH))
    return _host


def default_config(**kw):
    """rg_config_default() of librodgpu.so with keyword overrides (model
    accepts a name)."""
    return config_from(lib(), **kw)


class RgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS[code] if 0 <= code < len(STATUS) else code}: {msg}")
        self.code = code


class System:
    """One rg_system: device state of N capsules advanced by librodgpu."""

    def __init__(self, cfg, _borrowed=None):
        self._lib = lib()
        self.cfg = cfg
        self.n = cfg.n_bodies
        self._owned = _borrowed is None
        if _borrowed is not None:  # a batch member: the batch owns it
            self._h = ctypes.c_void_p(_borrowed)
            return
        h = ctypes.c_void_p()
        rc = self._lib.rg_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise RgError(rc, "rg_create failed")
        self._h = h

    def _check(self, rc, what):
        if rc != 0:
            msg = self._lib.rg_last_error(self._h)
            raise RgError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self._lib.rg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bodies(self, radius, half_height, mass, inertia, restitution=None):
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (radius, half_height, mass, inertia)]
        rest = None if restitution is None else np.ascontiguousarray(restitution, dtype=np.float64)
        self._keep = args + [rest]
        self._check(self._lib.rg_set_bodies(self._h, *[ptr(a) for a in args], ptr(rest)), "set_bodies")

    def set_state(self, x, q, v, w, f=None, tau=None):
        arr = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, q, v, w, f, tau)]
        self._check(self._lib.rg_set_state(self._h, *[ptr(a) for a in arr]), "set_state")

    def get_state(self):
        n = self.n
        x, v, w, f, t = (np.zeros((n, 3)) for _ in range(5))
        q = np.zeros((n, 4))
        self._check(self._lib.rg_get_state(self._h, ptr(x), ptr(q), ptr(v), ptr(w), ptr(f), ptr(t)), "get_state")
        return {"x": x, "q": q, "v": v, "w": w, "f": f, "tau": t}

    def step(self, nsteps=1):
        st = RgStepStats()
        self._check(self._lib.rg_step(self._h, int(nsteps), ctypes.byref(st)), "step")
        return st.as_dict()

    def detect(self, delta=0.0):
        n = ctypes.c_size_t()
        self._lib.rg_detect(self._h, delta, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        geom = np.zeros((cap, 12))
        shift = np.zeros((cap, 3))
        self._check(self._lib.rg_detect(self._h, delta, ptr(pairs, _i), ptr(geom), ptr(shift), cap,
                                        ctypes.byref(n)), "detect")
        m = n.value
        return pairs[:m], geom[:m], shift[:m]

    def impulses(self):
        n = ctypes.c_size_t()
        self._lib.rg_get_impulses(self._h, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        lam = np.zeros((cap, 3))
        col = np.zeros(cap, np.int32)
        self._check(self._lib.rg_get_impulses(self._h, ptr(pairs, _i), ptr(lam), ptr(col, _i), cap,
                                              ctypes.byref(n)), "impulses")
        m = n.value
        return pairs[:m], lam[:m], col[:m]

    def set_network_export(self, on=True):
        self._check(self._lib.rg_set_network_export(self._h, int(bool(on))), "set_network_export")

    def contact_network(self):
        """(pairs [C,2], rows [C,12]) of the last NSC velocity solve; rows are
        contact point (3), normal (3), phi, lambda_n, lambda_t1, lambda_t2,
        vn_pre, vn_post (the reference's network CSV columns)."""
        n = ctypes.c_size_t()
        self._lib.rg_get_contact_network(self._h, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        rows = np.zeros((cap, 12))
        self._check(self._lib.rg_get_contact_network(self._h, ptr(pairs, _i), ptr(rows), cap, ctypes.byref(n)),
                    "contact_network")
        return pairs[:n.value], rows[:n.value]

    def compute_forces(self):
        f = np.zeros((self.n, 3))
        t = np.zeros((self.n, 3))
        pe = ctypes.c_double()
        self._check(self._lib.rg_compute_forces(self._h, ptr(f), ptr(t), ctypes.byref(pe)), "compute_forces")
        return f, t, pe.value

    STAGES = ["integrate", "detect", "color", "manifolds", "psor", "project", "forces", "nsc_step"]

    def set_profiling(self, on=True):
        self._check(self._lib.rg_set_profiling(self._h, int(on)), "set_profiling")

    def profile(self):
        ms = np.zeros(8)
        cnt = np.zeros(8, np.int64)
        self._check(self._lib.rg_get_profile(self._h, ptr(ms), ptr(cnt, ctypes.c_int64)), "profile")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.STAGES)}

    PHASES = ["free_flight", "detect", "color", "manifolds", "psor", "position_update",
              "proj_detect", "proj_color", "proj_sweeps", "list_rebuild", "small_map_writeback",
              "small_sync"]

    def phase_times(self):
        ms = np.zeros(12)
        self._check(self._lib.rg_get_phase_times(self._h, ptr(ms), 12), "phase_times")
        return {k: float(ms[i]) for i, k in enumerate(self.PHASES)}

    def history(self):
        n = ctypes.c_size_t()
        self._lib.rg_get_history(self._h, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        val = np.zeros((cap, 3))
        fr = np.zeros(cap, np.int64)
        self._check(self._lib.rg_get_history(self._h, ptr(pairs, _i), ptr(val), ptr(fr, ctypes.c_int64),
                                             cap, ctypes.byref(n)), "history")
        m = n.value
        return pairs[:m], val[:m], fr[:m]

    # ---- learned PSOR warm start -------------------------------------------
    MLP_IN, MLP_OUT = 8, 3

    def mlp_param_count(self):
        return int(self._lib.rg_mlp_param_count())

    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self._lib.rg_mlp_set_params(self._h, ptr(p, ctypes.c_float), p.size), "mlp_set_params")

    def mlp_get_params(self):
        p = np.zeros(self.mlp_param_count(), np.float32)
        self._check(self._lib.rg_mlp_get_params(self._h, ptr(p, ctypes.c_float), p.size), "mlp_get_params")
        return p

    def mlp_record(self, enable=True, cap=1 << 20):
        self._check(self._lib.rg_mlp_record(self._h, int(enable), int(cap)), "mlp_record")

    def mlp_records(self):
        n = ctypes.c_size_t()
        self._lib.rg_mlp_records(self._h, None, None, 0, ctypes.byref(n))
        m = n.value
        x = np.zeros((max(m, 1), 8), np.float32)
        y = np.zeros((max(m, 1), 3), np.float32)
        rc = self._lib.rg_mlp_records(self._h, ptr(x, ctypes.c_float), ptr(y, ctypes.c_float), m, ctypes.byref(n))
        self._check(rc, "mlp_records")
        return x[:m], y[:m]

    def mlp_train(self, features, targets, epochs=20, batch=1024, lr=1e-3, seed=0):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(self._lib.rg_mlp_train(self._h, ptr(x, ctypes.c_float), ptr(y, ctypes.c_float), len(x),
                                           int(epochs), int(batch), float(lr), int(seed), ctypes.byref(loss)),
                    "mlp_train")
        return float(loss.value)

    def mlp_grad(self, features, targets):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(self.mlp_param_count(), np.float32)
        loss = ctypes.c_float()
        self._check(self._lib.rg_mlp_grad(self._h, ptr(x, ctypes.c_float), ptr(y, ctypes.c_float), len(x),
                                          ptr(g, ctypes.c_float), ctypes.byref(loss)), "mlp_grad")
        return g, float(loss.value)

    def mlp_infer(self, features):
        x = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros((len(x), 3), np.float32)
        self._check(self._lib.rg_mlp_infer(self._h, ptr(x, ctypes.c_float), ptr(out, ctypes.c_float), len(x)),
                    "mlp_infer")
        return out


class Batch:
    """rg_batch: independent systems of uneven size stepped by one persistent
    launch (CUDA-graph replayed) with an autotuned team schedule."""

    def __init__(self, cfgs):
        self._lib = lib()
        self.cfgs = list(cfgs)
        arr = (RgConfig * len(self.cfgs))(*self.cfgs)
        h = ctypes.c_void_p()
        rc = self._lib.rg_batch_create(arr, len(self.cfgs), ctypes.byref(h))
        if rc != 0:
            raise RgError(rc, "rg_batch_create failed")
        self._h = h
        self._keep = {}

    def __len__(self):
        return len(self.cfgs)

    def _check(self, rc, what):
        if rc != 0:
            msg = self._lib.rg_batch_last_error(self._h)
            raise RgError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def member(self, k):
        """Member k as a System (owned by the batch)."""
        h = self._lib.rg_batch_member(self._h, int(k))
        if not h:
            raise RgError(1, f"no member {k}")
        return System(self.cfgs[k], _borrowed=h)

    def set_bodies(self, k, radius, half_height, mass, inertia, restitution=None):
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (radius, half_height, mass, inertia)]
        rest = None if restitution is None else np.ascontiguousarray(restitution, dtype=np.float64)
        self._keep[k] = args + [rest]
        self._check(self._lib.rg_batch_set_bodies(self._h, int(k), *[ptr(a) for a in args], ptr(rest)),
                    "batch_set_bodies")

    def set_state(self, k, x, q, v, w):
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, q, v, w)]
        self._check(self._lib.rg_batch_set_state(self._h, int(k), *[ptr(a) for a in arr]), "batch_set_state")

    def get_state(self, k):
        n = self.cfgs[k].n_bodies
        x, v, w = (np.zeros((n, 3)) for _ in range(3))
        q = np.zeros((n, 4))
        self._check(self._lib.rg_batch_get_state(self._h, int(k), ptr(x), ptr(q), ptr(v), ptr(w)),
                    "batch_get_state")
        return {"x": x, "q": q, "v": v, "w": w}

    def total_rods(self):
        return sum(c.n_bodies for c in self.cfgs)

    def set_state_all(self, x, q, v, w):
        """All members' states, rods concatenated in member order (pass
        page-locked arrays for full transfer speed)."""
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, q, v, w)]
        self._check(self._lib.rg_batch_set_state_all(self._h, *[ptr(a) for a in arr]), "batch_set_state_all")

    def get_state_all(self, out=None):
        """All members' states as (x[T,3], q[T,4], v[T,3], w[T,3]); out, when
        given, is a tuple of such contiguous float64 arrays to fill."""
        T = self.total_rods()
        if out is None:
            out = (np.zeros((T, 3)), np.zeros((T, 4)), np.zeros((T, 3)), np.zeros((T, 3)))
        self._check(self._lib.rg_batch_get_state_all(self._h, *[ptr(a) for a in out]), "batch_get_state_all")
        return out

    def step(self, nsteps=1, stats=True):
        if not stats:
            self._check(self._lib.rg_batch_step(self._h, int(nsteps), None), "batch_step")
            return None
        st = (RgStepStats * len(self.cfgs))()
        self._check(self._lib.rg_batch_step(self._h, int(nsteps), st), "batch_step")
        return [s.as_dict() for s in st]

    def set_mlp(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self._lib.rg_batch_set_mlp(self._h, ptr(p, ctypes.c_float), p.size), "batch_set_mlp")

    def set_schedule(self, rods_per_block=0, use_graph=True):
        self._check(self._lib.rg_batch_set_schedule(self._h, int(rods_per_block), int(use_graph)),
                    "batch_set_schedule")

    def schedule(self):
        r, g, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.rg_batch_get_schedule(self._h, ctypes.byref(r), ctypes.byref(g), ctypes.byref(t)),
                    "batch_get_schedule")
        return {"rods_per_block": r.value, "grid": g.value, "teams": t.value}

    def costs(self):
        """(measured block-ms per step of each member, its team's blocks)."""
        c = np.zeros(len(self.cfgs))
        t = np.zeros(len(self.cfgs), np.int32)
        self._check(self._lib.rg_batch_get_costs(self._h, ptr(c), ptr(t, ctypes.c_int)), "batch_get_costs")
        return c, t

    def team_times(self):
        """Per team of the last launch: (device ms, blocks, members)."""
        cap = 4096
        ms = np.zeros(cap)
        nb = np.zeros(cap, np.int32)
        nm = np.zeros(cap, np.int32)
        nt = ctypes.c_int()
        self._check(self._lib.rg_batch_get_team_times(self._h, ptr(ms), ptr(nb, ctypes.c_int), ptr(nm, ctypes.c_int),
                                                      cap, ctypes.byref(nt)), "batch_get_team_times")
        k = min(nt.value, cap)
        return ms[:k], nb[:k], nm[:k]

    def autotune(self, candidates=(-1, 0, 1024, 2048, 4096, 8192), trial_steps=10):
        """Times each schedule candidate (rods per block; -1 the balanced
        plan, 0 all single-block) and keeps the fastest: (best, {R: ms})."""
        c = (ctypes.c_int * len(candidates))(*candidates)
        best = ctypes.c_int()
        ms = np.zeros(len(candidates))
        self._check(self._lib.rg_batch_autotune(self._h, c, len(candidates), int(trial_steps), ctypes.byref(best),
                                                ptr(ms)), "batch_autotune")
        return best.value, dict(zip(candidates, ms.tolist()))
