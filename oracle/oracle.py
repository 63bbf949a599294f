"""ctypes handles to the parity oracle and the compiled reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg; never by the product.

  Oracle     oracle/_build/librodoracle.so  FP64 restatement (rod_oracle.cpp)
  Reference  oracle/_ref/librodref.so       the reference's own src/physics
                                            sources (FP32, OpenMP) driven by
                                            ref_harness.cpp
Both take the same rg_config (include/rodgpu.h) as librodgpu.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "librodoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "librodref.so")
# The reference source tree: $RG_REFERENCE_TREE, else a checkout named
# "reference" beside this repository.  Absent on machines that only run the
# prebuilt libraries.
REF_TREE = os.environ.get("RG_REFERENCE_TREE") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))

_d = ctypes.c_double
_i = ctypes.c_int32
dp = ctypes.POINTER(_d)


def build(ref=True):
    """Compiles the oracle (and the reference's CPU and CUDA sources, when
    its tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(REF_TREE):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "refcuda", f"REF={REF_TREE}"], check=True)


def _p(a, t=_d):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


_orc = None
_ref = None


def oracle_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build(ref=False)
        L = ctypes.CDLL(ORACLE_LIB)
        P = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(P)]
        L.orc_destroy.argtypes = [P]
        L.orc_set_bodies.argtypes = [P, dp, dp, dp, dp, dp]
        L.orc_set_state.argtypes = [P, dp, dp, dp, dp, dp, dp]
        L.orc_get_state.argtypes = [P, dp, dp, dp, dp, dp, dp]
        L.orc_step.argtypes = [P, ctypes.c_int, ctypes.c_void_p]
        L.orc_detect.argtypes = [P, _d, ctypes.POINTER(_i), dp, dp, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_size_t)]
        L.orc_get_impulses.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.POINTER(_i), ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t)]
        L.orc_compute_forces.argtypes = [P, dp, dp, dp]
        L.orc_get_contact_network.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.c_size_t,
                                              ctypes.POINTER(ctypes.c_size_t)]
        L.orc_get_wall_contacts.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.POINTER(_i), ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_size_t)]
        L.orc_get_history.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.orc_color.argtypes = [P, ctypes.POINTER(_i), ctypes.c_size_t, ctypes.POINTER(_i),
                                ctypes.POINTER(ctypes.c_int)]
        L.orc_kinetic_energy.argtypes = [P]
        L.orc_kinetic_energy.restype = _d
        _orc = L
    return _orc


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            if not os.path.isdir(REF_TREE):
                raise RuntimeError("reference build absent and reference tree not mounted")
            build(ref=True)
        L = ctypes.CDLL(REF_LIB)
        P = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(P), ctypes.c_int, ctypes.c_int]
        L.ref_destroy.argtypes = [P]
        L.ref_set_bodies.argtypes = [P, dp, dp, dp, dp, ctypes.POINTER(_i)]
        L.ref_get_mass.argtypes = [P, dp, dp]
        L.ref_set_state.argtypes = [P, dp, dp, dp, dp]
        L.ref_get_state.argtypes = [P, dp, dp, dp, dp, dp, dp]
        L.ref_step.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), dp]
        L.ref_detect.argtypes = [P, _d, ctypes.c_int, ctypes.POINTER(_i), dp, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_size_t)]
        L.ref_get_impulses.argtypes = [P, ctypes.POINTER(_i), dp, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t)]
        L.ref_threads.restype = ctypes.c_int
        L.ref_compute_forces.argtypes = [P, dp, dp]
        _ref = L
    return _ref


REFCUDA_LIB = os.path.join(HERE, "_ref", "librodref_cuda.so")
_refcuda = None


def refcuda_lib():
    """The reference's FP32 two-pass CUDA broad phase (secondary GPU
    baseline), built for sm_100a by the Makefile's refcuda target."""
    global _refcuda
    if _refcuda is None:
        if not os.path.exists(REFCUDA_LIB):
            raise RuntimeError("reference CUDA broad phase not built (oracle/Makefile refcuda)")
        L = ctypes.CDLL(REFCUDA_LIB)
        L.refcuda_detect.argtypes = [ctypes.c_int, dp, dp, dp, dp, _d, ctypes.c_int, _d, _d, _d,
                                     ctypes.POINTER(_i), ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), dp, dp]
        _refcuda = L
    return _refcuda


def refcuda_detect(sc, margin, box):
    """Pairs (sorted) found by the reference's cudaDetectCapsulePairsTwoPass,
    its stage times (upload, aabb, broadphase, narrowphase, download ms;
    candidates; contacts) and the call's wall time in ms."""
    L = refcuda_lib()
    n = sc["n"]
    arr = [np.ascontiguousarray(sc[k], np.float64) for k in ("x", "q", "radius", "half_height")]
    cap = 64 * n + 16
    pairs = np.zeros((cap, 2), np.int32)
    cnt = ctypes.c_size_t()
    stats = np.zeros(7)
    wall = ctypes.c_double()
    rc = L.refcuda_detect(n, *[_p(a) for a in arr], float(margin), 1, float(box[0]), float(box[1]), float(box[2]),
                          _p(pairs, _i), cap, ctypes.byref(cnt), _p(stats), ctypes.byref(wall))
    assert rc == 0, rc
    return pairs[:min(cnt.value, cap)], stats, wall.value


class Oracle:
    """FP64 restatement; same surface as rodgpu.System."""

    def __init__(self, cfg):
        self.L = oracle_lib()
        self.n = cfg.n_bodies
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = self.L.orc_create(ctypes.addressof(cfg), ctypes.byref(h))
        assert rc == 0, rc
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self.L.orc_destroy(self._h)
            self._h = None

    def set_bodies(self, radius, half_height, mass, inertia, restitution=None):
        a = [np.ascontiguousarray(v, np.float64) for v in (radius, half_height, mass, inertia)]
        r = None if restitution is None else np.ascontiguousarray(restitution, np.float64)
        assert self.L.orc_set_bodies(self._h, *[_p(v) for v in a], _p(r)) == 0

    def set_state(self, x, q, v, w, f=None, tau=None):
        a = [None if v_ is None else np.ascontiguousarray(v_, np.float64) for v_ in (x, q, v, w, f, tau)]
        assert self.L.orc_set_state(self._h, *[_p(v_) for v_ in a]) == 0

    def get_state(self):
        n = self.n
        x, v, w, f, t = (np.zeros((n, 3)) for _ in range(5))
        q = np.zeros((n, 4))
        self.L.orc_get_state(self._h, _p(x), _p(q), _p(v), _p(w), _p(f), _p(t))
        return {"x": x, "q": q, "v": v, "w": w, "f": f, "tau": t}

    def step(self, nsteps=1):
        from rodgpu.abi import RgStepStats  # same struct layout (pure Python, loads nothing)
        st = RgStepStats()
        assert self.L.orc_step(self._h, int(nsteps), ctypes.addressof(st)) == 0
        return st.as_dict()

    def detect(self, delta=0.0):
        n = ctypes.c_size_t()
        self.L.orc_detect(self._h, delta, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        geom = np.zeros((cap, 12))
        shift = np.zeros((cap, 3))
        self.L.orc_detect(self._h, delta, _p(pairs, _i), _p(geom), _p(shift), cap, ctypes.byref(n))
        m = n.value
        return pairs[:m], geom[:m], shift[:m]

    def impulses(self):
        n = ctypes.c_size_t()
        self.L.orc_get_impulses(self._h, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        lam = np.zeros((cap, 3))
        col = np.zeros(cap, np.int32)
        self.L.orc_get_impulses(self._h, _p(pairs, _i), _p(lam), _p(col, _i), cap, ctypes.byref(n))
        m = n.value
        return pairs[:m], lam[:m], col[:m]

    def wall_contacts(self):
        n = ctypes.c_size_t()
        self.L.orc_get_wall_contacts(self._h, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        body = np.zeros(cap, np.int32)
        rows = np.zeros((cap, 10))
        col = np.zeros(cap, np.int32)
        self.L.orc_get_wall_contacts(self._h, _p(body, _i), _p(rows), _p(col, _i), cap, ctypes.byref(n))
        return body[:n.value], rows[:n.value], col[:n.value]

    def contact_network(self):
        n = ctypes.c_size_t()
        self.L.orc_get_contact_network(self._h, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        rows = np.zeros((cap, 12))
        self.L.orc_get_contact_network(self._h, _p(pairs, _i), _p(rows), cap, ctypes.byref(n))
        return pairs[:n.value], rows[:n.value]

    def compute_forces(self):
        f = np.zeros((self.n, 3))
        t = np.zeros((self.n, 3))
        pe = ctypes.c_double()
        self.L.orc_compute_forces(self._h, _p(f), _p(t), ctypes.byref(pe))
        return f, t, pe.value

    def history(self):
        n = ctypes.c_size_t()
        self.L.orc_get_history(self._h, None, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        val = np.zeros((cap, 3))
        fr = np.zeros(cap, np.int64)
        self.L.orc_get_history(self._h, _p(pairs, _i), _p(val), _p(fr, ctypes.c_int64), cap, ctypes.byref(n))
        m = n.value
        return pairs[:m], val[:m], fr[:m]

    def color(self, pairs):
        pairs = np.ascontiguousarray(pairs, np.int32)
        col = np.zeros(len(pairs), np.int32)
        k = ctypes.c_int()
        self.L.orc_color(self._h, _p(pairs, _i), len(pairs), _p(col, _i), ctypes.byref(k))
        return col, k.value

    def kinetic_energy(self):
        return self.L.orc_kinetic_energy(self._h)


class Reference:
    """The reference's own physics sources (FP32) behind ref_harness.cpp."""

    def __init__(self, cfg, threads=0, spatial_hash=True):
        self.L = ref_lib()
        self.n = cfg.n_bodies
        h = ctypes.c_void_p()
        assert self.L.ref_create(ctypes.addressof(cfg), ctypes.byref(h), int(threads), int(spatial_hash)) == 0
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self.L.ref_destroy(self._h)
            self._h = None

    def set_bodies(self, radius, half_height, density, restitution=None, is_static=None):
        a = [np.ascontiguousarray(v, np.float64) for v in (radius, half_height, density)]
        r = None if restitution is None else np.ascontiguousarray(restitution, np.float64)
        s = None if is_static is None else np.ascontiguousarray(is_static, np.int32)
        assert self.L.ref_set_bodies(self._h, *[_p(v) for v in a], _p(r), _p(s, _i)) == 0

    def mass(self):
        m = np.zeros(self.n)
        inertia = np.zeros((self.n, 3))
        self.L.ref_get_mass(self._h, _p(m), _p(inertia))
        return m, inertia

    def set_state(self, x, q, v, w):
        a = [np.ascontiguousarray(v_, np.float64) for v_ in (x, q, v, w)]
        assert self.L.ref_set_state(self._h, *[_p(v_) for v_ in a]) == 0

    def get_state(self):
        n = self.n
        x, v, w, f, t = (np.zeros((n, 3)) for _ in range(5))
        q = np.zeros((n, 4))
        self.L.ref_get_state(self._h, _p(x), _p(q), _p(v), _p(w), _p(f), _p(t))
        return {"x": x, "q": q, "v": v, "w": w, "f": f, "tau": t}

    def step(self, nsteps=1):
        c = ctypes.c_int64()
        r = ctypes.c_double()
        self.L.ref_step(self._h, int(nsteps), ctypes.byref(c), ctypes.byref(r))
        return {"contacts": c.value, "residual": r.value}

    def compute_forces(self):
        f = np.zeros((self.n, 3))
        t = np.zeros((self.n, 3))
        self.L.ref_compute_forces(self._h, _p(f), _p(t))
        return f, t

    def detect(self, delta=0.0, spatial_hash=True):
        n = ctypes.c_size_t()
        self.L.ref_detect(self._h, delta, int(spatial_hash), None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        dist = np.zeros(cap)
        self.L.ref_detect(self._h, delta, int(spatial_hash), _p(pairs, _i), _p(dist), cap, ctypes.byref(n))
        m = n.value
        return pairs[:m], dist[:m]

    def impulses(self):
        n = ctypes.c_size_t()
        self.L.ref_get_impulses(self._h, None, None, 0, ctypes.byref(n))
        cap = max(1, n.value)
        pairs = np.zeros((cap, 2), np.int32)
        lam = np.zeros((cap, 3))
        self.L.ref_get_impulses(self._h, _p(pairs, _i), _p(lam), cap, ctypes.byref(n))
        m = n.value
        return pairs[:m], lam[:m]

    def threads(self):
        return self.L.ref_threads()
