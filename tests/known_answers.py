"""Known-answer cases restated from the reference's own smoke tests
(tests/smoke_test.py) for capsules (a sphere is a capsule of half height 0
with sphere mass properties).  Each case takes a factory cls(cfg) that is
either rodgpu.System or the oracle, so the same checks run on both."""
import math

import numpy as np

import rodgpu


def capsule_props(r, h, rho):
    m = rho * math.pi * r * r * 2.0 * h
    L = 2.0 * h
    ixx = m * (3.0 * r * r + L * L) / 12.0
    return m, np.array([ixx, m * r * r / 2.0, ixx])


def sphere_props(r, rho):
    m = rho * 4.0 / 3.0 * math.pi * r ** 3
    i = 0.4 * m * r * r
    return m, np.array([i, i, i])


def _load(cls, cfg, bodies, x, q=None, v=None):
    n = len(bodies)
    s = cls(cfg)
    r = np.array([b[0] for b in bodies], float)
    h = np.array([b[1] for b in bodies], float)
    m = np.array([b[2] for b in bodies], float)
    I = np.array([b[3] for b in bodies], float)
    e = np.array([b[4] for b in bodies], float)
    s.set_bodies(r, h, m, I, e)
    q = np.tile([1.0, 0, 0, 0], (n, 1)) if q is None else np.asarray(q, float)
    v = np.zeros((n, 3)) if v is None else np.asarray(v, float)
    s.set_state(np.asarray(x, float), q, v, np.zeros((n, 3)))
    return s


def nsc_elastic_exchange(cls, cfm):
    """smoke_test.py:165-204: crossed thin rods, e=1, mu=0: equal masses
    exchange velocities (exact at cfm=0, small loss at cfm=0.05)."""
    c = math.sqrt(0.5)
    m, I = capsule_props(0.01, 0.5, 1000.0)
    cfg = rodgpu.default_config(n_bodies=2, model="nsc", dt=1e-3, gravity=(0, 0, 0), lin_damp=0.0, ang_damp=0.0,
                                nsc_mu=0.0, nsc_velocity_iters=200, nsc_beta=0.0, nsc_cfm=cfm, nsc_omega=1.0)
    body = (0.01, 0.5, m, I, 1.0)
    s = _load(cls, cfg, [body, body], [[-0.06, 0, 0], [0.06, 0, 0]], q=[[1, 0, 0, 0], [c, c, 0, 0]],
              v=[[0.1, 0, 0], [0, 0, 0]])
    s.step(3000)
    v = s.get_state()["v"]
    return v[0, 0], v[1, 0]


def spatial_hash_pbc(cls):
    """smoke_test.py:207-233: a capsule pair overlapping only through the
    periodic boundary is found."""
    m, I = capsule_props(0.05, 0.2, 1000.0)
    cfg = rodgpu.default_config(n_bodies=2, model="harmonic", dt=1e-4, gravity=(0, 0, 0), pbc_enabled=1,
                                pbc_min=(-0.5, -0.5, -0.5), pbc_max=(0.5, 0.5, 0.5))
    body = (0.05, 0.2, m, I, 0.2)
    s = _load(cls, cfg, [body, body], [[0.46, 0, 0], [-0.46, 0, 0]])
    s.step(5)
    pairs, geom, shift = s.detect(cfg.soft_delta)
    return len(pairs)


def sphere_capsule_pbc(cls, pbc):
    """smoke_test.py:129-162: a sphere-capsule pair overlapping only through
    the boundary is pushed apart (sphere -x, capsule +x); none without PBC."""
    ms, Is = sphere_props(0.1, 1000.0)
    mc, Ic = capsule_props(0.05, 0.2, 1000.0)
    kw = dict(pbc_enabled=1, pbc_min=(-0.5, -0.5, -0.5), pbc_max=(0.5, 0.5, 0.5)) if pbc else {}
    cfg = rodgpu.default_config(n_bodies=2, model="harmonic", dt=1e-4, gravity=(0, 0, 0), **kw)
    c = math.sqrt(0.5)  # capsule axis along x, so it reaches across the boundary
    s = _load(cls, cfg, [(0.1, 0.0, ms, Is, 0.2), (0.05, 0.2, mc, Ic, 0.2)], [[0.45, 0, 0], [-0.47, 0, 0]],
              q=[[1, 0, 0, 0], [c, 0, 0, -c]])
    s.step(50)
    pairs, _, _ = s.detect(cfg.soft_delta)
    v = s.get_state()["v"]
    return len(pairs), v[0, 0], v[1, 0]


def hertz_mindlin_repulsion(cls):
    """smoke_test.py:73-102: two overlapping bodies separate with bounded KE
    (the reference uses spheres; here two short parallel capsules, since a
    zero-length segment has no closest point in closestPointsSegmentSegment,
    contact_detector.cpp:978-1035, in the reference either)."""
    m, I = capsule_props(0.1, 0.05, 2500.0)
    cfg = rodgpu.default_config(n_bodies=2, model="hertz-mindlin", dt=1e-5, gravity=(0, 0, 0), lin_damp=0.0,
                                ang_damp=0.0, hm_youngs_modulus=1e7, hm_poisson_ratio=0.25, hm_restitution=0.5,
                                hm_friction=0.3, hm_enable_tangential=1, hm_enable_rolling=0)
    body = (0.1, 0.05, m, I, 0.5)
    s = _load(cls, cfg, [body, body], [[-0.09, 0, 0], [0.09, 0, 0]])
    x0 = s.get_state()["x"]
    s.step(2000)
    st = s.get_state()
    d0 = x0[1, 0] - x0[0, 0]
    d1 = st["x"][1, 0] - st["x"][0, 0]
    ke = 0.5 * m * float((st["v"] ** 2).sum())
    return d0, d1, st["v"][0, 0], st["v"][1, 0], ke
