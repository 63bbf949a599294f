"""Seeded synthetic rod packings and the five benchmark workloads.

The packings come from the host C++ generator (host/scene_gen.cpp): random
sequential addition in a periodic cube with overlap rejection, isotropic
axes, Gaussian velocities.  Box sides follow the capsule volume
V = pi r^2 L + 4/3 pi r^3 used by the reference's broad-phase benchmark
(src/tools/benchmark_broadphase.cpp:104-106).

Workloads (rod counts and physics as stated; values the description leaves
open are fixed here):
  hm_small    N=1000,  L=1, d=0.1,  phi=0.10, Hertz-Mindlin E=1e5 nu=0.3 e=0.5
              mu=0.5, dt=1e-4, 1000 steps
  nsc_dense   N=20000, L=1, d=0.05, phi=0.20, PSOR mu=0.3, omega=1, tol 1e-6,
              500 sweeps max, dt=5e-4, 500 steps, no gravity
  nsc_large   N=50000, same rods, mu ~ U[0.1, 0.8] per run
  hm_large    N=1e6,   L=1, d=0.02, phi=0.15, Hertz-Mindlin E=1e6 nu=0.3 e=0.3
              mu=0.5, dt=2e-5, 100 steps
Damping is zero and gravity is off in every workload.
"""
import math

import numpy as np

from .abi import config_from, ptr


def _gen(gen):
    """The library that generates scenes: librodhost.so unless the caller
    passes another library built from the same host sources."""
    if gen is not None:
        return gen
    from . import host
    return host()


def capsule_volume(L, d):
    r = 0.5 * d
    return math.pi * r * r * L + 4.0 / 3.0 * math.pi * r ** 3


def box_side(n, L, d, phi):
    return (n * capsule_volume(L, d) / phi) ** (1.0 / 3.0)


def make_rods(n, L, d, phi=None, side=None, seed=1, sigma_v=0.1, sigma_w=0.1, density=1.0,
              restitution=0.2, max_attempts=2000, gen=None):
    """RSA packing of n rods; returns a dict of body and state arrays.

    'placed' may be below n when the packing jams; arrays are trimmed to it.
    """
    if side is None:
        side = box_side(n, L, d, phi)
    lo = -0.5 * side
    H = _gen(gen)
    x = np.zeros((n, 3))
    q = np.zeros((n, 4))
    placed = H.rg_scene_rsa(int(n), float(L), float(d), float(lo), float(side), int(seed),
                            int(max_attempts), ptr(x), ptr(q))
    m = placed
    x, q = x[:m].copy(), q[:m].copy()
    v = np.zeros((m, 3))
    w = np.zeros((m, 3))
    H.rg_scene_velocities(int(m), float(sigma_v), float(sigma_w), int(seed), ptr(v), ptr(w))
    radius = np.full(m, 0.5 * d)
    half = np.full(m, 0.5 * L)
    dens = np.full(m, float(density))
    mass = np.zeros(m)
    inertia = np.zeros((m, 3))
    H.rg_capsule_mass(int(m), ptr(radius), ptr(half), ptr(dens), ptr(mass), ptr(inertia))
    phi_ach = m * capsule_volume(L, d) / side ** 3
    return {"n": m, "requested": n, "L": L, "d": d, "side": side, "lo": lo, "phi": phi_ach,
            "radius": radius, "half_height": half, "mass": mass, "inertia": inertia,
            "restitution": np.full(m, float(restitution)), "x": x, "q": q, "v": v, "w": w}


def make_rods_device(n, L, d, phi=None, side=None, seed=1, sigma_v=0.1, sigma_w=0.1, density=1.0,
                     restitution=0.2, max_attempts=2000):
    """make_rods with the positions and axes drawn by the device generator
    (rg_scene_rsa_device: parallel random sequential addition); velocities
    and mass properties as make_rods.  For packings too large for the host
    loop."""
    import ctypes
    from . import lib
    if side is None:
        side = box_side(n, L, d, phi)
    lo = -0.5 * side
    x = np.zeros((n, 3))
    q = np.zeros((n, 4))
    placed = ctypes.c_int()
    rc = lib().rg_scene_rsa_device(int(n), float(L), float(d), float(lo), float(side), int(seed),
                                   int(max_attempts), ptr(x), ptr(q), ctypes.byref(placed))
    if rc != 0:
        raise RuntimeError(f"rg_scene_rsa_device failed with status {rc}")
    m = placed.value
    H = _gen(None)
    v = np.zeros((m, 3))
    w = np.zeros((m, 3))
    H.rg_scene_velocities(int(m), float(sigma_v), float(sigma_w), int(seed), ptr(v), ptr(w))
    radius = np.full(m, 0.5 * d)
    half = np.full(m, 0.5 * L)
    mass = np.zeros(m)
    inertia = np.zeros((m, 3))
    H.rg_capsule_mass(int(m), ptr(radius), ptr(half), ptr(np.full(m, float(density))), ptr(mass), ptr(inertia))
    return {"n": m, "requested": n, "L": L, "d": d, "side": side, "lo": lo,
            "phi": m * capsule_volume(L, d) / side ** 3, "radius": radius, "half_height": half, "mass": mass,
            "inertia": inertia, "restitution": np.full(m, float(restitution)), "x": x[:m].copy(),
            "q": q[:m].copy(), "v": v, "w": w}


def morton_order(sc, bits=10):
    """The scene with its rods renumbered along a Morton (Z-order) curve of
    their centres in the box (2^bits cells per axis).  Rods that touch get
    nearby indices, so the device's gathers of neighbour records share cache
    lines; the physics is the same system, its contact lists come out in
    the new numbering."""
    lo, side = sc["lo"], sc["side"]
    g = np.clip(((sc["x"] - lo) / side * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    key = np.zeros(len(g), np.int64)
    for b in range(bits):
        for k in range(3):
            key |= ((g[:, k] >> b) & 1) << (3 * b + k)
    order = np.argsort(key, kind="stable")
    out = dict(sc)
    for k in ("radius", "half_height", "mass", "inertia", "restitution", "x", "q", "v", "w"):
        out[k] = np.ascontiguousarray(sc[k][order])
    return out


def pbc_kwargs(scene):
    lo, side = scene["lo"], scene["side"]
    return {"pbc_enabled": 1, "pbc_min": (lo, lo, lo), "pbc_max": (lo + side, lo + side, lo + side)}


WORKLOADS = {
    "hm_small": dict(n=1000, L=1.0, d=0.1, phi=0.10, steps=1000,
                     cfg=dict(model="hertz-mindlin", dt=1e-4, hm_youngs_modulus=1e5,
                              hm_poisson_ratio=0.3, hm_restitution=0.5, hm_friction=0.5)),
    "nsc_dense": dict(n=20000, L=1.0, d=0.05, phi=0.20, steps=500,
                      cfg=dict(model="nsc", dt=5e-4, nsc_mu=0.3, nsc_omega=1.0, nsc_tol=1e-6,
                               nsc_velocity_iters=500)),
    "nsc_large": dict(n=50000, L=1.0, d=0.05, phi=0.20, steps=200,
                      cfg=dict(model="nsc", dt=5e-4, nsc_mu=0.3, nsc_omega=1.0, nsc_tol=1e-6,
                               nsc_velocity_iters=500)),
    "hm_large": dict(n=1000000, L=1.0, d=0.02, phi=0.15, steps=100,
                     cfg=dict(model="hertz-mindlin", dt=2e-5, hm_youngs_modulus=1e6,
                              hm_poisson_ratio=0.3, hm_restitution=0.3, hm_friction=0.5)),
}


def workload(name, n=None, seed=1, gen=None, **overrides):
    """(config, scene) for a named workload; n overrides the rod count."""
    w = WORKLOADS[name]
    nn = w["n"] if n is None else n
    sc = make_rods(nn, w["L"], w["d"], phi=w["phi"], seed=seed, gen=gen)
    kw = dict(w["cfg"])
    kw.update(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
    kw.update(pbc_kwargs(sc))
    kw.update(overrides)
    cfg = config_from(_gen(gen), n_bodies=sc["n"], **kw)
    return cfg, sc


def config_dict(cfg):
    """rg_config as a plain dict (for the oracle and for fixtures)."""
    out = {}
    for k, _ in type(cfg)._fields_:
        v = getattr(cfg, k)
        if hasattr(v, "__len__"):
            v = list(v)
        out[k] = v
    return out


# Isotropic RSA jams near phi * (L/d) ~ 2.4 and slows down well before;
# batch members are capped at phi <= 1.6 / aspect ratio so every packing is
# placed in full within seconds.
def rsa_phi_max(ar):
    return 1.6 / ar


def batch_members(n_systems=256, seed=7, n_lo=500, n_hi=20000, ars=(5, 10, 20, 40), phi_lo=0.05,
                  phi_hi=0.25, models=("hertz-mindlin", "nsc")):
    """Member specs of the uneven-batch workload: N log-uniform in
    [n_lo, n_hi], aspect ratio from `ars` (L=1, d=1/AR), phi ~ U[phi_lo,
    phi_hi] capped at the RSA limit, mu ~ U[0, 1]; models alternate."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_systems):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        ar = int(ars[rng.integers(len(ars))])
        phi = float(min(rng.uniform(phi_lo, phi_hi), rsa_phi_max(ar)))
        mu = float(rng.uniform(0.0, 1.0))
        out.append(dict(n=n, ar=ar, phi=phi, mu=mu, model=models[k % len(models)], seed=seed * 1000 + k))
    return out


def batch_scenes(specs, threads=None, warm="cache", gen=None):
    """(config, scene) of every member, generated on host threads (the
    generator releases the interpreter lock)."""
    import concurrent.futures as cf
    import os
    gen = _gen(gen)
    with cf.ThreadPoolExecutor(threads or os.cpu_count() or 4) as ex:
        return list(ex.map(lambda s: batch_member_scene(s, warm, gen), specs))


def batch_member_scene(spec, warm="cache", gen=None):
    """(config, scene) of one batch member: NSC dt=5e-4, tol 1e-6, 500
    sweeps; Hertz-Mindlin E=1e5, nu=0.3, e=0.5, dt=1e-4."""
    gen = _gen(gen)
    d = 1.0 / spec["ar"]
    sc = make_rods(spec["n"], 1.0, d, phi=spec["phi"], seed=spec["seed"], max_attempts=20000, gen=gen)
    kw = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
    if spec["model"] == "nsc":
        kw.update(model="nsc", dt=5e-4, nsc_mu=spec["mu"], nsc_omega=1.0, nsc_tol=1e-6, nsc_velocity_iters=500,
                  nsc_warm_start=warm)
    else:
        kw.update(model="hertz-mindlin", dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3,
                  hm_restitution=0.5, hm_friction=spec["mu"])
    kw.update(pbc_kwargs(sc))
    return config_from(gen, n_bodies=sc["n"], **kw), sc
