"""Shared helpers for the parity tests (seeded scenes, comparisons)."""
import numpy as np

import rodgpu
from rodgpu import scene
from oracle import Oracle


def packed_scene(n, L=1.0, d=0.1, phi=0.1, seed=1, squeeze=0.8, sigma_v=0.1, sigma_w=0.1):
    """RSA packing generated with diameter squeeze*d, used with diameter d,
    so the rods overlap and contacts exist at every activation margin."""
    sc = scene.make_rods(n, L, squeeze * d, side=scene.box_side(n, L, d, phi), seed=seed,
                         sigma_v=sigma_v, sigma_w=sigma_w)
    m = sc["n"]
    sc["radius"] = np.full(m, 0.5 * d)
    sc["d"] = d
    dens = np.ones(m)
    mass = np.zeros(m)
    inertia = np.zeros((m, 3))
    rodgpu.host().rg_capsule_mass(m, rodgpu.ptr(sc["radius"]), rodgpu.ptr(sc["half_height"]),
                                  rodgpu.ptr(dens), rodgpu.ptr(mass), rodgpu.ptr(inertia))
    sc["mass"], sc["inertia"] = mass, inertia
    return sc


def make_pair(sc, **cfg_kw):
    """(gpu System, Oracle) loaded with the same bodies and state."""
    kw = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
    kw.update(scene.pbc_kwargs(sc))
    kw.update(cfg_kw)
    cfg = rodgpu.default_config(n_bodies=sc["n"], **kw)
    g = rodgpu.System(cfg)
    o = Oracle(cfg)
    for s in (g, o):
        s.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        s.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
    return g, o


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b)) / scale) if a.size else 0.0
