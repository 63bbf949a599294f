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


def tube_scene(n, L=1.0, d=0.1, radius=0.3, seed=1, tilt=0.7, sigma_v=0.5, sigma_w=1.0, spacing=None,
               overshoot=0.0):
    """Rods in a tube of the given radius along +y (periodic box, long in y):
    centres within the tube, axes tilted up to `tilt` radians from y, so
    rods touch the wall and each other from the first step.  With `spacing`
    the centres sit on a lattice along y (no rod-rod contacts when spacing >
    L); with `overshoot` > 0 every centre lies up to that far beyond the
    radius at which the capsule touches the wall (radius - d/2)."""
    rng = np.random.default_rng(seed)
    ly = 0.45 * n if spacing is None else spacing * n
    if overshoot > 0:
        r_c = (radius - 0.5 * d) + overshoot * rng.uniform(0.2, 1.0, n)
    else:
        r_c = (radius - 0.5 * d) * np.sqrt(rng.uniform(0.0, 1.0, n))
    ang = rng.uniform(0.0, 2 * np.pi, n)
    y = rng.uniform(0.0, ly, n) if spacing is None else (np.arange(n) + 0.5) * spacing
    x = np.stack([r_c * np.cos(ang), y, r_c * np.sin(ang)], 1)
    th = rng.uniform(0.0, tilt, n)
    az = rng.uniform(0.0, 2 * np.pi, n)
    # quaternion turning +y by th about the horizontal axis (cos az, 0, sin az)
    s = np.sin(0.5 * th)
    q = np.stack([np.cos(0.5 * th), s * np.cos(az), np.zeros(n), s * np.sin(az)], 1)
    radius_a = np.full(n, 0.5 * d)
    half = np.full(n, 0.5 * L)
    mass = np.zeros(n)
    inertia = np.zeros((n, 3))
    rodgpu.host().rg_capsule_mass(n, rodgpu.ptr(radius_a), rodgpu.ptr(half), rodgpu.ptr(np.ones(n)),
                                  rodgpu.ptr(mass), rodgpu.ptr(inertia))
    return {"n": n, "x": x, "q": q, "v": rng.normal(0.0, sigma_v, (n, 3)), "w": rng.normal(0.0, sigma_w, (n, 3)),
            "radius": radius_a, "half_height": half, "mass": mass, "inertia": inertia,
            "restitution": np.full(n, 0.2), "lo": -2.0, "side": ly + 4.0, "tube": radius,
            "box_min": (-2.0, 0.0, -2.0), "box_max": (2.0, ly, 2.0)}


def tube_config(sc, **cfg_kw):
    kw = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0, pbc_enabled=1, pbc_min=tuple(sc["box_min"]),
              pbc_max=tuple(sc["box_max"]), cylinder_enabled=1, cylinder_radius=float(sc["tube"]),
              cylinder_axis=(0.0, 1.0, 0.0))
    kw.update(cfg_kw)
    return rodgpu.default_config(n_bodies=sc["n"], **kw)
