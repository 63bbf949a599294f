"""Generates the golden fixtures that pin the FP64 oracle to the reference.

Runs the reference's own physics sources (compiled by oracle/Makefile into
oracle/_ref/librodref.so from the reference tree, FP32 + OpenMP, single
thread here so merge orders are deterministic) on small seeded packings and
stores inputs and outputs as .npz next to this script:

  detect_nsc.npz    contact pairs at delta = 0 (NSC activation), spatial hash
  detect_soft.npz   contact pairs at the soft margin delta = 0.005
  nsc_1step.npz     one NSC step (sorted sequential Gauss-Seidel), impulses
  nsc_5steps.npz    five NSC steps
  soft_5steps.npz   five Verlet steps of the soft-penalty model (first seed
                    whose contacts stay 5e-5 clear of the force jump at
                    d = h - delta)
  hm_5steps.npz     five Verlet steps of Hertz-Mindlin on capsules (the
                    harness's FP32 restatement; the reference's HM is
                    sphere-only)
  nsc_tube_5steps.npz, soft_tube_5steps.npz
                    five steps of rods in a cylindrical tube (wall
                    manifolds, spin projection; the soft wall spring)

Usage (in a tree where the reference is mounted):
  python tests/golden/make_golden.py [case ...]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rod-dynamics-3d_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
import rodgpu  # noqa: E402
from helpers import packed_scene, tube_config, tube_scene  # noqa: E402
from rodgpu import scene  # noqa: E402

CASES = {
    "detect_nsc": dict(n=400, d=0.1, phi=0.10, seed=3, delta=0.0, model="nsc"),
    "detect_soft": dict(n=400, d=0.1, phi=0.10, seed=4, delta=0.005, model="harmonic"),
    "nsc_1step": dict(n=300, d=0.1, phi=0.10, seed=5, steps=1, model="nsc",
                      cfg=dict(dt=5e-4, nsc_mu=0.3, nsc_tol=1e-6, nsc_velocity_iters=500, psor_order=1)),
    "nsc_5steps": dict(n=300, d=0.1, phi=0.10, seed=6, steps=5, model="nsc",
                       cfg=dict(dt=5e-4, nsc_mu=0.3, nsc_tol=1e-6, nsc_velocity_iters=500, psor_order=1)),
    "soft_5steps": dict(n=300, d=0.1, phi=0.10, seed=7, steps=5, model="harmonic",
                        cfg=dict(dt=1e-4, soft_delta=0.005, soft_k_scaler=1000.0)),
    "hm_5steps": dict(n=300, d=0.1, phi=0.10, seed=8, steps=5, model="hertz-mindlin",
                      cfg=dict(dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3, hm_restitution=0.5,
                               hm_friction=0.5)),
    # rods in a cylindrical tube (radius 0.3 about +y): wall manifolds and the
    # spin projection of the NSC step, the soft wall spring of the Verlet step
    "nsc_tube_5steps": dict(n=80, tube=True, seed=9, steps=5, model="nsc",
                            cfg=dict(dt=5e-4, nsc_mu=0.3, nsc_tol=1e-6, nsc_velocity_iters=500, psor_order=1)),
    "soft_tube_5steps": dict(n=40, tube=True, seed=10, steps=5, model="harmonic",
                             tube_kw=dict(tilt=0.3, spacing=1.6, overshoot=0.02),
                             cfg=dict(dt=1e-4, soft_delta=0.005, soft_k_scaler=1000.0, soft_damping=0.5)),
}


def case_config(c, sc):
    if c.get("tube"):
        return tube_config(sc, model=c["model"], **c.get("cfg", {}))
    kw = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0, model=c["model"])
    kw.update(scene.pbc_kwargs(sc))
    kw.update(c.get("cfg", {}))
    return rodgpu.default_config(n_bodies=sc["n"], **kw)


def inputs(c):
    if c.get("tube"):
        sc = tube_scene(c["n"], seed=c["seed"], **c.get("tube_kw", {}))
    else:
        sc = packed_scene(c["n"], d=c["d"], phi=c["phi"], seed=c["seed"], squeeze=0.9)
    cfg = case_config(c, sc)
    return sc, cfg


def soft_margin(sc, cfg, steps):
    """Smallest |d - (h - delta)| over the contacts of `steps` oracle steps.
    The soft potential's force jumps from ~0 to 2 k delta at d = h - delta
    (soft_contact.cpp:215-237, log barrier vs quadratic branch), so FP32 and
    FP64 runs that straddle it diverge; fixtures keep clear of it."""
    o = oracle.Oracle(cfg)
    o.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
    o.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
    m = np.inf
    for _ in range(steps + 1):
        _, g, _ = o.detect(cfg.soft_delta)
        if len(g):
            m = min(m, float(np.min(np.abs(g[:, 9] - (g[:, 10] - cfg.soft_delta)))))
        o.step(1)
    return m


def soft_inputs(c, margin=5e-5):
    for seed in range(c["seed"], c["seed"] + 200):
        sc = packed_scene(c["n"], d=c["d"], phi=c["phi"], seed=seed, squeeze=0.9)
        cfg = case_config(c, sc)
        if soft_margin(sc, cfg, c["steps"]) > margin:
            return sc, cfg, seed
    raise RuntimeError("no seed keeps the soft contacts clear of d = h - delta")


def main(names=None):
    oracle.build(ref=True)
    for name, c in CASES.items():
        if names and name not in names:
            continue
        if c["model"] == "harmonic" and "steps" in c and not c.get("tube"):
            sc, cfg, seed = soft_inputs(c)
            print(name, "seed", seed)
        else:
            sc, cfg = inputs(c)
        r = oracle.Reference(cfg, threads=1, spatial_hash=True)
        r.set_bodies(sc["radius"], sc["half_height"], np.ones(sc["n"]), sc["restitution"])
        r.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
        out = dict(x=sc["x"], q=sc["q"], v=sc["v"], w=sc["w"], radius=sc["radius"],
                   half_height=sc["half_height"], restitution=sc["restitution"], lo=sc["lo"], side=sc["side"])
        if c.get("tube"):
            out.update(box_min=np.array(sc["box_min"]), box_max=np.array(sc["box_max"]), tube=sc["tube"])
        m, inertia = r.mass()
        out.update(mass=m, inertia=inertia)
        if name.startswith("detect"):
            pairs, dist = r.detect(c["delta"], spatial_hash=True)
            order = np.lexsort((pairs[:, 1], pairs[:, 0]))
            out.update(pairs=pairs[order], dist=dist[order], delta=c["delta"])
        else:
            st = r.step(c["steps"])
            s = r.get_state()
            out.update(x_out=s["x"], q_out=s["q"], v_out=s["v"], w_out=s["w"], steps=c["steps"],
                       contacts=st["contacts"], residual=st["residual"])
            if c["model"] == "nsc":
                pairs, lam = r.impulses()
                out.update(imp_pairs=pairs, imp_lam=lam)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: np.shape(v) for k, v in out.items() if k in ("pairs", "x_out", "imp_lam")})


if __name__ == "__main__":
    main(sys.argv[1:])  # optional case names (default: every case)
