"""Cylinder walls (the reptation tube): device against the FP64 oracle.

NSC: wall manifolds for the capsules' end points and centre
(collideCapsuleInsideCylinder, src/physics/collision.cpp:197-241, added after
the pair manifolds, src/app/main.cpp:4431-4447), PSOR over pairs and walls,
spin about the rod axis projected out after the position update
(:4486-4494).  Soft model: the wall spring at both force evaluations
(:4661-4690, :4756-4787).  The oracle itself is pinned to the reference's
own sources on the same kind of scene (tests/golden/*tube*).

Bars as in test_gpu_parity: states, impulses and impulse sums within 1e-10 of
the largest magnitude; contact and impact counts, sweep counts and the
(pair) impulse list exact.
"""
import numpy as np
import pytest

import rodgpu
from helpers import rel_err, tube_config, tube_scene
from oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _pair(sc, **kw):
    cfg = tube_config(sc, **kw)
    g = rodgpu.System(cfg)
    o = Oracle(cfg)
    for s in (g, o):
        s.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        s.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
    return g, o


@pytest.mark.parametrize("n,team_blocks", [(80, 1), (400, 3)])
def test_nsc_tube_walls(n, team_blocks):
    sc = tube_scene(n, seed=9 + n)
    g, o = _pair(sc, model="nsc", dt=5e-4, nsc_mu=0.3, nsc_tol=1e-6, nsc_velocity_iters=500,
                 team_blocks=team_blocks)
    walls = 0
    for step in range(5):
        sg = g.step(1)
        so = o.step(1)
        body, _, _ = o.wall_contacts()
        walls += len(body)
        assert sg["contacts"] == so["contacts"], step
        assert sg["collisions"] == so["collisions"], step
        assert sg["psor_sweeps"] == so["psor_sweeps"], step
        for key in ("jn_sum", "jt_sum", "residual"):
            assert abs(sg[key] - so[key]) <= TOL * max(abs(so[key]), 1e-30), (step, key)
        pg, lg, cg = g.impulses()
        po, lo, co = o.impulses()
        np.testing.assert_array_equal(pg, po)
        np.testing.assert_array_equal(cg, co)
        assert rel_err(lg, lo) < TOL
        a, b = g.get_state(), o.get_state()
        for k in ("x", "q", "v", "w"):
            assert rel_err(a[k], b[k]) < TOL, (step, k)
    assert walls > 5 * n // 4  # the tube is in play every step
    if n > 300:
        assert sg["contacts"] > 256  # the multi-block (team) solve ran


def test_nsc_tube_spin_projection():
    """Inside the tube no rod keeps spin about its own axis after the position
    update (position stabilization, which rotates rods after the projection,
    is off here so the update is the last thing to touch w and q)."""
    sc = tube_scene(60, seed=3, sigma_w=5.0)
    g, _ = _pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=200, nsc_position_stabilization=0)
    g.step(3)
    st = g.get_state()
    w_, a, b, c = st["q"].T
    u = np.stack([2 * (a * b - w_ * c), 1 - 2 * (a * a + c * c), 2 * (b * c + w_ * a)], 1)
    spin = np.abs(np.sum(st["w"] * u, axis=1))
    assert np.max(spin) < 1e-12 * max(1.0, np.max(np.abs(st["w"])))


def test_soft_tube_wall_spring():
    sc = tube_scene(40, seed=10, tilt=0.3, spacing=1.6, overshoot=0.02)
    g, o = _pair(sc, model="harmonic", dt=1e-4, soft_delta=0.005, soft_k_scaler=1000.0, soft_damping=0.5)
    fg, _, _ = g.compute_forces()
    fo, _, _ = o.compute_forces()
    assert np.sum(np.linalg.norm(fo, axis=1) > 0) == 40  # every rod is pressed by the wall
    assert rel_err(fg, fo) < TOL
    for chunk in (1, 4):
        g.step(chunk)
        o.step(chunk)
        a, b = g.get_state(), o.get_state()
        for k in ("x", "q", "v", "w"):
            assert rel_err(a[k], b[k]) < TOL, k
