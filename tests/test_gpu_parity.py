"""GPU parity: librodgpu (through the C ABI) against the FP64 oracle.

Bars:
  * contact pair lists, minimum-image shifts and contact types: bit-exact;
  * contact geometry (closest points, normal, distance): bit-exact (both
    sides evaluate the same FP64 expressions without FMA contraction);
  * forces, torques, impulses and states: relative error <= 1e-10 of the
    array's largest magnitude (FP64; transcendental functions differ by a
    few ulp between CUDA and glibc, nothing else does).
"""
import numpy as np
import pytest

from helpers import make_pair, packed_scene, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def assert_contacts_equal(g, o, delta):
    pg, gg, sg = g.detect(delta)
    po, go, so = o.detect(delta)
    assert len(po) > 0
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(sg, so)
    np.testing.assert_array_equal(gg, go)  # points, normal, distance, surface, type
    return len(po)


@pytest.mark.parametrize("n,d,phi,seed", [(1000, 0.1, 0.10, 1), (3000, 0.05, 0.2, 2), (500, 0.2, 0.15, 3)])
def test_detect_bit_exact_nsc(n, d, phi, seed):
    sc = packed_scene(n, d=d, phi=phi, seed=seed)
    g, o = make_pair(sc, model="nsc")
    assert_contacts_equal(g, o, 0.0)


def test_detect_bit_exact_soft_margin():
    sc = packed_scene(1500, d=0.1, phi=0.1, seed=4, squeeze=0.95)
    g, o = make_pair(sc, model="harmonic")
    assert_contacts_equal(g, o, 0.005)


def test_detect_open_box():
    sc = packed_scene(800, d=0.1, phi=0.1, seed=5)
    g, o = make_pair(sc, model="nsc", pbc_enabled=0)
    assert_contacts_equal(g, o, 0.0)


def test_detect_tiny_periodic_box():
    # box smaller than twice the rod length: every pair is listed
    sc = packed_scene(40, L=1.0, d=0.1, phi=0.02, seed=6, squeeze=0.7)
    g, o = make_pair(sc, model="nsc")
    pg, gg, _ = g.detect(0.0)
    po, go, _ = o.detect(0.0)
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(gg, go)


def test_neighbor_list_overflow_grows():
    sc = packed_scene(1000, d=0.1, phi=0.1, seed=7)
    g, o = make_pair(sc, model="nsc", max_neighbors=2)
    assert_contacts_equal(g, o, 0.0)


@pytest.mark.parametrize("mode", ["smooth", "cundall", "karnopp"])
def test_soft_forces(mode):
    sc = packed_scene(1200, d=0.1, phi=0.1, seed=8, squeeze=0.9)
    g, o = make_pair(sc, model="harmonic", dt=1e-4, soft_friction_mode=mode, soft_damping=0.5,
                     soft_mu_static=0.8 if mode != "cundall" else 0.0)
    for _ in range(3):
        fg, tg, peg = g.compute_forces()
        fo, to, peo = o.compute_forces()
        assert rel_err(fg, fo) < TOL
        assert rel_err(tg, to) < TOL
        assert abs(peg - peo) <= TOL * abs(peo)
    if mode == "cundall":
        pg, vg, frg = g.history()
        po, vo, fro = o.history()
        np.testing.assert_array_equal(pg, po)
        np.testing.assert_array_equal(frg, fro)
        assert rel_err(vg, vo) < TOL


def test_hertz_mindlin_forces_and_history():
    sc = packed_scene(1200, d=0.1, phi=0.1, seed=9, squeeze=0.97)
    g, o = make_pair(sc, model="hertz-mindlin", dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3,
                     hm_restitution=0.5, hm_friction=0.5)
    for _ in range(3):
        fg, tg, peg = g.compute_forces()
        fo, to, peo = o.compute_forces()
        assert rel_err(fg, fo) < TOL
        assert rel_err(tg, to) < TOL
        assert abs(peg - peo) <= TOL * abs(peo)
    pg, vg, frg = g.history()
    po, vo, fro = o.history()
    assert len(po) > 0
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(frg, fro)
    assert rel_err(vg, vo) < TOL


@pytest.mark.parametrize("model", ["hertz-mindlin", "harmonic"])
def test_verlet_steps(model):
    sc = packed_scene(1000, d=0.1, phi=0.1, seed=10, squeeze=0.97)
    kw = dict(dt=1e-4)
    if model == "hertz-mindlin":
        kw.update(hm_youngs_modulus=1e5, hm_poisson_ratio=0.3, hm_restitution=0.5, hm_friction=0.5)
    else:
        kw.update(soft_friction_mode="cundall")
    g, o = make_pair(sc, model=model, **kw)
    for chunk in (1, 4, 10):
        sg = g.step(chunk)
        so = o.step(chunk)
        a, b = g.get_state(), o.get_state()
        for k in ("x", "q", "v", "w"):
            assert rel_err(a[k], b[k]) < TOL, k
        assert sg["contacts"] == so["contacts"]
        assert sg["history_size"] == so["history_size"]
        assert abs(sg["potential_energy"] - so["potential_energy"]) <= 1e-9 * max(1.0, abs(so["potential_energy"]))
    assert_contacts_equal(g, o, 0.0 if model == "hertz-mindlin" else 0.005)


@pytest.mark.parametrize("model", ["hertz-mindlin", "harmonic"])
def test_verlet_list_rebuilds_inside_graph_replays(model):
    """A small skin and fast rods make the neighbour and near lists rebuild
    every few steps while a 30-step call replays its captured step graph, so
    the rebuilds run from the conditional graph nodes; contacts and states
    must still match the oracle."""
    sc = packed_scene(1000, d=0.1, phi=0.1, seed=21, squeeze=0.97, sigma_v=3.0, sigma_w=3.0)
    kw = dict(dt=1e-4, skin=0.002)
    if model == "hertz-mindlin":
        kw.update(hm_youngs_modulus=1e5, hm_poisson_ratio=0.3, hm_restitution=0.5, hm_friction=0.5)
    else:
        kw.update(soft_friction_mode="cundall")
    g, o = make_pair(sc, model=model, **kw)
    for chunk in (1, 30):
        sg = g.step(chunk)
        so = o.step(chunk)
        a, b = g.get_state(), o.get_state()
        for k in ("x", "q", "v", "w"):
            assert rel_err(a[k], b[k]) < TOL, (chunk, k)
        assert sg["contacts"] == so["contacts"]
        assert sg["history_size"] == so["history_size"]
    assert sg["list_rebuilds"] >= 3  # rebuilt inside the replayed graph
    assert_contacts_equal(g, o, 0.0 if model == "hertz-mindlin" else 0.005)


def test_nsc_one_step_impulses_and_colors():
    sc = packed_scene(1500, d=0.1, phi=0.1, seed=11, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=200)
    sg = g.step(1)
    so = o.step(1)
    pg, lg, cg = g.impulses()
    po, lo, co = o.impulses()
    assert len(po) > 0
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(cg, co)
    assert rel_err(lg, lo) < TOL
    assert sg["psor_sweeps"] == so["psor_sweeps"]
    assert sg["colors"] == so["colors"]
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k


def test_nsc_multi_step_with_warm_start():
    sc = packed_scene(2000, d=0.05, phi=0.2, seed=12, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=500)
    for chunk in (1, 2, 3):
        sg = g.step(chunk)
        so = o.step(chunk)
        a, b = g.get_state(), o.get_state()
        for k in ("x", "q", "v", "w"):
            assert rel_err(a[k], b[k]) < TOL, k
        assert sg["psor_sweeps"] == so["psor_sweeps"]
        assert sg["contacts"] == so["contacts"]
    pg, lg, _ = g.impulses()
    po, lo, _ = o.impulses()
    np.testing.assert_array_equal(pg, po)
    assert rel_err(lg, lo) < TOL


@pytest.mark.parametrize("team", [1, 3, 16])
def test_nsc_team_sizes_agree(team):
    # the persistent step gives the oracle's result for any team size
    sc = packed_scene(3000, d=0.05, phi=0.2, seed=14, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=500, team_blocks=team)
    sg = g.step(3)
    so = o.step(3)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k
    assert sg["psor_sweeps"] == so["psor_sweeps"]
    assert sg["contacts"] == so["contacts"]


def test_nsc_open_box_steps():
    sc = packed_scene(1500, d=0.1, phi=0.1, seed=15, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=200, pbc_enabled=0, team_blocks=4)
    g.step(2)
    o.step(2)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k


def test_list_rebuild_keeps_exact_contacts():
    # large velocities force neighbour-list rebuilds within a few steps
    sc = packed_scene(800, d=0.1, phi=0.1, seed=13, squeeze=0.97, sigma_v=20.0, sigma_w=5.0)
    g, o = make_pair(sc, model="hertz-mindlin", dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3,
                     hm_restitution=0.5, hm_friction=0.5, skin=0.01)
    st = g.step(20)
    o.step(20)
    assert st["list_rebuilds"] >= 1
    a, b = g.get_state(), o.get_state()
    assert rel_err(a["x"], b["x"]) < 1e-9
    assert_contacts_equal(g, o, 0.0)


@pytest.mark.parametrize("team", [1, 4])
def test_nsc_long_call_carries_exact_contacts(team):
    # many steps in one call: the velocity-level detection reuses the hit
    # bits of the previous position-level one for rods that neither the
    # projection nor the periodic wrap moved; fast rods cross the box
    sc = packed_scene(1500, d=0.05, phi=0.2, seed=16, squeeze=0.97, sigma_v=3.0, sigma_w=2.0)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=500, team_blocks=team)
    sg = g.step(8)
    so = o.step(8)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k
    assert sg["psor_sweeps"] == so["psor_sweeps"]
    assert sg["contacts"] == so["contacts"]
    assert_contacts_equal(g, o, 0.0)


def test_nsc_team_larger_than_pair_ranges():
    # a team with more blocks than 64-pair words in the near list: the last
    # blocks own no pairs, and must neither clear nor count the last word
    sc = packed_scene(600, d=0.05, phi=0.2, seed=17, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=500, team_blocks=24)
    sg = g.step(6)
    so = o.step(6)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k
    assert sg["psor_sweeps"] == so["psor_sweeps"]
    assert sg["contacts"] == so["contacts"]
    assert_contacts_equal(g, o, 0.0)


def test_nsc_25_step_call_keeps_exact_contacts():
    # 25 steps in one call (carried hit bits, near-list rebuilds inside the
    # launch, a two-block team): the contact sets stay the oracle's
    sc = packed_scene(1200, d=0.05, phi=0.2, seed=18, squeeze=0.97, sigma_v=0.5, sigma_w=0.5)
    g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=500, team_blocks=2)
    sg = g.step(25)
    so = o.step(25)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, k
    assert sg["psor_sweeps"] == so["psor_sweeps"]
    assert sg["contacts"] == so["contacts"]
    assert_contacts_equal(g, o, 0.0)
