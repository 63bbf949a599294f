"""Oracle parity at the configurations the benchmark times.

The headline batch (the 128 NSC members of the uneven-batch workload, seed 1)
starts from RSA packings without contacts; its rods only meet after some
steps.  So the whole batch is first advanced ADVANCE steps on the GPU, then
fresh systems start from those states with cold warm caches - one GPU System
per member, one fresh Batch of all members, and the FP64 oracle - and are
compared step by step:

  * the largest member (19,928 rods, aspect ratio 40, mu ~0.85), the densest
    aspect-ratio-5 member and the smallest member, 5 steps each: contact
    pairs, shifts and geometry bit-exact; impulses, colours and sweep counts
    per step; states within 1e-10 of the largest magnitude;
  * a fresh Batch of all 128 members (multi-block teams for the large ones)
    against the oracle for its largest and smallest members;
  * the small Hertz-Mindlin workload (N = 1,000, 200 steps, checked every 50);
  * a 1e5-rod cut of the large Hertz-Mindlin workload's rods (L = 1,
    d = 0.02), 2 steps.
"""
import numpy as np
import pytest

import rodgpu
from helpers import packed_scene, rel_err
from oracle import Oracle
from rodgpu import scene

pytestmark = pytest.mark.gpu
TOL = 1e-10
ADVANCE = 100
STEPS = 5


def _load(obj, sc, state):
    obj.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
    obj.set_state(state["x"], state["q"], state["v"], state["w"])
    return obj


def _assert_state(a, b, what):
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < TOL, (what, k, rel_err(a[k], b[k]))


@pytest.fixture(scope="module")
def bench_batch():
    specs = [s for s in scene.batch_members(256, seed=1) if s["model"] == "nsc"]
    items = scene.batch_scenes(specs)
    b = rodgpu.Batch([c for c, _ in items])
    for k, (_, sc) in enumerate(items):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    b.set_schedule(4096, True)
    b.step(ADVANCE, stats=False)
    states = [b.get_state(k) for k in range(len(items))]
    b.close()
    n = np.array([sc["n"] for _, sc in items])
    ar5 = [k for k, s in enumerate(specs) if s["ar"] == 5]
    picks = {"largest": int(np.argmax(n)), "densest_ar5": max(ar5, key=lambda k: items[k][1]["phi"]),
             "smallest": int(np.argmin(n))}
    return items, states, picks


@pytest.fixture(scope="module")
def oracle_runs(bench_batch):
    """Per picked member: the oracle's contacts at the advanced state and its
    impulses, statistics and state after each of STEPS steps."""
    items, states, picks = bench_batch
    out = {}
    for name, k in picks.items():
        cfg, sc = items[k]
        o = _load(Oracle(cfg), sc, states[k])
        rec = {"contacts": o.detect(0.0), "steps": []}
        for _ in range(STEPS):
            st = o.step(1)
            rec["steps"].append((st, o.impulses(), o.get_state()))
        out[name] = rec
    return out


@pytest.mark.parametrize("name", ["largest", "densest_ar5", "smallest"])
def test_bench_member_vs_oracle(bench_batch, oracle_runs, name):
    items, states, picks = bench_batch
    k = picks[name]
    cfg, sc = items[k]
    g = _load(rodgpu.System(cfg), sc, states[k])
    pg, gg, sg = g.detect(0.0)
    po, go, so = oracle_runs[name]["contacts"]
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(sg, so)
    np.testing.assert_array_equal(gg, go)
    if name != "smallest":
        assert len(po) > 0, "the advanced state should hold contacts"
    solved = 0
    for step, (so_, (pio, lo, co), xo) in enumerate(oracle_runs[name]["steps"]):
        st = g.step(1)
        pig, lg, cg = g.impulses()
        np.testing.assert_array_equal(pig, pio)
        np.testing.assert_array_equal(cg, co)
        assert rel_err(lg, lo) < TOL, (step, rel_err(lg, lo))
        assert st["psor_sweeps"] == so_["psor_sweeps"], step
        assert st["contacts"] == so_["contacts"], step
        # profile-CSV columns from device counters (main.cpp:3276-3355)
        assert st["collisions"] == so_["collisions"], step
        for key in ("jn_sum", "jt_sum", "residual"):
            assert abs(st[key] - so_[key]) <= TOL * max(abs(so_[key]), 1e-30), (step, key)
        _assert_state(g.get_state(), xo, (name, step))
        solved += len(pio)
    if name != "smallest":
        assert solved > 0


def test_fresh_batch_vs_oracle(bench_batch, oracle_runs):
    items, states, picks = bench_batch
    b = rodgpu.Batch([c for c, _ in items])
    for k, (_, sc) in enumerate(items):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, states[k]["x"], states[k]["q"], states[k]["v"], states[k]["w"])
    b.set_schedule(4096, True)  # the largest member runs on a team of several blocks
    stats = b.step(STEPS)
    _, team_blocks = b.costs()
    assert team_blocks[picks["largest"]] > 1
    for name in ("largest", "smallest"):
        k = picks[name]
        so_, _, xo = oracle_runs[name]["steps"][-1]
        _assert_state(b.get_state(k), xo, name)
        assert stats[k]["contacts"] == so_["contacts"]
    b.close()


def test_hm_small_200_steps():
    cfg, sc = scene.workload("hm_small", seed=1)
    g = _load(rodgpu.System(cfg), sc, sc)
    o = _load(Oracle(cfg), sc, sc)
    touched = 0
    for chunk in range(4):
        sg = g.step(50)
        so = o.step(50)
        _assert_state(g.get_state(), o.get_state(), ("hm_small", 50 * (chunk + 1)))
        assert sg["contacts"] == so["contacts"]
        assert sg["history_size"] == so["history_size"]
        touched += sg["contacts"]
    assert touched > 0
    pg, vg, fg = g.history()
    po, vo, fo = o.history()
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(fg, fo)
    assert rel_err(vg, vo) < TOL


def test_hm_large_geometry_cut_1e5():
    # rods of the large Hertz-Mindlin workload (L=1, d=0.02) generated at
    # diameter 0.9 d so they overlap and every step has contacts
    sc = packed_scene(100000, L=1.0, d=0.02, phi=0.03, seed=5, squeeze=0.9)
    kw = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0, model="hertz-mindlin", dt=2e-5,
              hm_youngs_modulus=1e6, hm_poisson_ratio=0.3, hm_restitution=0.3, hm_friction=0.5)
    kw.update(scene.pbc_kwargs(sc))
    cfg = rodgpu.default_config(n_bodies=sc["n"], **kw)
    g = _load(rodgpu.System(cfg), sc, sc)
    o = _load(Oracle(cfg), sc, sc)
    pg, gg, _ = g.detect(0.0)
    po, go, _ = o.detect(0.0)
    assert len(po) > 10000
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(gg, go)
    sg = g.step(2)
    so = o.step(2)
    _assert_state(g.get_state(), o.get_state(), "hm_large cut")
    assert sg["contacts"] == so["contacts"]
    assert sg["history_size"] == so["history_size"]
