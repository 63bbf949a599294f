"""The FP64 oracle pinned to the reference (CPU).

1. Golden fixtures produced by the reference's own physics sources
   (tests/golden/make_golden.py): contact pair lists must match exactly;
   states after NSC / soft / Hertz-Mindlin steps within the FP32 precision of
   the reference, amplified by stiff contacts and the position projection:
   x, q within 5e-5 absolute; v, w within 2e-4 of their largest magnitude;
   NSC impulses within 1e-3 of the largest impulse.
2. The reference's known-answer smoke tests (tests/smoke_test.py), restated
   for capsules.
"""
import os

import numpy as np
import pytest

import known_answers as KA
import rodgpu
from oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(name):
    import make_golden as G  # noqa: F401  (case table)
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    sc = {k: f[k] for k in f.files}
    sc["n"] = len(f["x"])
    sc["lo"] = float(f["lo"])
    sc["side"] = float(f["side"])
    cfg = G.case_config(G.CASES[name], sc)
    o = Oracle(cfg)
    o.set_bodies(f["radius"], f["half_height"], f["mass"], f["inertia"], f["restitution"])
    o.set_state(f["x"], f["q"], f["v"], f["w"])
    return f, o, cfg


@pytest.fixture(scope="module", autouse=True)
def _golden_path():
    import sys
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)


@pytest.mark.parametrize("name", ["detect_nsc", "detect_soft"])
def test_pairs_match_reference(name):
    f, o, cfg = _fixture(name)
    pairs, geom, _ = o.detect(float(f["delta"]))
    assert np.array_equal(pairs, f["pairs"])
    assert np.max(np.abs(geom[:, 9] - f["dist"])) < 1e-6  # reference distances are FP32


@pytest.mark.parametrize("name", ["nsc_1step", "nsc_5steps", "soft_5steps", "hm_5steps", "nsc_tube_5steps",
                                  "soft_tube_5steps"])
def test_steps_match_reference(name):
    f, o, cfg = _fixture(name)
    o.step(int(f["steps"]))
    s = o.get_state()
    for k in ("x", "q"):
        assert np.max(np.abs(s[k] - f[k + "_out"])) < 5e-5, k
    for k in ("v", "w"):
        ref = f[k + "_out"]
        assert np.max(np.abs(s[k] - ref)) < 2e-4 * np.max(np.abs(ref)), k
    if "imp_lam" in f.files:
        # the reference lists wall manifolds (body a against the tube, shown
        # as (a, a)) after the pair manifolds; the oracle reports them apart
        wall = f["imp_pairs"][:, 0] == f["imp_pairs"][:, 1]
        scale = max(np.max(np.abs(f["imp_lam"])), 1e-12)
        pairs, lam, _ = o.impulses()
        assert np.array_equal(pairs, f["imp_pairs"][~wall])
        assert np.max(np.abs(lam - f["imp_lam"][~wall]), initial=0.0) <= 1e-3 * scale + 1e-12
        body, rows, _ = o.wall_contacts()
        assert np.array_equal(body, f["imp_pairs"][wall, 0])
        assert np.max(np.abs(rows[:, 7:10] - f["imp_lam"][wall]), initial=0.0) <= 1e-3 * scale + 1e-12
        if name.startswith("nsc_tube"):
            assert wall.sum() > 10 and (~wall).sum() > 0


def test_known_nsc_elastic_exchange():
    va, vb = KA.nsc_elastic_exchange(Oracle, 0.0)
    assert abs(va) < 1e-3 and abs(vb - 0.1) < 1e-3
    va, vb = KA.nsc_elastic_exchange(Oracle, 0.05)
    assert vb > 0.09 and (va * va + vb * vb) / 0.01 > 0.95


def test_known_spatial_hash_pbc():
    assert KA.spatial_hash_pbc(Oracle) >= 1


def test_known_sphere_capsule_pbc():
    n, _, _ = KA.sphere_capsule_pbc(Oracle, False)
    assert n == 0
    n, vs, vc = KA.sphere_capsule_pbc(Oracle, True)
    assert n >= 1 and vs < 0 < vc


def test_known_hertz_mindlin_repulsion():
    d0, d1, va, vb, ke = KA.hertz_mindlin_repulsion(Oracle)
    assert d1 > d0 and va < 0 < vb and np.isfinite(ke) and ke < 100.0
