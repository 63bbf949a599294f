"""Failure detection without a GPU fault.

* A team barrier of the persistent NSC step is made to wait for a block that
  never arrives (the rg_config test hook test_absent_blocks).  Its wait is
  the ordinary bounded one, given a short limit (spin_limit), so the call
  must come back promptly with RG_ERR_TIMEOUT, every block having returned,
  the state put back to where the call started, and the CUDA context still
  usable by the next system.
* A NaN in an uploaded state is refused (RG_ERR_NONFINITE) before it reaches
  the device state: on the host for rg_set_state, by a check kernel ahead of
  the scatter for the bulk batch upload.
"""
import time

import numpy as np
import pytest

import rodgpu
from helpers import make_pair, packed_scene, rel_err

pytestmark = pytest.mark.gpu

RG_ERR_NONFINITE = 4
RG_ERR_TIMEOUT = 7


@pytest.mark.parametrize("team_blocks", [1, 3])
def test_barrier_wait_runs_out_and_call_returns_timeout(team_blocks):
    sc = packed_scene(800, d=0.1, phi=0.1, seed=41, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4, team_blocks=team_blocks, spin_limit=20000,
                     test_absent_blocks=1)
    before = g.get_state()
    t0 = time.perf_counter()
    with pytest.raises(rodgpu.RgError) as ei:
        g.step(3)
    dt = time.perf_counter() - t0
    assert ei.value.code == RG_ERR_TIMEOUT
    assert dt < 10.0, dt  # the wait gave up after ~2e4 polls, not a hang
    after = g.get_state()
    for k in ("x", "q", "v", "w"):  # the call's starting state was put back
        np.testing.assert_array_equal(after[k], before[k])
    # the context is still usable: a fresh system steps and matches the oracle
    g2, _ = make_pair(sc, model="nsc", dt=5e-4, team_blocks=team_blocks)
    g2.step(2)
    o.step(2)
    a, b = g2.get_state(), o.get_state()
    for k in ("x", "q", "v", "w"):
        assert rel_err(a[k], b[k]) < 1e-10, k


def test_nonfinite_state_is_refused_on_upload():
    sc = packed_scene(600, d=0.1, phi=0.1, seed=42, squeeze=0.97)
    g, o = make_pair(sc, model="nsc", dt=5e-4)
    x = sc["x"].copy()
    x[17, 1] = np.nan
    with pytest.raises(rodgpu.RgError) as ei:
        g.set_state(x, sc["q"], sc["v"], sc["w"])
    assert ei.value.code == RG_ERR_NONFINITE
    w = sc["w"].copy()
    w[3, 0] = np.inf
    with pytest.raises(rodgpu.RgError) as ei:
        g.set_state(sc["x"], sc["q"], sc["v"], w)
    assert ei.value.code == RG_ERR_NONFINITE
    st = g.get_state()  # unchanged: the refused uploads never reached the device
    np.testing.assert_array_equal(st["x"], sc["x"])
    g.step(2)
    o.step(2)
    assert rel_err(g.get_state()["v"], o.get_state()["v"]) < 1e-10


def test_nonfinite_bulk_upload_is_refused():
    scs = [packed_scene(n, d=0.1, phi=0.1, seed=43 + n, squeeze=0.97) for n in (300, 500)]
    cfgs = []
    for sc in scs:
        g, _ = make_pair(sc, model="nsc", dt=5e-4)
        cfgs.append(g.cfg)
    b = rodgpu.Batch(cfgs)
    for k, sc in enumerate(scs):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    x, q, v, w = b.get_state_all()
    v_bad = v.copy()
    v_bad[len(v) - 5, 2] = np.nan
    with pytest.raises(rodgpu.RgError) as ei:
        b.set_state_all(x, q, v_bad, w)
    assert ei.value.code == RG_ERR_NONFINITE
    x2, q2, v2, w2 = b.get_state_all()
    np.testing.assert_array_equal(v2, v)  # no member's state changed
    np.testing.assert_array_equal(x2, x)
    b.close()
