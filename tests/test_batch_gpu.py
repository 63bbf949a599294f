"""Batches of independent systems of uneven size (one persistent launch):
every member's results equal the same system stepped alone, for every
schedule, with and without the CUDA graph."""
import numpy as np
import pytest

import rodgpu
from helpers import packed_scene
from rodgpu import scene

pytestmark = pytest.mark.gpu

# (n, aspect ratio, volume fraction, friction, model)
MEMBERS = [(300, 10, 0.10, 0.1, "nsc"), (2500, 20, 0.10, 0.5, "nsc"), (800, 5, 0.20, 0.9, "nsc"),
           (4000, 20, 0.08, 0.3, "nsc"), (600, 40, 0.05, 0.0, "nsc"), (700, 10, 0.10, 0.5, "hertz-mindlin")]


def _member(k, n, ar, phi, mu, model):
    d = 1.0 / ar
    sc = packed_scene(n, d=d, phi=phi, seed=100 + k, squeeze=0.9)
    cfg = dict(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0, model=model)
    if model == "nsc":
        cfg.update(dt=5e-4, nsc_mu=mu, nsc_velocity_iters=500, nsc_tol=1e-6)
    else:
        cfg.update(dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3, hm_restitution=0.5, hm_friction=mu)
    cfg.update(scene.pbc_kwargs(sc))
    return sc, rodgpu.default_config(n_bodies=sc["n"], **cfg)


@pytest.fixture(scope="module")
def specs():
    return [_member(k, *m) for k, m in enumerate(MEMBERS)]


def _batch(specs):
    b = rodgpu.Batch([c for _, c in specs])
    for k, (sc, _) in enumerate(specs):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    return b


@pytest.fixture(scope="module")
def alone(specs):
    """Each member stepped alone: 2 x 15 steps."""
    out = []
    for sc, cfg in specs:
        g = rodgpu.System(cfg)
        g.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        g.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
        g.step(15)
        r = g.step(15)
        out.append((g.get_state(), r))
    return out


def _check_same(b, alone):
    for k, (st, r) in enumerate(alone):
        got = b.get_state(k)
        for key in ("x", "q", "v", "w"):
            assert np.array_equal(got[key], st[key]), (k, key)


@pytest.mark.parametrize("rods_per_block,graph", [(0, True), (1024, True), (512, False), (-1, True)])
def test_batch_equals_members_alone(specs, alone, rods_per_block, graph):
    b = _batch(specs)
    b.set_schedule(rods_per_block, graph)
    b.step(15)
    stats = b.step(15)
    _check_same(b, alone)
    for k, (st, r) in enumerate(alone):
        assert stats[k]["contacts"] == r["contacts"]
        assert stats[k]["psor_sweeps"] == r["psor_sweeps"]
    sch = b.schedule()
    assert 1 <= sch["grid"] and sch["teams"] >= 1


def test_batch_autotune_keeps_state(specs, alone):
    b = _batch(specs)
    b.step(15)
    before = [b.get_state(k) for k in range(len(specs))]
    best, times = b.autotune(candidates=(-1, 0, 1024, 4096), trial_steps=5)
    assert best in (-1, 0, 1024, 4096) and all(t > 0 for t in times.values())
    for k in range(len(specs)):
        now = b.get_state(k)
        for key in ("x", "q", "v", "w"):
            assert np.array_equal(now[key], before[k][key])
    b.step(15)
    _check_same(b, alone)


def test_batch_member_handle_and_learned_warm_start(specs):
    import mlp_oracle as M
    cfgs = []
    for sc, c in specs[:4]:
        c2 = rodgpu.RgConfig.from_buffer_copy(c)
        c2.nsc_warm_start = rodgpu.WARM["mlp"]
        cfgs.append(c2)
    b = rodgpu.Batch(cfgs)
    for k, (sc, _) in enumerate(specs[:4]):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    with pytest.raises(rodgpu.RgError):
        b.step(1)  # no network yet
    x, y = M.synthetic_records(256, seed=3)
    b.set_mlp(M.init_params(x, y, seed=4))
    stats = b.step(10)
    for r in stats:
        assert r["not_converged"] == 0 and r["max_residual"] < 1e-6
    m = b.member(1)
    pairs, lam, _ = m.impulses()
    assert len(pairs) == stats[1]["contacts"]
    mu = specs[1][1].nsc_mu
    assert np.all(lam[:, 0] >= 0)
    assert np.all(np.hypot(lam[:, 1], lam[:, 2]) <= mu * lam[:, 0] * (1 + 1e-9) + 1e-15)


def test_bulk_state_transfer_matches_members(specs):
    b = _batch(specs)
    b.step(3)
    x, q, v, w = b.get_state_all()
    off = 0
    for k, (sc, _) in enumerate(specs):
        n = sc["n"]
        st = b.get_state(k)
        assert np.array_equal(x[off:off + n], st["x"]) and np.array_equal(q[off:off + n], st["q"])
        assert np.array_equal(v[off:off + n], st["v"]) and np.array_equal(w[off:off + n], st["w"])
        off += n
    # writing the same states back and stepping equals stepping on
    c = _batch(specs)
    c.step(3)
    c.set_state_all(x, q, v, w)
    b.step(4)
    c.step(4)
    for k in range(len(specs)):
        sb, sc_ = b.get_state(k), c.get_state(k)
        for key in ("x", "q", "v", "w"):
            assert np.array_equal(sb[key], sc_[key]), (k, key)
