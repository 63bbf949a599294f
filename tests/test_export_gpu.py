"""Exports that feed the reference's analysis tools: the NSC contact network
(App::logNetworkFrame, src/app/main.cpp:3620-3700) and the profile CSV
(App::logCsvFrame, :3276-3355), from device counters.

* rg_get_contact_network against the oracle's manifolds: pairs exact, rows
  within 1e-10 of each column group's largest magnitude.
* The drop-in module's writers: the reference's exact headers, one profile
  row per frame whose counters equal the library's statistics, and network
  rows equal to rg_get_contact_network of the same frame.
"""
import csv
import json

import numpy as np
import pytest

from helpers import make_pair, packed_scene, rel_err

pytestmark = pytest.mark.gpu

NSC_CSV_HEADER = (
    "frame,rods,integrate_ms,sleep_ms,broadphase_ms,bpCount_ms,bpPrefix_ms,bpFill_ms,bpPairs_ms,"
    "bpLongLong_ms,warmstart_ms,buildIslands_ms,solve_ms,floorSolve_ms,posCorrect_ms,pbcWrap_ms,"
    "render_ms,contacts,collisions,islands,KE,KE_after_integrate,KE_after_warmstart,KE_after_solve,"
    "KE_after_posCorrect,KE_after_pbcWrap,soft_PE,gyration_sq,reldisp_sq,jn_sum,jt_sum,nsc_residual,"
    "ent_pairs,ent_sum,step_ms")
NET_HEADER = ("frame,rod_i,rod_j,contact_x,contact_y,contact_z,normal_x,normal_y,normal_z,phi,lambda_n,"
              "lambda_t1,lambda_t2,vn_pre,vn_post")


def test_contact_network_matches_oracle():
    sc = packed_scene(1500, d=0.1, phi=0.1, seed=61, squeeze=0.97)
    for team_blocks in (1, 4):  # single-block solve and the team path
        g, o = make_pair(sc, model="nsc", dt=5e-4, nsc_velocity_iters=200, team_blocks=team_blocks)
        g.set_network_export(True)
        for _ in range(3):
            g.step(1)
            o.step(1)
            pg, rg = g.contact_network()
            po, ro = o.contact_network()
            assert len(po) > 0
            np.testing.assert_array_equal(pg, po)
            for cols in (slice(0, 3), slice(3, 6), slice(6, 7), slice(7, 10), slice(10, 12)):
                assert rel_err(rg[:, cols], ro[:, cols]) < 1e-10, cols


def test_simulator_profile_and_network_csv(tmp_path):
    import build  # rod-dynamics-3d_b200/build.py
    build.build()
    import rod_dynamics_py as m
    cfg = {"scene": {"periodic": {"enabled": True, "min": [-1.5, -1.5, -1.5], "max": [1.5, 1.5, 1.5]},
                     "populate": {"count": 300, "mode": "nonoverlap", "seed": 7, "length": 1.0, "radius": 0.03,
                                  "density": 1000.0},
                     "randomInit": {"enabled": True, "mode": "gaussian", "vSigma": 2.0, "wSigma": 4.0, "seed": 3}},
           "physics": {"dt": 5e-4, "gravity": [0, 0, 0], "lin_damp": 0.0, "ang_damp": 0.0,
                       "nsc": {"enabled": True, "mu": 0.3, "velocity_iters": 500}}}
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(cfg))
    sim = m.Simulator(str(p))
    prof, net = tmp_path / "profile.csv", tmp_path / "network.csv"
    sim.enable_csv(str(prof))
    sim.enable_network(str(net), 2)
    stats = []
    for _ in range(40):
        sim.step(1)
        stats.append(sim.stats())
    del sim  # flushes and closes the files
    rows = list(csv.reader(open(prof)))
    assert ",".join(rows[0]) == NSC_CSV_HEADER
    body = rows[1:]
    assert [int(r[0]) for r in body] == list(range(1, 41))
    col = {k: i for i, k in enumerate(rows[0])}
    for r, st in zip(body, stats):
        assert int(r[col["contacts"]]) == st["contacts"]
        assert float(r[col["nsc_residual"]]) == pytest.approx(st["residual"], rel=1e-5, abs=1e-12)
        assert int(r[col["rods"]]) == 300
    assert sum(int(r[col["contacts"]]) for r in body) > 0
    assert sum(int(r[col["collisions"]]) for r in body) > 0
    nrows = list(csv.reader(open(net)))
    assert ",".join(nrows[0]) == NET_HEADER
    frames = {int(r[0]) for r in nrows[1:]}
    assert frames and all(f % 2 == 0 for f in frames)
    per_frame = {}
    for r in nrows[1:]:
        per_frame[int(r[0])] = per_frame.get(int(r[0]), 0) + 1
    for f, k in per_frame.items():
        assert k == int(body[f - 1][col["contacts"]]), f
