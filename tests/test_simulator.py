"""The drop-in Python module rod_dynamics_py (C++ host code over the C ABI)
with the reference's Simulator surface (src/python/rod_dynamics_py.cpp)."""
import json
import math

import pytest


def _mod():
    import build  # rod-dynamics-3d_b200/build.py
    build.build()
    import rod_dynamics_py
    return rod_dynamics_py


def _scene(tmp_path, name, cfg):
    p = tmp_path / f"{name}.json"
    p.write_text(json.dumps(cfg))
    return str(p)


def test_module_surface_and_errors(tmp_path):
    m = _mod()
    for meth in ("step", "diagnostics", "rods", "stats"):
        assert hasattr(m.Simulator, meth)
    with pytest.raises(RuntimeError):
        m.Simulator(str(tmp_path / "missing.json"))
    bad = tmp_path / "bad.json"
    bad.write_text("{\"physics\": [1, 2,}")
    with pytest.raises(RuntimeError, match="JSON"):
        m.Simulator(str(bad))
    sph = _scene(tmp_path, "sphere", {"scene": {"bodies": [{"shape": "sphere", "radius": 0.1}]}})
    with pytest.raises(RuntimeError, match="capsule"):
        m.Simulator(sph)
    mj = _scene(tmp_path, "mj", {"physics": {"contact_model": "mujoco"}, "scene": {"bodies": [{}]}})
    with pytest.raises(RuntimeError, match="mujoco"):
        m.Simulator(mj)


def _elastic(cfm):
    c = math.sqrt(0.5)
    rod = {"shape": "capsule", "radius": 0.01, "length": 1.0, "density": 1000.0, "restitution": 1.0,
           "friction": 0.0}
    a = dict(rod, pos=[-0.06, 0, 0], v_lin=[0.1, 0, 0])
    b = dict(rod, pos=[0.06, 0, 0], rot_quat=[c, c, 0, 0])
    return {"scene": {"bodies": [a, b]},
            "physics": {"dt": 1e-3, "gravity": [0, 0, 0], "lin_damp": 0.0, "ang_damp": 0.0,
                        "nsc": {"enabled": True, "mu": 0.0, "velocity_iters": 200, "beta": 0.0, "cfm": cfm,
                                "omega": 1.0}}}


@pytest.mark.gpu
def test_simulator_nsc_elastic_exchange(tmp_path):
    """smoke_test.py:165-204 through the drop-in module."""
    m = _mod()
    sim = m.Simulator(_scene(tmp_path, "el0", _elastic(0.0)))
    r0 = sim.rods()
    assert r0[0]["mass"] < 1.0 and r0[0]["shape"] == "capsule"
    ea = r0[1]["endpoint_a"]  # 90 degrees about x: the rod axis lies along z
    assert abs(abs(ea[2]) - 0.5) < 1e-9 and abs(ea[1]) < 1e-9
    sim.step(3000)
    d = sim.diagnostics()
    assert d["frame_index"] == 3000 and d["rod_count"] == 2
    va = sim.rods()[0]["linear_velocity"][0]
    vb = sim.rods()[1]["linear_velocity"][0]
    assert abs(va) < 1e-3 and abs(vb - 0.1) < 1e-3
    sim = m.Simulator(_scene(tmp_path, "el5", _elastic(0.05)))
    sim.step(3000)
    va = sim.rods()[0]["linear_velocity"][0]
    vb = sim.rods()[1]["linear_velocity"][0]
    assert vb > 0.09 and (va * va + vb * vb) / 0.01 > 0.95


@pytest.mark.gpu
def test_simulator_populated_periodic_scene(tmp_path):
    """A populated periodic NSC scene shaped like the reference's
    assets/scenes/default_entangled_nsc.json."""
    m = _mod()
    cfg = {"scene": {"periodic": {"enabled": True, "min": [-2, -2, -2], "max": [2, 2, 2]},
                     "populate": {"count": 400, "mode": "nonoverlap", "seed": 5, "length": 1.0, "radius": 0.025,
                                  "density": 1000.0},
                     "randomInit": {"enabled": True, "mode": "gaussian", "vSigma": 0.1, "wSigma": 0.2, "seed": 42}},
           "physics": {"dt": 5e-4, "gravity": [0, 0, 0], "lin_damp": 0.0, "ang_damp": 0.0,
                       "nsc": {"enabled": True, "mu": 0.3, "velocity_iters": 500}}}
    sim = m.Simulator(_scene(tmp_path, "pop", cfg))
    assert sim.diagnostics()["rod_count"] == 400
    ke0 = sim.diagnostics()["last_ke"]
    assert ke0 > 0
    sim.step(50)
    d = sim.diagnostics()
    assert d["frame_index"] == 50 and math.isfinite(d["last_ke"])
    for r in sim.rods():
        assert all(-2 <= c < 2 for c in r["position"])
    st = sim.stats()
    assert st["not_converged"] == 0 and st["max_residual"] < 1e-6
