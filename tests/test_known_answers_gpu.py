"""The reference's known-answer smoke tests (tests/smoke_test.py) on the
GPU library, restated for capsules as in test_oracle_pin.py."""
import numpy as np
import pytest

import known_answers as KA
import rodgpu

pytestmark = pytest.mark.gpu


def test_nsc_elastic_exchange():
    va, vb = KA.nsc_elastic_exchange(rodgpu.System, 0.0)
    assert abs(va) < 1e-3 and abs(vb - 0.1) < 1e-3
    va, vb = KA.nsc_elastic_exchange(rodgpu.System, 0.05)
    assert vb > 0.09 and (va * va + vb * vb) / 0.01 > 0.95


def test_spatial_hash_pbc():
    assert KA.spatial_hash_pbc(rodgpu.System) >= 1


def test_sphere_capsule_pbc():
    n, _, _ = KA.sphere_capsule_pbc(rodgpu.System, False)
    assert n == 0
    n, vs, vc = KA.sphere_capsule_pbc(rodgpu.System, True)
    assert n >= 1 and vs < 0 < vc


def test_hertz_mindlin_repulsion():
    d0, d1, va, vb, ke = KA.hertz_mindlin_repulsion(rodgpu.System)
    assert d1 > d0 and va < 0 < vb and np.isfinite(ke) and ke < 100.0
