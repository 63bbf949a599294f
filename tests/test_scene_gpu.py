"""The device packing generator (rg_scene_rsa_device), which replaces the
host populate (src/app/main.cpp:1857-2140) for large scenes.

* valid: no two rods closer than one diameter (checked with the oracle's
  contact detection at the generated diameter);
* deterministic: the same arguments give the same packing;
* isotropic and uniform: axis moments and centre octants within a few
  standard errors;
* jamming: a target beyond the random-sequential-addition limit stops at the
  first rod that uses all its draws and returns the valid partial packing.
"""
import ctypes

import numpy as np
import pytest

import rodgpu
from oracle import Oracle
from rodgpu import scene

pytestmark = pytest.mark.gpu


def _device_rsa(n, L, d, phi, seed, max_attempts=2000):
    side = scene.box_side(n, L, d, phi)
    lo = -0.5 * side
    x = np.zeros((n, 3))
    q = np.zeros((n, 4))
    placed = ctypes.c_int()
    rc = rodgpu.lib().rg_scene_rsa_device(n, L, d, lo, side, seed, max_attempts, rodgpu.ptr(x), rodgpu.ptr(q),
                                          ctypes.byref(placed))
    assert rc == 0, rc
    m = placed.value
    return x[:m], q[:m], side, lo


def _min_gap(x, q, L, d, side, lo):
    """Smallest surface gap found by the oracle's detection at diameter d."""
    n = len(x)
    cfg = rodgpu.default_config(n_bodies=n, model="nsc", pbc_enabled=1, pbc_min=(lo,) * 3,
                                pbc_max=(lo + side,) * 3)
    o = Oracle(cfg)
    r = np.full(n, 0.5 * d)
    h = np.full(n, 0.5 * L)
    o.set_bodies(r, h, np.ones(n), np.ones((n, 3)), np.full(n, 0.2))
    o.set_state(x, q, np.zeros((n, 3)), np.zeros((n, 3)))
    pairs, geom, _ = o.detect(0.0)
    return len(pairs), (geom[:, 9].min() - d if len(pairs) else np.inf)


def test_device_packing_valid_deterministic_isotropic():
    n, L, d, phi = 20000, 1.0, 0.05, 0.08
    x, q, side, lo = _device_rsa(n, L, d, phi, seed=11)
    assert len(x) == n
    x2, q2, _, _ = _device_rsa(n, L, d, phi, seed=11)
    np.testing.assert_array_equal(x, x2)
    np.testing.assert_array_equal(q, q2)
    x3, _, _, _ = _device_rsa(n, L, d, phi, seed=12)
    assert not np.array_equal(x, x3)
    contacts, gap = _min_gap(x, q, L, d, side, lo)
    assert contacts == 0 or gap > -1e-12 * d, (contacts, gap)
    # unit quaternions; axes uniform on the sphere
    np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-12)
    w, a, b, c = q.T
    u = np.stack([2 * (a * b - w * c), 1 - 2 * (a * a + c * c), 2 * (b * c + w * a)], 1)
    se = 1.0 / np.sqrt(n)
    assert np.all(np.abs(u.mean(0)) < 5 * se * np.sqrt(1 / 3))
    assert abs(np.abs(u[:, 1]).mean() - 0.5) < 5 * se * np.sqrt(1 / 12)
    assert abs((u[:, 0] ** 2).mean() - 1 / 3) < 5 * se * np.sqrt(4 / 45)
    # centres uniform: octant counts
    octant = ((x - lo) // (0.5 * side)).astype(int) @ np.array([1, 2, 4])
    counts = np.bincount(octant, minlength=8)
    assert np.all(np.abs(counts - n / 8) < 5 * np.sqrt(n / 8))


def test_device_packing_stops_when_jammed():
    # aspect ratio 20 at phi 0.3 is far beyond the isotropic RSA limit
    n, L, d = 6000, 1.0, 0.05
    x, q, side, lo = _device_rsa(n, L, d, 0.3, seed=5, max_attempts=200)
    assert 0 < len(x) < n
    contacts, gap = _min_gap(x, q, L, d, side, lo)
    assert contacts == 0 or gap > -1e-12 * d, (contacts, gap)
