"""rg_detect_noalloc: contact detection for callers that cannot allocate
device memory (the library uses a fixed file-scope device array instead of
cudaMalloc).  Checked through the C ABI against rg_detect on two calls in a
row with different systems, so stale scratch contents would show.  Pair lists
and geometry must be bit-identical (the same FP64 predicate and arithmetic).

Collected last on purpose (tests/test_zz_*): if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import rodgpu
from helpers import make_pair, packed_scene

pytestmark = pytest.mark.gpu

MAX_BODIES = 8192  # RG_NOALLOC_MAX_BODIES (include/rodgpu.h)


def _dev(a, torch, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).cuda()


def _noalloc_detect(sc, delta, cfg, torch, cap=None, inv_mass=True):
    L = rodgpu.lib()
    n = sc["n"]
    x = _dev(sc["x"], torch, torch.float64)
    q = _dev(sc["q"], torch, torch.float64)
    r = _dev(sc["radius"], torch, torch.float64)
    h = _dev(sc["half_height"], torch, torch.float64)
    im = _dev(np.where(sc["mass"] > 0, 1.0 / np.maximum(sc["mass"], 1e-300), 0.0), torch, torch.float64)
    im_ptr = im.data_ptr() if inv_mass else ctypes.c_void_p(0)
    cap = cap or 8 * n + 16
    pairs = torch.full((cap, 2), -1, dtype=torch.int32, device="cuda")
    geom = torch.zeros((cap, 12), dtype=torch.float64, device="cuda")
    count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    lo = (ctypes.c_double * 3)(*cfg.pbc_min)
    hi = (ctypes.c_double * 3)(*cfg.pbc_max)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.rg_detect_noalloc(x.data_ptr(), q.data_ptr(), r.data_ptr(), h.data_ptr(), im_ptr, n,
                             int(cfg.pbc_enabled), lo, hi, float(delta), pairs.data_ptr(), geom.data_ptr(), cap,
                             count.data_ptr(), ctypes.c_void_p(stream))
    assert rc == 0, rc
    torch.cuda.synchronize()
    m = int(count.item())
    return pairs[:m].cpu().numpy(), geom[:m].cpu().numpy(), m


def test_noalloc_matches_rg_detect_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    scenes = [(packed_scene(3000, d=0.05, phi=0.2, seed=31, squeeze=0.97), "nsc", 0.0),
              (packed_scene(1200, d=0.1, phi=0.1, seed=32, squeeze=0.95), "harmonic", 0.005)]
    for sc, model, delta in scenes:  # two calls in a row, different sizes
        g, _ = make_pair(sc, model=model)
        pg, gg, _ = g.detect(delta)
        pn, gn, m = _noalloc_detect(sc, delta, g.cfg, torch)
        assert m == len(pg) > 0
        np.testing.assert_array_equal(pn, pg)
        np.testing.assert_array_equal(gn, gg)


def test_noalloc_rejects_oversize_and_counts_overflow():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    L = rodgpu.lib()
    z = ctypes.c_void_p(0)
    one = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    cnt = torch.zeros((1,), dtype=torch.int32, device="cuda")
    rc = L.rg_detect_noalloc(z, z, z, z, z, MAX_BODIES + 1, 0, one, one, 0.0, z, z, 0, cnt.data_ptr(), z)
    assert rc == 3  # RG_ERR_CAPACITY, before any device work
    sc = packed_scene(1500, d=0.1, phi=0.1, seed=33, squeeze=0.9)
    g, _ = make_pair(sc, model="nsc")
    pg, gg, _ = g.detect(0.0)
    assert len(pg) > 4
    pn, gn, m = _noalloc_detect(sc, 0.0, g.cfg, torch, cap=4)  # output smaller than the contact set
    assert m == len(pg)
    np.testing.assert_array_equal(pn[:4], pg[:4])


def test_noalloc_open_box_static_bodies_and_no_inv_mass():
    """The branches the periodic scenes above do not reach: an open box (no
    minimum image), pairs of two static bodies (skipped), and inv_mass NULL
    (every body dynamic).  Checked against rg_detect and the oracle."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    sc = packed_scene(1000, d=0.1, phi=0.12, seed=34, squeeze=0.95)
    sc["mass"] = sc["mass"].copy()
    sc["mass"][::5] = 0.0  # every fifth body static: some contacts join two of them
    g, o = make_pair(sc, model="nsc", pbc_enabled=0)
    pg, gg, _ = g.detect(0.0)
    po, go, _ = o.detect(0.0)
    np.testing.assert_array_equal(pg, po)
    np.testing.assert_array_equal(gg, go)
    static = sc["mass"] <= 0
    assert not np.any(static[pg[:, 0]] & static[pg[:, 1]])
    pn, gn, m = _noalloc_detect(sc, 0.0, g.cfg, torch)
    assert m == len(pg) > 0
    np.testing.assert_array_equal(pn, pg)
    np.testing.assert_array_equal(gn, gg)
    # inv_mass NULL: every body dynamic, so pairs of two "static" bodies come
    # back; it must equal a system whose bodies are all dynamic
    sd = dict(sc)
    sd["mass"] = np.where(static, np.median(sc["mass"][~static]), sc["mass"])
    g2, o2 = make_pair(sd, model="nsc", pbc_enabled=0)
    p2, g2g, _ = g2.detect(0.0)
    p2o, _, _ = o2.detect(0.0)
    np.testing.assert_array_equal(p2, p2o)
    assert len(p2) > len(pg)
    pn2, gn2, m2 = _noalloc_detect(sd, 0.0, g2.cfg, torch, inv_mass=False)
    assert m2 == len(p2)
    np.testing.assert_array_equal(pn2, p2)
    np.testing.assert_array_equal(gn2, g2g)
