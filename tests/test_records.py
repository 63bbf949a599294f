"""The PSOR training-record file format (rodgpu.records): round trip,
validation and merging, on CPU."""
import numpy as np
import pytest

from rodgpu import records


def _data(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(n, 8)).astype(np.float32), rng.normal(size=(n, 3)).astype(np.float32),
            rng.integers(0, 3, n).astype(np.int32), rng.integers(0, 50, n).astype(np.int32),
            [{"seed": seed + k, "rods": 100, "mu": 0.1 * k} for k in range(3)])


def test_round_trip_and_merge(tmp_path):
    a, b = _data(500, 1), _data(300, 2)
    pa, pb = tmp_path / "a.npz", tmp_path / "b.npz"
    records.save(pa, *a)
    records.save(pb, *b)
    da, db = records.load(pa), records.load(pb)
    for k, arr in zip(("features", "targets", "run", "step"), a[:4]):
        np.testing.assert_array_equal(da[k], arr)
    assert da["runs"] == a[4]
    m = records.merge([da, db])
    assert len(m["features"]) == 800 and len(m["runs"]) == 6
    np.testing.assert_array_equal(m["run"][500:], b[2] + 3)


def test_rejects_bad_shapes_and_foreign_files(tmp_path):
    f, t, r, s, runs = _data(10, 3)
    with pytest.raises(ValueError):
        records.save(tmp_path / "x.npz", f[:, :7], t, r, s, runs)
    np.savez(tmp_path / "other.npz", format=np.array("something-else"), features=f)
    with pytest.raises(ValueError):
        records.load(tmp_path / "other.npz")

