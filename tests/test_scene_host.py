"""Host-side scene helpers (no GPU): the Morton renumbering of a packing."""
import numpy as np


def test_morton_order_renumbers_rods_only():
    """morton_order is a renumbering: the same rods (every per-rod array
    permuted alike), neighbours closer in index than in generation order."""
    from rodgpu import scene
    sc = scene.make_rods(1500, 1.0, 0.05, phi=0.1, seed=4)
    m = scene.morton_order(sc)
    assert m["n"] == sc["n"] and m["side"] == sc["side"]
    # the same rods: match each rod by its centre, then every array agrees
    key = lambda d: np.lexsort(d["x"].T)  # noqa: E731
    a, b = key(sc), key(m)
    for k in ("x", "q", "v", "w", "radius", "half_height", "mass", "inertia", "restitution"):
        np.testing.assert_array_equal(sc[k][a], m[k][b])
    step = lambda d: np.linalg.norm(np.diff(d["x"], axis=0), axis=1).mean()  # noqa: E731
    assert step(m) < 0.5 * step(sc)
