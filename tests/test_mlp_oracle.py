"""The learned warm start's CPU oracle, pinned by finite differences (CPU)."""
import numpy as np

import mlp_oracle as M


def test_bf16_rounding_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-4], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even mantissa
    assert r[2] == 1.0 + 2 ** -6            # tie -> even (rounds up)
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-4) / 3.0e-4 < 2 ** -8


def test_fp64_gradient_matches_finite_differences():
    x, y = M.synthetic_records(48, seed=3)
    P = M.init_params(x, y, seed=5).astype(np.float64)
    loss, G = M.loss_and_grad(P, x, y, emulate_bf16=False)
    rng = np.random.default_rng(0)
    blocks = [(M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B3, M.OFF_W4),
              (M.OFF_W4, M.OFF_B4), (M.OFF_B4, M.OFF_IN_MEAN)]
    for lo, hi in blocks:
        for i in rng.integers(lo, hi, 4):
            h = 1e-6 * max(1.0, abs(P[i]))
            Pp, Pm = P.copy(), P.copy()
            Pp[i] += h
            Pm[i] -= h
            lp, _ = M.loss_and_grad(Pp, x, y, emulate_bf16=False)
            lm, _ = M.loss_and_grad(Pm, x, y, emulate_bf16=False)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - G[i]) <= 1e-6 * max(1e-3, abs(fd)) + 1e-9, (i, fd, G[i])


def test_bf16_emulation_close_to_fp64():
    x, y = M.synthetic_records(256, seed=4)
    P = M.init_params(x, y, seed=6)
    l64, g64 = M.loss_and_grad(P, x, y, emulate_bf16=False)
    l16, g16 = M.loss_and_grad(P, x, y, emulate_bf16=True)
    assert abs(l16 - l64) / l64 < 2e-2
    cos = g16 @ g64 / (np.linalg.norm(g16) * np.linalg.norm(g64))
    assert cos > 0.999
