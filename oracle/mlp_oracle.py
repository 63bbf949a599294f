"""CPU oracle of the learned PSOR warm start (test infrastructure only).

Restates, in numpy, the network and the loss that the library's training and
inference kernels compute (rod-dynamics-3d_b200/csrc/rg_mlp.cu and
rg_mlp_dev.cuh): 8 -> 128 -> 128 -> 128 -> 3, SiLU, a mean-squared loss on
the normalised impulse change (target - previous impulse) / output scale.
The reference has no learned part (its warm start is the impulse cache of
src/physics/nsc_contact.cpp:305-317), so this oracle is pinned by finite
differences of its own FP64 gradient, not by reference outputs.

`emulate_bf16=True` rounds exactly where the device rounds to BF16 (the
normalised input, the weights, the hidden activations and the backward
deltas that feed GEMMs) and accumulates in float64 otherwise, so device
gradients agree with it to a few BF16 ulps of accumulation-order noise.
"""
import numpy as np

IN, H, OUT = 8, 128, 3
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + OUT * H
OFF_IN_MEAN = OFF_B4 + OUT
OFF_IN_SCALE = OFF_IN_MEAN + IN
OFF_OUT_SCALE = OFF_IN_SCALE + IN
N_PARAMS = OFF_OUT_SCALE + OUT


def bf16(x):
    """Round float32 values to BF16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    return dict(
        W1=P[OFF_W1:OFF_B1].reshape(H, IN), b1=P[OFF_B1:OFF_W2],
        W2=P[OFF_W2:OFF_B2].reshape(H, H), b2=P[OFF_B2:OFF_W3],
        W3=P[OFF_W3:OFF_B3].reshape(H, H), b3=P[OFF_B3:OFF_W4],
        W4=P[OFF_W4:OFF_B4].reshape(OUT, H), b4=P[OFF_B4:OFF_IN_MEAN],
        mean=P[OFF_IN_MEAN:OFF_IN_SCALE], scale=P[OFF_IN_SCALE:OFF_OUT_SCALE],
        oscale=P[OFF_OUT_SCALE:N_PARAMS])


def init_params(feat, tgt, seed=0):
    """Normalisation from the data and He-uniform weights (the library draws
    its own weights; this generator is only for oracle-side tests)."""
    feat = np.asarray(feat, np.float64)
    tgt = np.asarray(tgt, np.float64)
    P = np.zeros(N_PARAMS, np.float64)
    m = feat.mean(0)
    sd = feat.std(0)
    P[OFF_IN_MEAN:OFF_IN_SCALE] = m
    P[OFF_IN_SCALE:OFF_OUT_SCALE] = np.where(sd > 1e-30, 1.0 / np.maximum(sd, 1e-300), 1.0)
    d = tgt - feat[:, 4:7]
    rms = np.sqrt((d * d).mean(0))
    P[OFF_OUT_SCALE:] = np.where(rms > 1e-30, rms, 1.0)
    rng = np.random.default_rng(seed)
    for off, fan, cnt in ((OFF_W1, IN, H * IN), (OFF_W2, H, H * H), (OFF_W3, H, H * H), (OFF_W4, H, OUT * H)):
        lim = np.sqrt(6.0 / fan)
        P[off:off + cnt] = rng.uniform(-lim, lim, cnt)
    P[OFF_W4:OFF_B4] *= 0.1
    return P.astype(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _rounder(emulate_bf16):
    return bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))


def forward(P, feat, emulate_bf16=True):
    """Network output (normalised units) and the intermediates."""
    r = _rounder(emulate_bf16)
    p = unpack(P)
    X = r((np.asarray(feat, np.float64) - p["mean"]) * p["scale"])
    W = [r(p[k]) for k in ("W1", "W2", "W3", "W4")]
    Z1 = X @ W[0].T + p["b1"]
    H1 = r(silu(Z1))
    Z2 = H1 @ W[1].T + p["b2"]
    H2 = r(silu(Z2))
    Z3 = H2 @ W[2].T + p["b3"]
    H3 = r(silu(Z3))
    Y = H3 @ W[3].T + p["b4"]
    return Y, dict(X=X, W=W, Z=(Z1, Z2, Z3), H=(H1, H2, H3))


def predict(P, feat, emulate_bf16=True):
    """Predicted impulses: previous impulse + output x output scale."""
    Y, _ = forward(P, feat, emulate_bf16)
    return np.asarray(feat, np.float64)[:, 4:7] + Y * unpack(P)["oscale"]


def loss_and_grad(P, feat, tgt, emulate_bf16=True):
    """Mean squared error on the normalised impulse change and its gradient
    in the parameter layout (normalisation entries 0)."""
    r = _rounder(emulate_bf16)
    p = unpack(P)
    feat = np.asarray(feat, np.float64)
    n = len(feat)
    Y, c = forward(P, feat, emulate_bf16)
    T = (np.asarray(tgt, np.float64) - feat[:, 4:7]) / p["oscale"]
    D = Y - T
    loss = float((D * D).sum() / (n * OUT))
    dY = 2.0 * D / (n * OUT)
    dYb = r(dY)
    G = np.zeros(N_PARAMS, np.float64)
    (Z1, Z2, Z3), (H1, H2, H3), W, X = c["Z"], c["H"], c["W"], c["X"]
    G[OFF_W4:OFF_B4] = (dYb.T @ H3).ravel()
    G[OFF_B4:OFF_IN_MEAN] = dY.sum(0)
    dH = dYb @ W[3]
    for (Z, Hprev, Wl, offw, offb, fan) in ((Z3, H2, W[2], OFF_W3, OFF_B3, H), (Z2, H1, W[1], OFF_W2, OFF_B2, H),
                                            (Z1, X, W[0], OFF_W1, OFF_B1, IN)):
        dZ = dH * dsilu(Z)
        dZb = r(dZ)
        G[offw:offw + H * fan] = (dZb.T @ Hprev).ravel()
        G[offb:offb + H] = dZ.sum(0)
        dH = dZb @ Wl
    return loss, G


def synthetic_records(n, seed=0):
    """Seeded records with the scales of NSC contact features: gaps ~1e-3,
    velocities ~1e-1, impulses ~1e-4, degrees 0-12; the converged impulse
    is a smooth function of them."""
    rng = np.random.default_rng(seed)
    x = np.zeros((n, IN), np.float64)
    x[:, 0] = -np.abs(rng.normal(0, 1e-3, n))
    x[:, 1] = rng.normal(0, 0.1, n)
    x[:, 2:4] = rng.normal(0, 0.05, (n, 2))
    x[:, 4] = np.abs(rng.normal(0, 1e-4, n)) * (rng.random(n) < 0.7)
    x[:, 5:7] = rng.normal(0, 3e-5, (n, 2)) * (x[:, 4:5] > 0)
    x[:, 7] = rng.integers(0, 13, n)
    y = np.zeros((n, OUT), np.float64)
    y[:, 0] = np.maximum(0.0, 0.8 * x[:, 4] - 4e-4 * x[:, 1] - 0.02 * x[:, 0] + 1e-6 * x[:, 7])
    y[:, 1] = 0.9 * x[:, 5] - 2e-4 * x[:, 2] * np.tanh(y[:, 0] / 1e-4)
    y[:, 2] = 0.9 * x[:, 6] - 2e-4 * x[:, 3] * np.tanh(y[:, 0] / 1e-4)
    return x.astype(np.float32), y.astype(np.float32)
