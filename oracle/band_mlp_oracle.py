"""NumPy restatement of the band predictor's MLP (test checker only).

Forward with BF16-rounded weights (round to nearest even, as the CUDA kernels store
them), ReLU hidden layers, pinball loss on the log2 band, and the analytic backward
pass in float64 -- the reference the GPU forward/backward kernels are checked against.
"""
from __future__ import annotations

import numpy as np

NIN, NH1, NH2 = 16, 64, 32
O_W1, O_B1 = 0, NH1 * NIN
O_W2, O_B2 = O_B1 + NH1, O_B1 + NH1 + NH2 * NH1
O_W3, O_B3 = O_B2 + NH2, O_B2 + NH2 + NH2
NPARAMS = O_B3 + 1


def bf16_round(w: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(w):
    return (w[O_W1:O_B1].reshape(NH1, NIN), w[O_B1:O_W2], w[O_W2:O_B2].reshape(NH2, NH1), w[O_B2:O_W3],
            w[O_W3:O_B3], w[O_B3])


def forward(w, mean, std, x):
    W1, b1, W2, b2, W3, b3 = unpack(bf16_round(w).astype(np.float64))
    inv = np.where(std > 1e-12, 1.0 / std.astype(np.float64), 1.0)
    xn = (x.astype(np.float64) - mean.astype(np.float64)) * inv
    a1 = xn @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    return xn, h1, h2, y


def grad(w, mean, std, x, target, tau):
    W1, b1, W2, b2, W3, b3 = unpack(bf16_round(w).astype(np.float64))
    xn, h1, h2, y = forward(w, mean, std, x)
    n = len(x)
    r = target.astype(np.float64) - y
    loss = np.where(r >= 0, tau * r, (tau - 1) * r).mean()
    dy = np.where(r > 0, -tau, np.where(r < 0, 1 - tau, 0.0)) / n
    g = np.zeros(NPARAMS)
    g[O_W3:O_B3] = dy @ h2
    g[O_B3] = dy.sum()
    d2 = (dy[:, None] * W3[None, :]) * (h2 > 0)
    g[O_W2:O_B2] = (d2.T @ h1).reshape(-1)
    g[O_B2:O_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    g[O_W1:O_B1] = (d1.T @ xn).reshape(-1)
    g[O_B1:O_W2] = d1.sum(0)
    return g, loss


def first_band(y, margin: float, w_min: int, wj):
    """The predicted first band of a job from the network output y (log2 band):
    ceil(2^(y + margin)) with the exponent clamped to [0, 16], raised to w_min, rounded
    up to the ladder 2^k / 3*2^(k-1), and the configured band wj when twice that
    exceeds wj."""
    e = np.clip(np.asarray(y, np.float64) + margin, 0.0, 16.0)
    band = np.maximum(np.ceil(np.exp2(e)).astype(np.int64), w_min)
    p2 = np.where(band > 2, 1 << np.ceil(np.log2(np.maximum(band, 2))).astype(np.int64), band)
    three = 3 * p2 // 4
    band = np.where(band > 2, np.where(three >= band, three, p2), band)
    wj = np.asarray(wj, np.int64)
    band = np.where(2 * band > wj, wj, band)
    return np.minimum(band, wj).astype(np.int32)
