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


def features(max_score: int, jobs, qseq, tseq, hints=None) -> np.ndarray:
    """The 16 per-job features of the band predictor (band_model.cu), restated per job:
    mismatch statistics of the seed diagonal (ungapped alignment of query and target),
    of 8-position blocks along it, and of the best of the diagonals shifted by -4..4
    over the query's second half."""
    x = np.zeros((len(jobs), 16), np.float32)
    for i, jb in enumerate(jobs):
        qlen, tlen = int(jb["qlen"]), int(jb["tlen"])
        q = qseq[int(jb["q_off"]):int(jb["q_off"]) + qlen].astype(np.int64)
        t = tseq[int(jb["t_off"]):int(jb["t_off"]) + tlen].astype(np.int64)
        L = min(qlen, tlen)
        nblk = (L + 7) // 8
        half = qlen // 2
        d = (q[:L] != t[:L]) | (q[:L] > 3)
        mm = int(d.sum())
        last_mm = int(np.nonzero(d)[0].max()) if mm else -1
        nq = int((q > 3).sum())
        blk = [bool(d[8 * b:8 * b + 8].any()) for b in range(nblk)]
        mmblk = sum(blk)
        first = next((b for b in range(nblk) if blk[b]), -1)
        lastq = sum(1 for b in range(nblk) if blk[b] and b * 4 >= nblk * 3)
        best_run = run = 0
        for b in range(nblk):
            if blk[b]:
                run = 0
            else:
                run += 1
                best_run = max(best_run, run)
        best_s, best_c, best_n, best_last = 0, -1, 1, -1
        for sh in range(-4, 5):
            ks = np.arange(half, qlen)
            ts = ks + sh
            ok = (ts >= 0) & (ts < tlen)
            ks, ts = ks[ok], ts[ok]
            dd = (q[ks] != t[ts]) | (q[ks] > 3)
            cs, ns = int(dd.sum()), len(ks)
            ls = int(ks[dd].max()) if cs else -1
            if ns > 0 and (best_c < 0 or cs * best_n < best_c * ns or
                           (cs * best_n == best_c * ns and abs(sh) < abs(best_s))):
                best_s, best_c, best_n, best_last = sh, cs, ns, ls
        fb = np.float32(max(nblk, 1))
        o = x[i]
        o[0] = np.float32(jb["h0"]) / np.float32(max_score) if max_score > 0 else np.float32(jb["h0"])
        o[1] = qlen
        o[2] = qlen - last_mm
        o[3] = qlen - max(best_last, half - 1)
        o[4] = hints[i]["diag_spread"] if hints is not None else 0
        o[5] = float(hints[i]["has_partner"] != 0) if hints is not None else 0
        o[6] = mmblk
        o[7] = np.float32(mmblk) / fb
        o[8] = 1.0 if first < 0 else np.float32(first) / fb
        o[9] = lastq
        o[10] = np.float32(mm) / np.float32(max(L, 1))
        o[11] = np.float32(best_run) / fb
        o[12] = nq
        o[13] = tlen - qlen
        o[14] = abs(best_s)
        o[15] = 1.0 if best_c < 0 else np.float32(best_c) / np.float32(best_n)
    return x
