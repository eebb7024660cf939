"""The insert-size statistics kernels (csrc/insert_size_kernel.cu) against the CPU
restatement of calculate_insert_size_stats (oracle/insert_size_oracle.py): every field of
the four orientations, the doubles bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = 50_000_000


def pairs_mix(rng, n, fr_mean=400, fr_sd=50):
    p1 = rng.integers(0, L - 20000, n)
    kind = rng.choice(4, n, p=[0.02, 0.9, 0.05, 0.03])
    ins = np.maximum(rng.normal(fr_mean, fr_sd, n).astype(np.int64), 1)
    ins[rng.random(n) < 0.01] = rng.integers(10001, 30000)      # beyond MAX_INS: dropped
    ins[rng.random(n) < 0.02] = rng.integers(1, 5000)           # outliers
    rev2 = (2 * L) - 1 - (p1 + ins - 1)
    p2 = np.where(kind == 1, rev2, np.where(kind == 0, p1 + ins, np.where(kind == 2, (2 * L) - 1 - (p1 - ins),
                                                                           p1 - ins)))
    p2 = np.where(kind == 2, np.clip(p2, 0, 2 * L - 1), np.clip(p2, 0, 2 * L - 1))
    flip = rng.random(n) < 0.5                                   # read 1 on the reverse strand
    a = np.where(flip, (2 * L) - 1 - p1, p1)
    b = np.where(flip, (2 * L) - 1 - p2, p2)
    return np.stack([a, b], 1).astype(np.int64)


def test_stats_match_oracle_bit_for_bit(built):
    from ferrousalign_b200 import mate_rescue as R
    from oracle import insert_size_oracle as S
    rng = np.random.default_rng(9)
    for n, mean, sd in ((5000, 400, 50), (200_000, 350, 80), (40, 300, 10), (0, 1, 1)):
        pairs = pairs_mix(rng, n, mean, sd) if n else np.zeros((0, 2), np.int64)
        got = R.calculate_insert_size_stats(L, pairs)
        want = S.stats(L, [tuple(p) for p in pairs])
        for g, w in zip(got, want):
            assert (int(g["low"]), int(g["high"]), int(g["failed"])) == (w["low"], w["high"], w["failed"]), (n, g, w)
            assert np.float64(g["avg"]).tobytes() == np.float64(w["avg"]).tobytes(), (n, g["avg"], w["avg"])
            assert np.float64(g["std"]).tobytes() == np.float64(w["std"]).tobytes(), (n, g["std"], w["std"])
    b = R.insert_bounds(got)
    assert list(b["failed"]) == [int(x) for x in got["failed"]]
