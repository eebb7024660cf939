"""CPU restatement of calculate_insert_size_stats (insert_size.rs:73-243).

Test infrastructure only: the parity checker of csrc/insert_size_kernel.cu.  Pure Python
floats (IEEE doubles, each operation rounded, no fused multiply-add), in the reference's
order: distances per orientation (infer_orientation, :34-51) in (0, 10000], sorted;
percentiles at trunc(q n + 0.499); bounds from 2 IQR for the mean and deviation (:118-131),
3 IQR widened to 4 deviations for proper pairs (:133-150); fewer than 10 pairs, or fewer
than 5% of the largest orientation's, fail (:130-133, 226-236).
"""
from __future__ import annotations

import math

MAX_INS, MIN_DIR_CNT, MIN_DIR_RATIO = 10000, 10, 0.05
OUTLIER_BOUND, MAPPING_BOUND, MAX_STDDEV = 2.0, 3.0, 4.0


def as_i32(x: float) -> int:
    if math.isnan(x):
        return 0
    if x >= 2**31 - 1:
        return 2**31 - 1
    if x <= -2**31:
        return -2**31
    return int(x)


def infer_orientation(l_pac: int, pos1: int, pos2: int):
    r1, r2 = int(pos1 >= l_pac), int(pos2 >= l_pac)
    p2 = pos2 if r1 == r2 else (l_pac << 1) - 1 - pos2
    dist = p2 - pos1 if p2 > pos1 else pos1 - p2
    return (0 if r1 == r2 else 1) ^ (0 if p2 > pos1 else 3), dist


def stats(l_pac: int, pairs) -> list[dict]:
    sizes = [[], [], [], []]
    for p1, p2 in pairs:
        o, d = infer_orientation(l_pac, int(p1), int(p2))
        if 0 < d <= MAX_INS:
            sizes[o].append(d)
    out = [{"avg": 0.0, "std": 0.0, "low": 0, "high": 0, "failed": 1} for _ in range(4)]
    for d in range(4):
        s = sorted(sizes[d])
        n = len(s)
        if n < MIN_DIR_CNT:
            continue
        p25 = s[int(0.25 * n + 0.499)]
        p75 = s[int(0.75 * n + 0.499)]
        iqr = p75 - p25
        low = as_i32((p25 - OUTLIER_BOUND * iqr) + 0.499)
        low = max(low, 1)
        high_o = as_i32((p75 + OUTLIER_BOUND * iqr) + 0.499)
        inb = [v for v in s if low <= v <= high_o]
        if not inb:
            continue
        avg = sum(inb) / len(inb)
        ss = 0.0
        for v in inb:
            diff = v - avg
            ss += diff * diff
        sd = math.sqrt(ss / len(inb))
        lo = as_i32((p25 - MAPPING_BOUND * iqr) + 0.499)
        hi = as_i32((p75 + MAPPING_BOUND * iqr) + 0.499)
        lo_sd = as_i32(avg - MAX_STDDEV * sd + 0.499)
        hi_sd = as_i32(avg + MAX_STDDEV * sd + 0.499)
        lo = min(lo, lo_sd)
        hi = max(hi, hi_sd)
        lo = max(lo, 1)
        out[d] = {"avg": avg, "std": sd, "low": lo, "high": hi, "failed": 0}
    mx = max(len(v) for v in sizes)
    for d in range(4):
        if not out[d]["failed"] and len(sizes[d]) < int(mx * MIN_DIR_RATIO):
            out[d]["failed"] = 1
    return out
