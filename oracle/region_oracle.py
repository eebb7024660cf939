"""CPU restatement of the region merge (merge_scores_to_regions).

Test infrastructure only: the parity checker of the region-merge kernel
(ferrousalign_b200/csrc/region_kernel.cu).  Pure Python over plain integers, restating
src/pipelines/linear/region.rs:737-890 step by step:

* region.rs:772-781  bounds start at the seed, total score = seed.len * a;
* region.rs:784-809  left result present (index inside the left results): total = its score;
  local when gscore <= 0 or gscore <= score - pen_clip5 (qb = query_pos - qle,
  rb = ref_pos - tle, truesc = score), else qb = 0, rb = ref_pos - gtle, truesc = gscore;
  no left job and query_pos == 0: truesc = len * a;
* region.rs:816-836  right result present: total += its score; local when gscore <= 0 or
  gscore <= score - pen_clip3 (qe = query_pos + len + qle, re = ref_pos + len + tle), else
  qe = query_len, re = ref_pos + len + gtle;
* region.rs:841-845  score = total, truesc = total where it is still 0;
* region.rs:847-858  seedcov = summed length of the chain's seeds inside [qb,qe) x [rb,re);
* region.rs:868-872  the chain keeps the first seed with the strictly highest total.

Reference positions are u64 in the reference (Rust `as u64` sign-extends an i32 and the
subtraction wraps in release builds), restated with arithmetic modulo 2^64.
Parity is pinned against this restatement and hand-derived cases in the tests: the
reference has no unit test of this function (it needs a loaded index).
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1
INT32_MIN = -(1 << 31)

SEED_EXT_DT = np.dtype([("ref_pos", "<u8"), ("query_pos", "<i4"), ("len", "<i4"), ("left_job", "<i4"),
                        ("right_job", "<i4")])
REGION_DT = np.dtype([("rb", "<u8"), ("re", "<u8"), ("qb", "<i4"), ("qe", "<i4"), ("score", "<i4"),
                      ("truesc", "<i4"), ("seedcov", "<i4"), ("seedlen0", "<i4"), ("w", "<i4"), ("seed", "<i4")])


def _u64(x: int) -> int:
    return x & M64


def merge_chain(opt: dict, seeds: list[dict], query_len: int, left, right) -> dict:
    """One chain: `seeds` in the reference's mapping order; left/right are sequences of
    result records (dicts or numpy records with score, qle, tle, gtle, gscore)."""
    a, clip5, clip3, w = opt["a"], opt["pen_clip5"], opt["pen_clip3"], opt["w"]
    best = {"rb": 0, "re": 0, "qb": 0, "qe": 0, "score": 0, "truesc": 0, "seedcov": 0, "seedlen0": 0, "w": w,
            "seed": -1}
    best_score = INT32_MIN
    for k, sd in enumerate(seeds):
        qpos, ln, rpos = int(sd["query_pos"]), int(sd["len"]), int(sd["ref_pos"])
        lj, rj = int(sd["left_job"]), int(sd["right_job"])
        qb, qe = qpos, qpos + ln
        rb, re = rpos, _u64(rpos + ln)
        truesc = 0
        total = ln * a
        if lj >= 0:
            if lj < len(left):
                L = left[lj]
                total = int(L["score"])
                if int(L["gscore"]) <= 0 or int(L["gscore"]) <= int(L["score"]) - clip5:
                    qb = qpos - int(L["qle"])
                    rb = _u64(rpos - int(L["tle"]))
                    truesc = int(L["score"])
                else:
                    qb = 0
                    rb = _u64(rpos - int(L["gtle"]))
                    truesc = int(L["gscore"])
        elif qpos == 0:
            truesc = ln * a
        if rj >= 0 and rj < len(right):
            R = right[rj]
            total += int(R["score"])
            if int(R["gscore"]) <= 0 or int(R["gscore"]) <= int(R["score"]) - clip3:
                qe = qpos + ln + int(R["qle"])
                re = _u64(rpos + ln + int(R["tle"]))
            else:
                qe = query_len
                re = _u64(rpos + ln + int(R["gtle"]))
        if truesc == 0:
            truesc = total
        cov = 0
        for so in seeds:
            sq, sl, sr = int(so["query_pos"]), int(so["len"]), int(so["ref_pos"])
            if sq >= qb and sq + sl <= qe and sr >= rb and _u64(sr + sl) <= re:
                cov += sl
        if total > best_score:
            best_score = total
            best = {"rb": rb, "re": re, "qb": qb, "qe": qe, "score": total, "truesc": truesc, "seedcov": cov,
                    "seedlen0": ln, "w": w, "seed": k}
    return best


def merge_regions(opt: dict, chain_first, query_len, seeds, left, right) -> np.ndarray:
    """All chains; out[c]["seed"] is an index into `seeds` (-1: no region)."""
    n = len(chain_first) - 1
    out = np.zeros(n, REGION_DT)
    for c in range(n):
        s0, s1 = int(chain_first[c]), int(chain_first[c + 1])
        r = merge_chain(opt, [seeds[k] for k in range(s0, s1)], int(query_len[c]), left, right)
        if r["seed"] >= 0:
            r["seed"] += s0
        out[c] = tuple(r[f] for f in REGION_DT.names)
    return out
