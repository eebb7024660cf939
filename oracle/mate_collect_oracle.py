"""CPU restatement of the mate-rescue job collection (collect_rescue_jobs_for_read_soa).

Test infrastructure only: the parity checker of the rescue-job kernels
(ferrousalign_b200/csrc/mate_collect_kernel.cu).  Pure Python, restating
src/pipelines/linear/paired/mate_rescue.rs:1804-2045 step by step:

* :1822-1870  best score of the read's alignments (0 without any), threshold
  best - pen_unpaired (i32 saturating), no rescue unless some alignment reaches it (at most
  max_matesw counted; a negative max_matesw counts all) and the primary one does;
* :1894-1904  the anchor's FM-index start (reverse strand: 2 l_pac - 1 - its rightmost base);
* :1907-1940  orientations skipped when their statistics failed or one of the read's own
  alignments on the anchor's sequence sits at a consistent distance (mem_infer_dir,
  mate_rescue.rs:537-551);
* :1956-2044  per orientation the window [anchor +/- insert bounds (+/- read length)], clamped to
  [0, 2 l_pac), cut to the sequence under its midpoint (bns_fetch_seq, bntseq.rs:700-739, with
  bns_pos2rid's binary search, :535-559), kept when that is the anchor's sequence and at least
  min_seed_len long; the read reverse complemented (N stays N) for orientations 1 and 2.
Windows' bases come from the packed reference as in bns_get_seq (bntseq.rs:581-621).
"""
from __future__ import annotations

from oracle.collect_oracle import get_pac


def _sat_i32(x: int) -> int:
    return max(-2**31, min(2**31 - 1, x))


def pos2rid(chr_off, l_pac: int, pos_f: int) -> int:
    if pos_f >= l_pac:
        return -1
    left, right, mid = 0, len(chr_off), 0
    while left < right:
        mid = (left + right) >> 1
        if pos_f >= chr_off[mid]:
            if mid == len(chr_off) - 1:
                break
            if pos_f < chr_off[mid + 1]:
                break
            left = mid + 1
        else:
            right = mid
    return mid


def get_seq(pac, l_pac: int, beg: int, end: int) -> list[int]:
    if end < beg:
        beg, end = end, beg
    end = min(end, l_pac << 1)
    beg = max(beg, 0)
    if beg >= l_pac or end <= l_pac:
        if beg >= l_pac:
            beg_f, end_f = (l_pac << 1) - 1 - end, (l_pac << 1) - 1 - beg
            fwd = [get_pac(pac, p) for p in range(beg_f + 1, end_f + 1)]
            return [3 - b for b in reversed(fwd)]
        return [get_pac(pac, p) for p in range(beg, end)]
    return []


def infer_dir(l_pac: int, b1: int, b2: int):
    r1, r2 = int(b1 >= l_pac), int(b2 >= l_pac)
    p2 = b2 if r1 == r2 else (l_pac << 1) - 1 - b2
    dist = p2 - b1 if p2 > b1 else b1 - p2
    d = (0 if r1 == r2 else 1) ^ (0 if p2 > b1 else 3)
    return d, dist


def collect(opt: dict, bounds: list[dict], pac, l_pac: int, chr_off, chr_len, reads: list, alns: list,
            cands: list) -> list[dict]:
    """Jobs in order: dicts with cand, orientation, is_rev, rid, adj_rb, adj_re, query,
    target and xtra."""
    jobs = []
    for ci, c in enumerate(cands):
        own = alns[c["aln_first"]:c["aln_first"] + c["aln_count"]]
        best = max((a["score"] for a in own), default=0)
        thr = _sat_i32(best - opt["pen_unpaired"])
        above = sum(1 for a in own if a["score"] >= thr)
        if opt["max_matesw"] >= 0:
            above = min(above, opt["max_matesw"])
        if above == 0 or alns[c["primary"]]["score"] < thr:
            continue
        anc = c["anchor"]
        off = chr_off[anc["ref_id"]]

        def rb_of(a):
            g = off + a["pos"]
            return (l_pac << 1) - 1 - (g + a["ref_len"] - 1) if a["is_rev"] else g
        a_rb = rb_of(anc)
        skip = [bool(b["failed"]) for b in bounds]
        for a in own:
            if a["ref_id"] == anc["ref_id"]:
                d, dist = infer_dir(l_pac, a_rb, rb_of(a))
                if bounds[d]["low"] <= dist <= bounds[d]["high"]:
                    skip[d] = True
        if all(skip):
            continue
        read = reads[c["read"]]
        lms = len(read)
        for r in range(4):
            if skip[r]:
                continue
            is_rev = (r >> 1) != (r & 1)
            is_larger = (r >> 1) == 0
            lo, hi = bounds[r]["low"], bounds[r]["high"]
            if not is_rev:
                rb = a_rb + lo if is_larger else a_rb - hi
                re = (a_rb + hi if is_larger else a_rb - lo) + lms
            else:
                rb = (a_rb + lo if is_larger else a_rb - hi) - lms
                re = a_rb + hi if is_larger else a_rb - lo
            rb, re = max(rb, 0), min(re, l_pac << 1)
            if rb >= re:
                continue
            mid = (rb + re) >> 1
            mrev = mid >= l_pac
            rid = pos2rid(chr_off, l_pac, (l_pac << 1) - 1 - mid if mrev else mid)
            beg, end = rb, re
            if rid >= 0:
                fb, fe = chr_off[rid], chr_off[rid] + chr_len[rid]
                if mrev:
                    fb, fe = (l_pac << 1) - fe, (l_pac << 1) - fb
                beg, end = max(beg, fb), min(end, fe)
            if rid != anc["ref_id"] or end - beg < opt["min_seed_len"]:
                continue
            q = [(3 - b if b < 4 else 4) for b in reversed(read)] if is_rev else list(read)
            xtra = 0x40000 | 0x80000 | (opt["min_seed_len"] * opt["match_score"])
            if lms * opt["match_score"] < 250:
                xtra |= 0x10000
            jobs.append({"cand": ci, "orientation": r, "is_rev": int(is_rev), "rid": rid, "adj_rb": beg,
                         "adj_re": end, "query": q, "target": get_seq(pac, l_pac, beg, end), "xtra": xtra})
    return jobs
