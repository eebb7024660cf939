"""CPU restatement of the extension-job collection (collect_extension_jobs_batch_soa).

Test infrastructure only: the parity checker of the job-collection kernels
(ferrousalign_b200/csrc/collect_kernel.cu).  Pure Python, restating step by step:

* chaining.rs:1108-1116   cal_max_gap, in floating point with Rust's saturating `as i32`;
* collect_soa.rs:74-91    chains not kept, or without seeds, give no jobs and no mappings;
* collect_soa.rs:97-122   the window [rmax0, rmax1): per seed, query_pos + cal_max_gap(query_pos)
  before it (saturating at 0) and the remaining query + cal_max_gap(remaining) after it;
  rmax1 capped at 2 l_pac; a window across l_pac is cut to the strand of the chain's first
  seed;
* bntseq.rs:451-535, 564-575  the window's bases from the packed reference (two bits per base,
  base k in bits 7-6 of byte k/4 for k % 4 == 0 ... bits 1-0 for k % 4 == 3; positions at or
  past l_pac are the reverse complement of forward position 2 l_pac - 1 - p);
* collect_soa.rs:140-215  seeds last to first: a left job when query_pos > 0 and
  0 < ref_pos - rmax0 <= window length (reversed read prefix, reversed window prefix,
  h0 = len * a), a right job when query_pos + len < read length and
  ref_pos + len - rmax0 < window length (read suffix, window suffix, h0 = 0); u64
  differences wrap as in a release build.

Job indices in the seed table run across the whole batch (the reference counts them per
read and indexes per-read score vectors with them: the same jobs).  Parity is pinned
against this restatement and hand-derived cases in the tests; the reference's own tests
of this function need a loaded index.
"""
from __future__ import annotations

import math

M64 = (1 << 64) - 1


def _as_i32(x: float) -> int:
    """Rust `f64 as i32`: truncation toward zero, saturating, NaN -> 0."""
    if math.isnan(x):
        return 0
    if x >= 2**31 - 1:
        return 2**31 - 1
    if x <= -2**31:
        return -2**31
    return int(x)


def cal_max_gap(opt: dict, qlen: int) -> int:
    def part(o, e):
        num = float(qlen * opt["a"] - o)
        q = num / e if e != 0 else (math.inf if num > 0 else (-math.inf if num < 0 else math.nan))
        return _as_i32(q + 1.0)
    l_del = part(opt["o_del"], opt["e_del"])
    l_ins = part(opt["o_ins"], opt["e_ins"])
    ln = l_del if l_del > l_ins else l_ins
    ln = ln if ln > 1 else 1
    return ln if ln < (opt["w"] << 1) else (opt["w"] << 1)


def get_pac(pac, pos: int) -> int:
    return (pac[pos >> 2] >> (((~pos) & 3) << 1)) & 3


def reference_segment(pac, l_pac: int, start: int, length: int) -> list[int]:
    end = start + length
    if start < l_pac < end:
        return []
    if start >= l_pac:
        beg_f, end_f = max(2 * l_pac - end, 0), max(2 * l_pac - start, 0)
        fwd = [get_pac(pac, p) for p in range(beg_f, end_f)]
        return [3 - b for b in reversed(fwd)]
    return [get_pac(pac, p) for p in range(start, end)]


def collect(opt: dict, pac, l_pac: int, reads: list, chains: list, seeds: list) -> dict:
    """reads: list of code lists; chains: dicts (read, seed_first, n_seeds, kept); seeds:
    dicts (ref_pos, query_pos, len).  Returns left/right job lists (query, target, h0, w,
    dir), the seed table (dicts as fa_seed_ext), chain_first and the chain windows."""
    left, right, table, first, win = [], [], [], [0], []
    for ch in chains:
        sidx = list(range(ch["seed_first"], ch["seed_first"] + ch["n_seeds"]))
        if not ch["kept"] or not sidx:
            first.append(len(table))
            win.append((0, 0))
            continue
        q = reads[ch["read"]]
        qlen = len(q)
        r0, r1 = l_pac << 1, 0
        for k in sidx:
            s = seeds[k]
            lm = s["query_pos"] + cal_max_gap(opt, s["query_pos"])
            b = max(s["ref_pos"] - lm, 0)
            rem = qlen - s["query_pos"] - s["len"]
            e = s["ref_pos"] + s["len"] + rem + cal_max_gap(opt, rem)
            r0, r1 = min(r0, b), max(r1, e)
        r1 = min(r1, l_pac << 1)
        if r0 < l_pac < r1:
            if seeds[sidx[0]]["ref_pos"] < l_pac:
                r1 = l_pac
            else:
                r0 = l_pac
        rseq = reference_segment(pac, l_pac, r0, r1 - r0) if r1 > r0 else []
        win.append((r0, r1))
        for k in reversed(sidx):
            s = seeds[k]
            lj = rj = -1
            if s["query_pos"] > 0:
                tmp = (s["ref_pos"] - r0) & M64
                if 0 < tmp <= len(rseq):
                    lj = len(left)
                    left.append((q[:s["query_pos"]][::-1], rseq[:tmp][::-1], s["len"] * opt["a"], opt["w"], 0))
            qend = s["query_pos"] + s["len"]
            if qend < qlen:
                tmp = (s["ref_pos"] + s["len"] - r0) & M64
                if tmp < len(rseq):
                    rj = len(right)
                    right.append((q[qend:], rseq[tmp:], 0, opt["w"], 1))
            table.append({"ref_pos": s["ref_pos"], "query_pos": s["query_pos"], "len": s["len"], "left_job": lj,
                          "right_job": rj})
        first.append(len(table))
    return {"left": left, "right": right, "seed_ext": table, "chain_first": first, "chain_win": win}
