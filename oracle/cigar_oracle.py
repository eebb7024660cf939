"""CPU restatement of scalar_banded_swa (CIGAR regeneration) and infer_band_width.

Test infrastructure only: the parity checker of the CIGAR kernel
(ferrousalign_b200/csrc/cigar_kernel.cu).  Pure Python with the reference's full
(tlen+1) x (qlen+1) traceback matrix, restating
src/core/alignment/banded_swa/scalar/implementation.rs step by step:

* :17-47    empty query or target: zero OutScore, nothing else;
* :55-75    query profile (codes above 4 count as 4), first row h0, h0 - oe_ins, then -e_ins;
* :77-85    traceback edges: row 0 insertions, column 0 deletions, every other cell M;
* :97-227   rows: band [max(beg, i-w), min(end, i+w+1, qlen)), first column
            max(h0 - (o_del + e_del (i+1)), 0) when the band starts at 0, the match term
            clamped at 0, M >= E >= F tie order, first maximum of the row, E/F updates, the
            row end word, gscore at the query end, stop on a zero row or z-drop, and the
            beg/end rescans;
* :239-321  traceback from (max_i+1, max_j+1): runs of M, D and I with the aligned bases,
            at most 10000 steps, stop when a step makes no progress;
* :340-412  5' soft clip of the query left before the traceback's end, 3' soft clip or
            M run by gscore <= 0 or gscore <= score - pen_clip3.

CIGAR operations are returned as (op, len) with op in 'MIDS'; scores as a dict in
OutScore's order.  Parity is pinned against this restatement and hand-derived cases in the
tests; the reference's own tests of this function need the pipeline around it.
"""
from __future__ import annotations

import math

TB_M, TB_D, TB_I = 0, 1, 2


def _as_i32(x: float) -> int:
    if math.isnan(x):
        return 0
    return max(-2**31, min(2**31 - 1, int(x))) if math.isfinite(x) else (2**31 - 1 if x > 0 else -2**31)


def infer_band_width(l_query, l_ref, score, a, o_del, e_del, o_ins, e_ins, cmd_w, region_w) -> int:
    """region.rs:1277-1316."""
    def one(o, e):
        if l_query == l_ref and l_query * a - score < (o + e - a) * 2:
            return 0
        num = float(min(l_query, l_ref) * a - score - o)
        q = num / e if e != 0 else (math.inf if num > 0 else (-math.inf if num < 0 else math.nan))
        return max(_as_i32(q + 2.0), abs(l_query - l_ref))
    w2 = max(one(o_del, e_del), one(o_ins, e_ins))
    if w2 > cmd_w:
        w2 = min(w2, region_w)
    return min(w2, cmd_w * 4)


def banded_swa(p: dict, query, target, w: int, h0: int):
    """p: mat (25 ints, [target * 5 + query]), o_del, e_del, o_ins, e_ins, zdrop, pen_clip3.
    Returns (out_score dict, cigar [(op, len)], ref_aligned, query_aligned)."""
    qlen, tlen = len(query), len(target)
    zero = {"score": 0, "qle": 0, "tle": 0, "gtle": 0, "gscore": 0, "max_off": 0}
    if qlen == 0 or tlen == 0:
        return zero, [], [], []
    mat = p["mat"]
    oe_del, oe_ins = p["o_del"] + p["e_del"], p["o_ins"] + p["e_ins"]
    eh_h = [0] * (qlen + 1)
    eh_e = [0] * (qlen + 1)
    eh_h[0] = h0
    eh_h[1] = h0 - oe_ins if h0 > oe_ins else 0
    for j in range(2, qlen + 1):
        eh_h[j] = eh_h[j - 1] - p["e_ins"] if eh_h[j - 1] > p["e_ins"] else 0
    tb = [[TB_M] * (qlen + 1) for _ in range(tlen + 1)]
    for j in range(1, qlen + 1):
        tb[0][j] = TB_I
    for i in range(1, tlen + 1):
        tb[i][0] = TB_D
    max_score, max_i, max_j, max_ie, gscore, max_off = h0, -1, -1, -1, -1, 0
    beg, end = 0, qlen
    for i in range(tlen):
        tbase = min(int(target[i]), 4)
        cb, ce = beg, end
        if cb < i - w:
            cb = i - w
        if ce > i + w + 1:
            ce = i + w + 1
        if ce > qlen:
            ce = qlen
        h1 = max(h0 - (p["o_del"] + p["e_del"] * (i + 1)), 0) if cb == 0 else 0
        f, m_val, mj = 0, 0, -1
        for j in range(cb, ce):
            m = eh_h[j]
            e = eh_e[j]
            eh_h[j] = h1
            m += mat[tbase * 5 + min(int(query[j]), 4)]
            if m < 0:
                m = 0
            if m >= e and m >= f:
                h, code = m, TB_M
            elif e >= f:
                h, code = e, TB_D
            else:
                h, code = f, TB_I
            h1 = h
            tb[i + 1][j + 1] = code
            if m_val < h:
                m_val, mj = h, j
            e = max(e - p["e_del"], max(m - oe_del, 0))
            eh_e[j] = e
            f = max(f - p["e_ins"], max(m - oe_ins, 0))
        eh_h[ce] = h1
        eh_e[ce] = 0
        if ce == qlen and gscore < h1:
            gscore, max_ie = h1, i
        if m_val == 0:
            break
        if m_val > max_score:
            max_score, max_i, max_j = m_val, i, mj
            max_off = max(max_off, abs(mj - i))
        elif p["zdrop"] > 0:
            di, dj = i - max_i, mj - max_j
            if di > dj:
                if max_score - m_val - (di - dj) * p["e_del"] > p["zdrop"]:
                    break
            elif max_score - m_val - (dj - di) * p["e_ins"] > p["zdrop"]:
                break
        nb = cb
        while nb < ce and eh_h[nb] == 0 and eh_e[nb] == 0:
            nb += 1
        beg = nb
        ne = ce
        while ne >= beg and eh_h[ne] == 0 and eh_e[ne] == 0:
            ne -= 1
        end = min(ne + 2, qlen)
    cigar, ra, qa = [], [], []
    ci, cj = max_i + 1, max_j + 1
    steps = 0
    while ci > 0 or cj > 0:
        if steps >= 10000:
            break
        steps += 1
        pi, pj = ci, cj
        code = tb[ci][cj]
        cnt = 0
        if code == TB_M:
            while ci > 0 and cj > 0 and tb[ci][cj] == TB_M:
                ra.append(int(target[ci - 1]))
                qa.append(int(query[cj - 1]))
                ci, cj, cnt = ci - 1, cj - 1, cnt + 1
            if cnt:
                cigar.append(("M", cnt))
        elif code == TB_D:
            while ci > 0 and tb[ci][cj] == TB_D:
                ra.append(int(target[ci - 1]))
                ci, cnt = ci - 1, cnt + 1
            if cnt:
                cigar.append(("D", cnt))
        elif code == TB_I:
            while cj > 0 and tb[ci][cj] == TB_I:
                qa.append(int(query[cj - 1]))
                cj, cnt = cj - 1, cnt + 1
            if cnt:
                cigar.append(("I", cnt))
        else:
            break
        if ci == pi and cj == pj:
            break
    cigar.reverse()
    ra.reverse()
    qa.reverse()
    qs, qe = cj, max_j + 1
    final = ([("S", qs)] if qs > 0 else []) + cigar
    if qe < qlen:
        clip = gscore <= 0 or gscore <= max_score - p["pen_clip3"]
        final.append(("S" if clip else "M", qlen - qe))
    out = {"score": max_score, "qle": max_j + 1, "tle": max_i + 1, "gtle": max_ie + 1, "gscore": gscore,
           "max_off": max_off}
    return out, final, ra, qa
