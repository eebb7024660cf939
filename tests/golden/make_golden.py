"""Generates the golden fixtures of tests/golden/ from an independent pure-Python
restatement of the reference's algorithms.

The reference (Rust) cannot be built or imported in this image, so its outputs cannot
be recorded directly.  This file restates, in plain Python with no shared code with
the C oracle or the CUDA kernels:
  ksw_extend2  src/core/alignment/ksw_affine_gap.rs:952-1169
  ksw_align2   src/core/alignment/ksw_affine_gap.rs:773-861 with the u8/i16 striped
               kernels it runs (ksw_u8_impl :267-494, ksw_i16_impl :503-735) on the
               128-bit engine (16 u8 / 8 i16 lanes)
and records seeded small cases.  Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import random
from pathlib import Path

HERE = Path(__file__).resolve().parent


# ---------------------------------------------------------------- ksw_extend2
def ksw_extend2(query, target, mat, o_del, e_del, o_ins, e_ins, w, end_bonus, zdrop, h0, m=5):
    assert h0 > 0 and len(query) > 0
    qlen, tlen = len(query), len(target)
    oe_del, oe_ins = o_del + e_del, o_ins + e_ins
    qp = [mat[k * m + query[j]] for k in range(m) for j in range(qlen)]
    H = [0] * (qlen + 1)
    E = [0] * (qlen + 1)
    H[0] = h0
    H[1] = h0 - oe_ins if h0 > oe_ins else 0
    j = 2
    while j <= qlen and H[j - 1] > e_ins:
        H[j] = H[j - 1] - e_ins
        j += 1
    max_score = 0
    for v in mat[:m * m]:
        if v > max_score:
            max_score = v

    def as_i32(x):
        if math.isnan(x):
            return 0
        if x >= 2147483647:
            return 2147483647
        if x <= -2147483648:
            return -2147483648
        return int(x)  # truncation toward zero

    def div(a, b):
        if b == 0:
            return math.copysign(math.inf, a) if a != 0 else math.nan
        return a / b

    max_ins = max(as_i32(div(float(qlen * max_score + end_bonus - o_ins), float(e_ins)) + 1.0), 1)
    w = min(w, max_ins)
    max_del = max(as_i32(div(float(qlen * max_score + end_bonus - o_del), float(e_del)) + 1.0), 1)
    w = min(w, max_del)

    best, max_i, max_j, max_ie, gscore, max_off = h0, -1, -1, -1, -1, 0
    beg, end = 0, qlen
    for i in range(tlen):
        f = 0
        m_row = 0
        mj = -1
        base = target[i] * qlen
        if beg < i - w:
            beg = i - w
        if end > i + w + 1:
            end = i + w + 1
        if end > qlen:
            end = qlen
        h1 = max(h0 - (o_del + e_del * (i + 1)), 0) if beg == 0 else 0
        for j in range(beg, end):
            M, e = H[j], E[j]
            H[j] = h1
            M = M + qp[base + j] if M != 0 else 0
            h = max(M, e, f)
            h1 = h
            if m_row < h:
                mj, m_row = j, h
            E[j] = max(e - e_del, max(M - oe_del, 0))
            f = max(f - e_ins, max(M - oe_ins, 0))
        H[end] = h1
        E[end] = 0
        if beg <= qlen - 1 < end or end == qlen:
            h_end = h1 if end == qlen else H[qlen - 1]
            if gscore < h_end:
                gscore, max_ie = h_end, i
        if m_row == 0:
            break
        if m_row > best:
            best, max_i, max_j = m_row, i, mj
            max_off = max(max_off, abs(mj - i))
        elif zdrop > 0:
            di, dj = i - max_i, mj - max_j
            if di > dj:
                if best - m_row - (di - dj) * e_del > zdrop:
                    break
            elif best - m_row - (dj - di) * e_ins > zdrop:
                break
        nb = beg
        while nb < end and H[nb] == 0 and E[nb] == 0:
            nb += 1
        beg = nb
        ne = end
        while ne > beg and H[ne] == 0 and E[ne] == 0:
            ne -= 1
        end = min(ne + 2, qlen)
    return [best, max_j + 1, max_i + 1, max_ie + 1, gscore, max_off]


# ---------------------------------------------------------------- ksw_align2
XBYTE, XSTOP, XSUBO, XSTART = 0x10000, 0x20000, 0x40000, 0x80000


def _striped(query, target, mat, o_del, e_del, o_ins, e_ins, xtra, size, m=5):
    qlen = len(query)
    P = 16 if size == 1 else 8
    slen = (qlen + P - 1) // P
    mn = min(min(mat[:m * m]), 127)
    mx = max(max(mat[:m * m]), 0)
    shift = (256 - mn) & 0xFF
    qmax = mx & 0xFF
    u8 = size == 1

    def sat(x):
        if u8:
            return 0 if x < 0 else 255 if x > 255 else x
        return -32768 if x < -32768 else 32767 if x > 32767 else x

    # profile[a][k] for linear position k (striped storage order does not change values)
    prof = []
    for a in range(m):
        row = []
        for k in range(slen * P):
            s = mat[a * m + query[k]] if k < qlen else 0
            row.append(((s + shift) & 0xFF) if u8 else s)
        prof.append(row)
    minsc = xtra & 0xffff if xtra & XSUBO else 0x10000
    endsc = xtra & 0xffff if xtra & XSTOP else 0x10000
    n = slen * P
    pos = lambda j, l: j + l * slen  # noqa: E731
    H0 = [0] * n
    Ecol = [0] * n
    Hmax = [0] * n
    gmax, te = 0, -1
    b = []
    for i in range(tlen_of(target)):
        H1 = [0] * n
        fl = [0] * P
        mxl = [0] * P
        hl = [0] + [H0[pos(slen - 1, l - 1)] for l in range(1, P)]
        S = prof[target[i]]
        for j in range(slen):
            for l in range(P):
                k = pos(j, l)
                if u8:
                    h = sat(sat(hl[l] + S[k]) - shift)
                else:
                    h = sat(hl[l] + S[k])
                e = Ecol[k]
                h = max(h, e, fl[l])
                mxl[l] = max(mxl[l], h)
                H1[k] = h
                Ecol[k] = max(sat(e - e_del), sat(h - oe(o_del, e_del)))
                fl[l] = max(sat(fl[l] - e_ins), sat(h - oe(o_ins, e_ins)))
                hl[l] = H0[k]
        for _ in range(P):
            fl = [0] + fl[:-1]
            changed = False
            for j in range(slen):
                for l in range(P):
                    k = pos(j, l)
                    hb = H1[k]
                    hn = max(hb, fl[l])
                    H1[k] = hn
                    fl[l] = sat(fl[l] - e_ins)
                    changed |= hn != hb
            if not changed:
                break
        imax = max(mxl)
        if imax >= minsc:
            if not b or b[-1][1] + 1 != i:
                b.append([imax, i])
            elif b[-1][0] < imax:
                b[-1] = [imax, i]
        if imax > gmax:
            gmax, te = imax, i
            Hmax = list(H1)
            if (u8 and gmax + shift >= 255) or (not u8 and gmax >= 0x7FFF) or gmax >= endsc:
                break
        H0 = H1
    r = {"score": 0, "te": -1, "qe": -1, "score2": -1, "te2": -1, "tb": -1, "qb": -1}
    sat_v = 255 if u8 else 0x7FFF
    r["score"] = (gmax if gmax + shift < 255 else 255) if u8 else gmax
    r["te"] = te
    if r["score"] != sat_v:
        best_v, best_k = -1, -1
        for kk in range(n):
            seg, lane = kk // P, kk % P
            cand = seg + lane * slen
            if cand >= qlen:
                continue
            v = Hmax[pos(seg, lane)]
            v = (v - 256 if v >= 128 else v) if u8 else v  # lanes are read back as signed
            if v > best_v:
                best_v, best_k = v, cand
            elif v == best_v and cand < best_k:
                best_k = cand
        r["qe"] = best_k
        if b:
            iv = (r["score"] + qmax - 1) // qmax
            low, high = te - iv, te + iv
            for sc, row in b:
                if (row < low or row > high) and sc > r["score2"]:
                    r["score2"], r["te2"] = sc, row
    return r


def oe(o, e):
    return o + e


def tlen_of(t):
    return len(t)


def ksw_align2(query, target, mat, o_del, e_del, o_ins, e_ins, xtra):
    size = 1 if xtra & XBYTE else 2
    r = _striped(query, target, mat, o_del, e_del, o_ins, e_ins, xtra, size)
    find_start = bool(xtra & XSTART) and not (bool(xtra & XSUBO) and r["score"] < (xtra & 0xffff))
    if find_start and r["qe"] >= 0 and r["te"] >= 0:
        q2 = list(reversed(query[:r["qe"] + 1]))
        t2 = list(reversed(target[:r["te"] + 1])) + list(target[r["te"] + 1:])
        rr = _striped(q2, t2, mat, o_del, e_del, o_ins, e_ins, XSTOP | r["score"], size)
        if rr["score"] >= r["score"]:
            r["tb"] = r["te"] - rr["te"]
            r["qb"] = r["qe"] - rr["qe"]
    return [r[k] for k in ("score", "te", "qe", "score2", "te2", "tb", "qb")]


# ---------------------------------------------------------------- case generation
def bwa_mat(a, b, n):
    mat = [n] * 25
    for i in range(4):
        for j in range(4):
            mat[i * 5 + j] = a if i == j else -b
    return mat


def mutate(rng, seq, sub, indel):
    out = []
    for c in seq:
        u = rng.random()
        if u < indel / 2:
            continue
        if u < indel:
            out.append(rng.randrange(4))
        out.append(rng.randrange(4) if rng.random() < sub else c)
    return out


def ext_cases(rng):
    cases = []
    std = dict(mat=bwa_mat(1, 4, -1), o_del=6, e_del=1, o_ins=6, e_ins=1, end_bonus=5, zdrop=100)
    kat_mat = [1 if (i == j and i < 4) else -1 for i in range(5) for j in range(5)]
    for k in range(5):
        kat_mat[4 * 5 + k] = 0
        kat_mat[k * 5 + 4] = 0
    enc = lambda s: ["ACGT".index(c) if c in "ACGT" else 4 for c in s]  # noqa: E731
    kat = dict(mat=kat_mat, o_del=5, e_del=1, o_ins=5, e_ins=1, end_bonus=0)
    # the reference's own unit-test inputs (ksw_affine_gap.rs:1252-1358)
    for q, t, zd, name in [("ACGT", "ACGT", 100, "ref_simple_match"), ("ACGT", "ACCT", 100, "ref_mismatch"),
                           ("ACGGT", "ACGT", 100, "ref_insertion"), ("AAAAAAAAAA", "TTTTTTTTTT", 5, "ref_zdrop"),
                           ("ACGTAAAAACGT", "ACGTCGT", 100, "ref_large_indel")]:
        cases.append(dict(name=name, query=enc(q), target=enc(t), w=50, h0=10, zdrop=zd, **kat))
    cases.append(dict(name="ref_asym_gaps", query=enc("ACGT"), target=enc("ACGT"), mat=kat_mat, o_del=5, e_del=1,
                      o_ins=3, e_ins=2, w=50, end_bonus=0, zdrop=100, h0=10))
    cases.append(dict(name="ref_15bp_insertion", query=enc("AGCTAGCTAGGGGGGGGGGGGGGGGAGCTAGCTAGCTAGCTAGCT"),
                      target=enc("AGCTAGCTAGAGCTAGCTAGCTAGCTAGCT"), w=100, h0=10, zdrop=100, **kat))
    # edge cases
    cases.append(dict(name="tlen0", query=[0, 1, 2], target=[], w=100, h0=5, **std))
    cases.append(dict(name="qlen1", query=[2], target=[2, 2, 1], w=100, h0=3, **std))
    cases.append(dict(name="all_N", query=[4] * 20, target=[4] * 30, w=100, h0=20, **std))
    cases.append(dict(name="h0_small", query=[0, 1, 2, 3] * 5, target=[3, 2, 1, 0] * 6, w=100, h0=1, **std))
    cases.append(dict(name="h0_eq_oe", query=[0, 1] * 10, target=[0, 1] * 12, w=100, h0=7, **std))
    cases.append(dict(name="w0", query=[0, 1, 2, 3] * 4, target=[0, 1, 2, 3] * 5, w=0, h0=10, **std))
    cases.append(dict(name="w1", query=[0, 1, 2, 3] * 4, target=[0, 1, 3, 3] * 5, w=1, h0=10, **std))
    cases.append(dict(name="zdrop0", query=[0] * 30, target=[1] * 10 + [0] * 30, w=100, h0=30,
                      **{**std, "zdrop": 0}))
    cases.append(dict(name="ties", query=[0, 0, 0, 0, 0, 0], target=[0, 0, 0, 0, 0, 0, 0, 0], w=100, h0=4, **std))
    for k in range(40):
        ql = rng.randrange(1, 60)
        q = [rng.randrange(5) if rng.random() < 0.03 else rng.randrange(4) for _ in range(ql)]
        t = mutate(rng, q, 0.05, 0.05) + [rng.randrange(4) for _ in range(rng.randrange(0, 40))]
        if rng.random() < 0.3:
            t = [rng.randrange(4) for _ in range(rng.randrange(0, 80))]
        a, b = rng.choice([(1, 4), (2, 3), (1, 1), (3, 5)])
        od, ed, oi, ei = rng.choice([(6, 1, 6, 1), (5, 2, 3, 1), (0, 1, 0, 1), (4, 0, 4, 1), (6, 1, 4, 3)])
        cases.append(dict(name=f"rand{k}", query=q, target=t, mat=bwa_mat(a, b, rng.choice([-1, 0, -2])), o_del=od,
                          e_del=ed, o_ins=oi, e_ins=ei, w=rng.choice([1, 3, 10, 30, 100]),
                          end_bonus=rng.choice([0, 5]), zdrop=rng.choice([0, 5, 20, 100]),
                          h0=rng.randrange(1, 40)))
    for c in cases:
        c["expect"] = ksw_extend2(c["query"], c["target"], c["mat"], c["o_del"], c["e_del"], c["o_ins"],
                                  c["e_ins"], c["w"], c["end_bonus"], c["zdrop"], c["h0"])
    return cases


MATE_MAT = [1, -4, -4, -4, 0, -4, 1, -4, -4, 0, -4, -4, 1, -4, 0, -4, -4, -4, 1, 0, 0, 0, 0, 0, 0]


def mate_cases(rng):
    cases = []
    enc = lambda s: ["ACGT".index(c) if c in "ACGT" else 4 for c in s]  # noqa: E731
    kat_mat = [1 if (i == j and i < 4) else -1 for i in range(5) for j in range(5)]
    for k in range(5):
        kat_mat[4 * 5 + k] = 0
        kat_mat[k * 5 + 4] = 0
    # the reference's own ksw_align inputs (ksw_affine_gap.rs:1393-1497)
    cases.append(dict(name="ref_align_basic", query=enc("ACGTACGT"), target=enc("ACGTACGT"), mat=kat_mat,
                      o_del=5, e_del=1, o_ins=5, e_ins=1, xtra=0))
    cases.append(dict(name="ref_align_start", query=enc("ACGTACGT"), target=enc("ACGTACGT"), mat=kat_mat,
                      o_del=5, e_del=1, o_ins=5, e_ins=1, xtra=XSTART))
    cases.append(dict(name="ref_align_u8", query=enc("ACGT"), target=enc("ACGT"), mat=kat_mat,
                      o_del=5, e_del=1, o_ins=5, e_ins=1, xtra=XBYTE))
    cases.append(dict(name="ref_align_asym", query=enc("ACGTACGT"), target=enc("ACGTACGT"), mat=kat_mat,
                      o_del=5, e_del=1, o_ins=3, e_ins=2, xtra=0))
    for k in range(24):
        ql = rng.randrange(1, 70)
        q = [rng.randrange(4) if rng.random() > 0.02 else 4 for _ in range(ql)]
        pre = [rng.randrange(4) for _ in range(rng.randrange(0, 30))]
        post = [rng.randrange(4) for _ in range(rng.randrange(0, 30))]
        t = pre + mutate(rng, q, 0.04, 0.04) + post
        if rng.random() < 0.2:
            t = [rng.randrange(4) for _ in range(rng.randrange(1, 90))]
        byte = rng.random() < 0.6
        xtra = XSUBO | XSTART | (XBYTE if byte else 0) | rng.choice([0, 5, 19])
        if rng.random() < 0.15:
            xtra = XBYTE if byte else 0
        cases.append(dict(name=f"mrand{k}", query=q, target=t, mat=MATE_MAT, o_del=6, e_del=1, o_ins=6, e_ins=1,
                          xtra=xtra))
    for c in cases:
        c["expect"] = ksw_align2(c["query"], c["target"], c["mat"], c["o_del"], c["e_del"], c["o_ins"],
                                 c["e_ins"], c["xtra"])
    return cases


if __name__ == "__main__":
    rng = random.Random(20261203)
    (HERE / "ext_cases.json").write_text(json.dumps(ext_cases(rng)))
    (HERE / "mate_cases.json").write_text(json.dumps(mate_cases(rng)))
    print("wrote", HERE / "ext_cases.json", HERE / "mate_cases.json")
