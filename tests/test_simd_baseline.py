"""The reference's SIMD CPU path restated (oracle/simd_baseline.cpp), the timed CPU baseline.

Its outputs are the reference SIMD kernels' own (score and 0-based ends; for the mate SW
the Kswr record with an estimated tb/qb), not ksw_extend2's, so it is checked the way the
reference checks those kernels:
- the assertions of tests/kernel_optimization_test.rs on the int8 kernel (identical
  sequences end at len - 1 with a positive score, partial matches and varying lengths stay
  inside their lanes, mismatches never go negative);
- the int16 kernel gives identical lanes on the AVX2 (16 lanes), AVX-512BW (32 lanes) and a
  portable lane-by-lane (8 lanes) engine;
- the mate-rescue kernel's score / te / qe on AVX2 (32 lanes) and AVX-512BW (64 lanes) agree,
  and score / te equal the ksw_align2 restatement's wherever the u8 score does not saturate
  and no N faces an N (kswv scores N/N as a match through its XOR table,
  kswv_avx2.rs:126-146); qe as well while the score stays below 128.
"""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O
from oracle import simd_baseline as S


@pytest.fixture(scope="module")
def lib(built):
    return S.load()


def chunk(seq_q, seq_t, qlen, tlen, max_len):
    lanes = len(qlen)
    q = np.zeros((max_len, lanes), np.uint8)
    t = np.zeros((max_len, lanes), np.uint8)
    for pos in range(max_len):
        for ln in range(lanes):
            q[pos, ln] = seq_q(pos, ln)
            t[pos, ln] = seq_t(pos, ln)
    p = fa.BandedPairWiseSW().to_struct()
    return S.i8_chunk(q.reshape(-1), t.reshape(-1), qlen, tlen, [0] * lanes, [10] * lanes, max_len, max_len, p)


def test_i8_identical_sequences(lib):
    """kernel_optimization_test.rs:47-110: ACGTACGTAC against itself, 16 lanes."""
    out = chunk(lambda p, l: p % 4, lambda p, l: p % 4, [10] * 16, [10] * 16, 10)
    assert (out["score"] > 0).all()
    assert (out["qe"] == 9).all() and (out["te"] == 9).all()


def test_i8_complete_mismatch_and_saturation(lib):
    """kernel_optimization_test.rs:112-160, :340-400: all-A against all-T stays at 0; AAA then
    TTT against all A never goes negative."""
    out = chunk(lambda p, l: 0, lambda p, l: 3, [8] * 16, [8] * 16, 8)
    assert (out["score"] >= 0).all() and (out["score"] <= 0).all()
    out = chunk(lambda p, l: 0, lambda p, l: 0 if p < 3 else 3, [6] * 16, [6] * 16, 6)
    assert (out["score"] >= 0).all() and (out["qe"] >= 0).all() and (out["te"] >= 0).all()
    assert (out["score"] == 3).all()


def test_i8_partial_and_varying_lengths(lib):
    """kernel_optimization_test.rs:162-280: a partial match scores > 0; lanes of lengths 4-11
    end inside their own lengths."""
    out = chunk(lambda p, l: 0 if p < 4 else p % 4, lambda p, l: p % 4, [10] * 16, [10] * 16, 10)
    assert (out["score"] > 0).all()
    ql = [4 + ln // 2 for ln in range(16)]
    out = chunk(lambda p, l: p % 4, lambda p, l: p % 4, ql, ql, 12)
    assert (out["score"] > 0).all()
    assert (out["qe"] <= np.array(ql) - 1).all()


def test_i16_widths_agree(lib):
    b = synth.workload_ext_plain(4000)
    p = fa.BandedPairWiseSW().to_struct()
    outs = []
    for isa in ("port", "avx2") + (("avx512",) if S.cpu_has("avx512") else ()):
        o, bits = S.ext_batch(p, b.jobs, b.qseq, b.tseq, isa=isa)
        assert bits == 16     # 151-bp jobs: the int16 kernel
        outs.append(o)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    assert (outs[0]["score"] > 0).mean() > 0.99


def perfect_jobs(n, length, h0, w):
    rng = np.random.default_rng(4)
    q = rng.integers(0, 4, (n, length)).astype(np.uint8).reshape(-1)
    jobs = np.zeros(n, N.JOB_DT)
    jobs["q_off"] = jobs["t_off"] = np.arange(n) * length
    jobs["qlen"] = jobs["tlen"] = length
    jobs["h0"], jobs["w"], jobs["dir"] = h0, w, 1
    return jobs, q


@pytest.mark.parametrize("force_i16", [True, False])
def test_i16_matches_ksw_extend2_on_unclipped_jobs(lib, force_i16):
    """Where neither kernel's rules bite (a perfect match inside the first row's band, no
    z-drop), the SIMD kernels' score and 0-based ends equal ksw_extend2's score and lengths - 1
    (90-bp jobs take the int8 kernel unless the int16 one is forced)."""
    jobs, q = perfect_jobs(64, 90, 20, 100)
    p = fa.BandedPairWiseSW().to_struct()
    out, bits = S.ext_batch(p, jobs, q, q, isa="avx2", force_i16=force_i16)
    ref, _ = O.ext_batch(p, jobs, q, q)
    assert bits == (16 if force_i16 else 8)
    assert (ref["score"] == 110).all()
    assert np.array_equal(out["score"], ref["score"])
    assert np.array_equal(out["te"] + 1, ref["tle"]) and np.array_equal(out["qe"] + 1, ref["qle"])


def test_i16_band_end_never_grows(lib):
    """kernel_i16.rs:149-161 stores each row's clamped band end and takes the next row's from
    it, so no row reaches past column w: a 140-bp perfect match at w = 100 stops at column 100
    (score h0 + 101), where ksw_extend2's adaptive band goes on to h0 + 140."""
    jobs, q = perfect_jobs(32, 140, 20, 100)
    p = fa.BandedPairWiseSW().to_struct()
    out, _ = S.ext_batch(p, jobs, q, q, isa="avx2")
    ref, _ = O.ext_batch(p, jobs, q, q)
    assert (out["score"] == 121).all() and (out["qe"] == 100).all()
    assert (ref["score"] == 160).all()


def test_kswv_widths_agree_and_match_ksw_align2(lib):
    m = synth.workload_mate(3000)
    a = S.kswv_batch(m.jobs, m.qseq, m.tseq, isa="avx2")
    if S.cpu_has("avx512"):
        b = S.kswv_batch(m.jobs, m.qseq, m.tseq, isa="avx512")
        for f in ("score", "te", "qe"):
            assert np.array_equal(a[f], b[f])
    mp = fa.make_mate_params()
    ref, _ = O.mate_batch(mp, m.jobs, m.qseq, m.tseq)
    def has_n(buf, off, ln):
        return bool(np.any(buf[int(off):int(off) + int(ln)] == 4))
    nn = np.array([has_n(m.qseq, j["q_off"], j["qlen"]) and has_n(m.tseq, j["t_off"], j["tlen"]) for j in m.jobs])
    ok = (a["score"] < 250) & ~nn
    assert ok.mean() > 0.8
    for f in ("score", "te"):
        assert np.array_equal(a[f][ok], ref[f][ok]), f
    # ksw_align2's query-end search reads its u8 lanes as signed (ksw_affine_gap.rs:436-473,
    # restated as such), so the two agree on qe while the score stays below 128
    lo = ok & (a["score"] < 128)
    assert lo.sum() > 100 and np.array_equal(a["qe"][lo], ref["qe"][lo])
    assert ((a["qb"] == 0) | (a["score"] == 0)).all()    # qb estimated as 0 (kswv_avx2.rs:627-637)
