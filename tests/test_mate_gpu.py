"""Mate-rescue kernel parity: ksw_align2 semantics through the C ABI against the oracle."""
import json
from pathlib import Path

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def diff_report(a, b):
    bad = np.nonzero(a != b)[0]
    return f"{len(bad)} mismatches, first {bad[:5]}: gpu={a[bad[:3]]} oracle={b[bad[:3]]}"


@pytest.mark.parametrize("case", json.loads((GOLD / "mate_cases.json").read_text()), ids=lambda c: c["name"])
def test_golden_case(ctx, case):
    p = fa.make_mate_params(case["mat"], case["o_del"], case["e_del"], case["o_ins"], case["e_ins"])
    jobs = np.zeros(1, N.MATE_JOB_DT)
    jobs[0] = (0, 0, len(case["query"]), len(case["target"]), case["xtra"], 0)
    q = np.array(case["query"], np.uint8)
    t = np.array(case["target"] if case["target"] else [0], np.uint8)
    out, _ = fa.mate_sw_batch(p, jobs, q, t, ctx=ctx)
    assert list(out[0]) == case["expect"]


def test_mate_workload_bit_exact(ctx):
    b = synth.workload_mate(20_000)
    p = fa.make_mate_params()
    out, stats = fa.mate_sw_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)
    ref, cells = O.mate_batch(p, b.jobs, b.qseq, b.tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert stats["cells"] == cells.sum()


def test_i16_lanes_and_random_flags_bit_exact(ctx):
    ref_seq = synth.reference(2_000_000, seed=8, n_rate=0.005)
    b = synth.mate_jobs(ref_seq, 4000, seed=9, read_len=200, insert_sd=30.0, sub_rate=0.03, indel_rate=0.01)
    rng = np.random.default_rng(1)
    flags = rng.choice([0, N.KSW_XSTART, N.KSW_XSUBO | N.KSW_XSTART | 19, N.KSW_XSUBO | 40, N.KSW_XBYTE,
                        N.KSW_XBYTE | N.KSW_XSTART | N.KSW_XSUBO | 19], size=len(b.jobs))
    b.jobs["xtra"] = flags.astype(np.uint32)
    for mat in (fa.MATE_RESCUE_SCORING_MATRIX, fa.bwa_fill_scmat(2, 3, -1)):
        p = fa.make_mate_params(mat, 5, 2, 4, 1)
        out, _ = fa.mate_sw_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)
        ref, _ = O.mate_batch(p, b.jobs, b.qseq, b.tseq)
        assert np.array_equal(out, ref), diff_report(out, ref)


@pytest.mark.parametrize("qlen", [125, 126])
def test_short_form_boundary_bit_exact(ctx, qlen):
    """Match 2 / mismatch -3 (shift 3): 125-base queries keep (qlen + 1) * 2 + 3 <= 255, the
    batch takes the unsaturated u8 form; 126-base queries do not, and an exact copy of the
    query in the window scores 252, which saturates (score 255) in the u8 engine."""
    rng = np.random.default_rng(qlen)
    qs, ts, jobs = [], [], np.zeros(600, N.MATE_JOB_DT)
    qo = to = 0
    for k in range(len(jobs)):
        q = rng.integers(0, 4, qlen).astype(np.uint8)
        t = rng.integers(0, 5, 400).astype(np.uint8)
        if k % 3 == 0:
            pos = int(rng.integers(0, 400 - qlen))
            t[pos:pos + qlen] = q
            if k % 2 == 0:
                t[pos + qlen // 2] = (q[qlen // 2] + 1) % 4
        jobs[k] = (qo, to, qlen, len(t), N.KSW_XBYTE | N.KSW_XSTART | N.KSW_XSUBO | 30, 0)
        qs.append(q); ts.append(t); qo += qlen; to += len(t)
    qseq, tseq = np.concatenate(qs), np.concatenate(ts)
    p = fa.make_mate_params(fa.bwa_fill_scmat(2, 3, -1), 6, 1, 6, 1)
    out, _ = fa.mate_sw_batch(p, jobs, qseq, tseq, ctx=ctx)
    ref, _ = O.mate_batch(p, jobs, qseq, tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert (ref["score"] == 255).any() == (qlen == 126)


def test_reference_style_interface(ctx):
    rng = np.random.default_rng(2)
    jobs = []
    for k in range(40):
        q = rng.integers(0, 4, 151).astype(np.uint8)
        t = np.concatenate([rng.integers(0, 4, 200), q, rng.integers(0, 4, 200)]).astype(np.uint8)
        jobs.append(fa.MateRescueJob(q, t, 151))
    res = fa.execute_mate_rescue_batch_with_engine(jobs)
    for k, r in enumerate(res):
        o = O.ksw_align2(jobs[k].query_seq, jobs[k].ref_seq, fa.MATE_RESCUE_SCORING_MATRIX, 6, 1, 6, 1,
                         fa.mate_xtra(151, 1, 19))
        assert (r.aln.score, r.aln.te, r.aln.qe, r.aln.score2, r.aln.te2, r.aln.tb, r.aln.qb) == tuple(o)
    assert fa.execute_mate_rescue_batch_with_engine([]) == []


def test_device_entry_point_matches_host_entry_point(ctx):
    import ctypes
    import torch
    b = synth.workload_mate(6000, seed=41)
    rng = np.random.default_rng(9)
    b.jobs["xtra"] = np.where(rng.random(len(b.jobs)) < 0.3, b.jobs["xtra"] & ~np.uint32(N.KSW_XBYTE),
                              b.jobs["xtra"]).astype(np.uint32)
    p = fa.make_mate_params()
    ref, st = fa.mate_sw_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)
    lib = N.load()
    dev = torch.device("cuda", 0)
    s = torch.cuda.Stream(dev)
    with torch.cuda.stream(s):
        d_jobs = torch.from_numpy(b.jobs.view(np.uint8)).to(dev)
        d_q = torch.from_numpy(b.qseq).to(dev)
        d_t = torch.from_numpy(b.tseq).to(dev)
        d_out = torch.zeros(len(b.jobs) * 7, dtype=torch.int32, device=dev)
    s.synchronize()
    N.check(lib.fa_mate_sw_batch_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), len(b.jobs), d_q.data_ptr(),
                                        d_t.data_ptr(), d_out.data_ptr(), ctypes.c_void_p(s.cuda_stream)))
    N.check(lib.fa_ctx_sync(ctx.handle))
    cells = ctypes.c_ulonglong()
    N.check(lib.fa_ctx_last_cells(ctx.handle, ctypes.byref(cells)))
    out = d_out.cpu().numpy().view(N.KSWR_DT).reshape(-1)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert cells.value == st["cells"]


def test_packed_input_equals_byte_input(ctx):
    """fa_mate_sw_batch_packed: the same records and cells as the byte form on the same
    bases (a reference with N runs, so reads and windows carry them); a bad run list fails."""
    ref_seq = synth.reference(3_000_000, seed=21, n_rate=0.01)
    b = synth.mate_jobs(ref_seq, 6000, seed=22, read_len=151, insert_sd=50.0, sub_rate=0.02, indel_rate=0.005)
    p = fa.make_mate_params()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    assert len(tp.runs) > 10
    got, st = fa.mate_sw_batch_packed(p, b.jobs, qp, tp, ctx=ctx)
    want, sw = fa.mate_sw_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)
    assert np.array_equal(got, want), diff_report(got, want)
    assert int(st["cells"]) == int(sw["cells"])
    r = tp.runs.copy()
    r[[0, 1]] = r[[1, 0]]
    with pytest.raises(N.NativeError) as e:
        fa.mate_sw_batch_packed(p, b.jobs, qp, fa.PackedSeq(tp.bases, tp.n_bases, r), ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG
    again, _ = fa.mate_sw_batch_packed(p, b.jobs[:100], qp, tp, ctx=ctx)
    assert np.array_equal(again, want[:100])


def test_sliced_host_batch(ctx):
    """A host batch of 32,768 jobs or more runs in job-index slices whose uploads overlap
    the kernels: results into a page-locked and into a pageable buffer equal the unsliced
    call's and the oracle's on a sample; a bad job in the last slice fails the call before
    anything runs, named by its index in the batch."""
    import torch
    b = synth.workload_mate(100_000, seed=29)
    mp = fa.make_mate_params()
    c = fa.Context(0)
    try:
        c.set_slices(1, 1)
        want, wst = fa.mate_sw_batch(mp, b.jobs, b.qseq, b.tseq, ctx=c)
        c.set_slices(-1, -1)
        pinned = torch.from_numpy(np.zeros(len(b.jobs), N.KSWR_DT).view(np.uint8)).pin_memory().numpy().view(N.KSWR_DT)
        for out in (pinned, None):
            got, st = fa.mate_sw_batch(mp, b.jobs, b.qseq, b.tseq, ctx=c, out=out)
            assert np.array_equal(got, want)
            assert int(st["cells"]) == int(wst["cells"])
        ref, _ = O.mate_batch(mp, b.jobs[:3000], b.qseq, b.tseq)
        assert np.array_equal(want[:3000], ref)
        bad = b.jobs.copy()
        bad["tlen"][97_123] = -1
        with pytest.raises(N.NativeError) as e:
            fa.mate_sw_batch(mp, bad, b.qseq, b.tseq, ctx=c)
        assert e.value.code == N.FA_ERR_ARG and "97123" in str(e.value)
    finally:
        c.close()


def test_sliced_packed_batch_with_n_runs(ctx):
    """The packed entry's sliced form (each slice's packed words uploaded, unpacked on the
    device with its N runs) equals the byte entry on a 100k-job batch whose sequences carry N
    bases and runs of N anywhere, slice boundaries included; bad runs are rejected."""
    b = synth.workload_mate(100_000, seed=33)
    q, t = b.qseq.copy(), b.tseq.copy()
    rng = np.random.default_rng(7)
    for buf in (q, t):
        for k in rng.choice(len(buf) - 8, 3000, replace=False):
            buf[k:k + int(rng.integers(1, 8))] = 4
    mp = fa.make_mate_params()
    want, wst = fa.mate_sw_batch(mp, b.jobs, q, t, ctx=ctx)
    qp, tp = fa.pack(q), fa.pack(t)
    got, st = fa.mate_sw_batch_packed(mp, b.jobs, qp, tp, ctx=ctx)
    assert np.array_equal(got, want)
    assert int(st["cells"]) == int(wst["cells"])
    bad = fa.PackedSeq(qp.bases, qp.n_bases, qp.runs[::-1].copy())
    with pytest.raises(N.NativeError) as e:
        fa.mate_sw_batch_packed(mp, b.jobs, bad, tp, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG


def test_sliced_batch_out_of_sequence_order(ctx):
    """Mate jobs in random order (a slice's jobs reach anywhere in the buffers): the sliced
    host path, byte and packed forms, still equals the unsliced call."""
    b = synth.workload_mate(60_000, seed=35)
    jobs = b.jobs[np.random.default_rng(2).permutation(len(b.jobs))]
    mp = fa.make_mate_params()
    c = fa.Context(0)
    try:
        c.set_slices(1, 1)
        want, _ = fa.mate_sw_batch(mp, jobs, b.qseq, b.tseq, ctx=c)
        c.set_slices(-1, -1)
        got, _ = fa.mate_sw_batch(mp, jobs, b.qseq, b.tseq, ctx=c)
        assert np.array_equal(got, want)
        got_p, _ = fa.mate_sw_batch_packed(mp, jobs, fa.pack(b.qseq), fa.pack(b.tseq), ctx=c)
        assert np.array_equal(got_p, want)
    finally:
        c.close()
