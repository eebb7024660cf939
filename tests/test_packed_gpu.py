"""2-bit packed input (fa_ext_batch_packed, fa_ext_batch_learned_packed,
fa_ext_batch_packed_device): the kernels read packed bases and N runs on the device and
must give exactly the byte-code path's results -- and so the oracle's -- on every path:
the serial and the pipelined host batch, the sliced retry-policy and learned rounds, every
kernel kind, and the device-resident entry point."""
import ctypes

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import band_model as B
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrich(built):
    """Uneven left/right jobs over a reference with 2% N (runs of N at job edges too)."""
    ref_seq = synth.reference(5_000_000, seed=31, n_rate=0.02, repeat_frac=0.05)
    return synth.ext_jobs(ref_seq, 40_000, seed=37, read_len=(30, 300), seed_at_start=False)


@pytest.fixture(scope="module")
def big(built):
    return synth.workload_ext_1m(120_000, seed=41)


@pytest.mark.parametrize("kernel", [N.FA_KERNEL_AUTO, N.FA_KERNEL_INT32, N.FA_KERNEL_ROWS2, N.FA_KERNEL_INT16X2])
def test_packed_equals_bytes_and_oracle(nrich, kernel):
    b = nrich
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    assert len(qp.runs) > 100 and len(tp.runs) > 100
    with fa.Context(0) as ctx:
        ctx.set_kernel(kernel)
        for sub in (b.jobs[:5000], b.jobs):            # serial path, then the pipelined one
            out, st, _ = fa.extend_batch_packed(p, sub, qp, tp, ctx=ctx)
            ref, tr = O.ext_batch(p, sub, b.qseq, b.tseq)
            assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]
            assert int(st["cells"]) == int(tr["cells"].sum())


@pytest.mark.parametrize("mode", ["bwa", "learned_w_first"])
def test_sliced_policy_rounds_match_serial(big, mode):
    """>= 32768 in-order jobs run the retry rounds slice by slice; the results, final bands
    and cell counts equal the serial byte-code path's (and the oracle's policy)."""
    b = big
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    if mode == "bwa":
        pol, wf = fa.make_policy(N.FA_POLICY_BWA, 2), None
    else:
        pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_LEARNED, 2)
        wf = np.random.default_rng(5).choice([2, 4, 8, 16, 100], len(b.jobs)).astype(np.int32)
    with fa.Context(0) as ctx:
        out_p, st_p, wfin_p = fa.extend_batch_packed(p, b.jobs, qp, tp, policy=pol, w_first=wf, ctx=ctx)
        out_b, st_b, wfin_b = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, w_first=wf, ctx=ctx)
    with fa.Context(0) as ctx:
        ctx.set_graph(True)          # graph mode takes the serial path: the reference run
        out_s, st_s, wfin_s = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, w_first=wf, ctx=ctx)
    assert np.array_equal(out_p, out_s) and np.array_equal(out_b, out_s)
    assert np.array_equal(wfin_p, wfin_s) and np.array_equal(wfin_b, wfin_s)
    for k in ("cells", "cells_executed", "retries", "misses"):
        assert int(st_p[k]) == int(st_s[k]) == int(st_b[k]), k
    sample = np.arange(0, len(b.jobs), 37)
    ref, _, _, _ = O.ext_batch_policy(p, pol, b.jobs[sample], b.qseq, b.tseq,
                                      w_first=None if wf is None else wf[sample])
    assert np.array_equal(out_p[sample], ref)


def test_learned_packed_matches_learned_bytes(big):
    b = big
    p = fa.BandedPairWiseSW().to_struct()
    model = B.BandModel.load()
    hints = B.hints_from_info(b.info)
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    with fa.Context(0) as ctx:
        lp, sp, wfp, wfinp = fa.extend_batch_learned_packed(p, b.jobs, qp, tp, model, hints=hints, ctx=ctx)
        lb, sb, wfb, wfinb = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, model, hints=hints, ctx=ctx)
        small = slice(0, 20_000)          # the serial learned path
        ls, _, wfs, _ = fa.extend_batch_learned_packed(p, b.jobs[small], qp, tp, model, hints=hints[small], ctx=ctx)
        plain, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    assert np.array_equal(wfp, wfb) and np.array_equal(wfs, wfb[small])    # same features, same bands
    assert np.array_equal(lp, lb) and np.array_equal(wfinp, wfinb)
    assert np.array_equal(lp, plain) and np.array_equal(ls, plain[small])  # exact: the plain policy's results
    assert int(sp["misses"]) == int(sb["misses"]) and int(sp["cells_executed"]) == int(sb["cells_executed"])


@pytest.mark.parametrize("slices", [(2, 3), (5, 8), (1, 1), (-1, -1)])
def test_slice_counts_give_identical_results(big, slices):
    """fa_ctx_set_slices changes only how copies and kernels overlap: single-band, retry and
    learned results and cell counts are the same for every slice count."""
    b = big
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    model = B.BandModel.load()
    hints = B.hints_from_info(b.info)
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    with fa.Context(0) as ctx:
        want = [fa.extend_batch_packed(p, b.jobs, qp, tp, ctx=ctx),
                fa.extend_batch_packed(p, b.jobs, qp, tp, policy=bwa, ctx=ctx),
                fa.extend_batch_learned_packed(p, b.jobs, qp, tp, model, hints=hints, ctx=ctx)]
        ctx.set_slices(*slices)
        got = [fa.extend_batch_packed(p, b.jobs, qp, tp, ctx=ctx),
               fa.extend_batch_packed(p, b.jobs, qp, tp, policy=bwa, ctx=ctx),
               fa.extend_batch_learned_packed(p, b.jobs, qp, tp, model, hints=hints, ctx=ctx)]
        with pytest.raises(N.NativeError):
            ctx.set_slices(9, 0)
    for g, w in zip(got, want):
        assert np.array_equal(g[0], w[0])
        assert int(g[1]["cells_executed"]) == int(w[1]["cells_executed"])


def test_out_of_order_jobs_fall_back(big):
    """Jobs whose sequences are not in job order cannot be sliced: the serial path runs."""
    b = big
    p = fa.BandedPairWiseSW().to_struct()
    perm = np.random.default_rng(9).permutation(len(b.jobs))
    jobs = b.jobs[perm]
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    pol = fa.make_policy(N.FA_POLICY_BWA, 2)
    out, _, _ = fa.extend_batch_packed(p, jobs, qp, tp, policy=pol)
    want, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol)
    assert np.array_equal(out, want[perm])


def test_packed_device_entry(nrich):
    import torch
    b = nrich
    lib = N.load()
    dev = torch.device("cuda", 0)
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    n = len(b.jobs)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to(dev)  # noqa: E731
    d_jobs, d_qb, d_tb, d_qr, d_tr = t(b.jobs), t(qp.bases), t(tp.bases), t(qp.runs), t(tp.runs)
    dq = np.zeros(1, N.PACKED_SEQ_DT)
    dq[0] = (d_qb.data_ptr(), qp.n_bases, d_qr.data_ptr(), len(qp.runs))
    dt = np.zeros(1, N.PACKED_SEQ_DT)
    dt[0] = (d_tb.data_ptr(), tp.n_bases, d_tr.data_ptr(), len(tp.runs))
    d_out = torch.zeros(n * 6, dtype=torch.int32, device=dev)
    with fa.Context(0) as ctx:
        N.check(lib.fa_ext_batch_packed_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), n, N.ptr(dq), N.ptr(dt),
                                               None, d_out.data_ptr(), None))
        N.check(lib.fa_ctx_sync(ctx.handle))
    got = d_out.cpu().numpy().view(N.EXT_RESULT_DT)
    ref, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    assert np.array_equal(got, ref)


def test_bad_runs_rejected(nrich):
    b = nrich
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    for bad in ("unsorted", "outside", "empty"):
        r = qp.runs.copy()
        if bad == "unsorted":
            r[[0, 1]] = r[[1, 0]]
        elif bad == "outside":
            r[-1]["len"] = qp.n_bases
        else:
            r[3]["len"] = 0
        q2 = fa.PackedSeq(qp.bases, qp.n_bases, r)
        with pytest.raises(N.NativeError) as e:
            fa.extend_batch_packed(p, b.jobs[:100], q2, tp)
        assert e.value.code == N.FA_ERR_ARG


def test_streamed_n_rich_batches_equal_unsliced(nrich):
    """The streamed host path on the N-rich packed batch (N runs across slice boundaries, left
    and right jobs of 30-300 bases): single band, bwa-mem2 policy and learned band give the
    unsliced call's results, cells and bands."""
    b = nrich
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    model = B.BandModel.load()
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    with fa.Context(0) as ctx:
        def run():
            return [fa.extend_batch_packed(p, b.jobs, qp, tp, ctx=ctx),
                    fa.extend_batch_packed(p, b.jobs, qp, tp, policy=bwa, ctx=ctx),
                    fa.extend_batch_learned_packed(p, b.jobs, qp, tp, model, ctx=ctx)]
        ctx.set_slices(1, 1)
        want = run()
        for slices in ((-1, -1), (8, 8), (2, 2)):
            ctx.set_slices(*slices)
            got = run()
            for g, w in zip(got, want):
                assert np.array_equal(g[0], w[0]), slices
                assert int(g[1]["cells_executed"]) == int(w[1]["cells_executed"]), slices
            assert np.array_equal(got[1][2], want[1][2]) and np.array_equal(got[2][3], want[2][3])


def test_streamed_batch_at_the_threshold():
    """Exactly 32,768 jobs in eight slices (the smallest about a thousand jobs): byte and packed
    forms, single band and bwa-mem2 policy, equal to the unsliced call."""
    b = synth.workload_ext_1m(32_768, seed=55)
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    with fa.Context(0) as ctx:
        def run():
            return [fa.extend_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)[0].copy(),
                    fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=bwa, ctx=ctx)[0].copy(),
                    fa.extend_batch_packed(p, b.jobs, qp, tp, ctx=ctx)[0].copy(),
                    fa.extend_batch_packed(p, b.jobs, qp, tp, policy=bwa, ctx=ctx)[0].copy()]
        ctx.set_slices(1, 1)
        want = run()
        ctx.set_slices(8, 8)
        got = run()
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
