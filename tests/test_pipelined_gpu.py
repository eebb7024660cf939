"""The pipelined host batch (fa_ext_batch, >= 32,768 jobs) with pinned host buffers: the
sequences stream up in slices, and when each slice's jobs form one index range their
results come back as soon as the slice has run.  Bit-exact against the oracle with the
jobs in sequence order (every slice returns early) and shuffled (one copy at the end)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).pin_memory()
    return t, t.numpy().view(a.dtype)


@pytest.mark.parametrize("shuffle", [False, True])
def test_pinned_batch_matches_oracle(built, shuffle):
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, synth
    from oracle import ksw_oracle as O
    b = synth.workload_ext_1m(120_000, seed=77)
    jobs = b.jobs.copy()
    if shuffle:
        jobs = jobs[np.random.default_rng(3).permutation(len(jobs))]
    p = fa.BandedPairWiseSW().to_struct()
    keep = []
    tj, pj = pinned(jobs)
    tq, pq = pinned(b.qseq)
    tt, pt = pinned(b.tseq)
    to, out = pinned(np.zeros(len(jobs), N.EXT_RESULT_DT))
    keep += [tj, tq, tt, to]
    lib = N.load()
    ctx = N.Context(0)
    stats = np.zeros(1, N.STATS_DT)
    for _ in range(2):
        out[:] = np.zeros(1, N.EXT_RESULT_DT)
        N.check(lib.fa_ext_batch(ctx.handle, N.ptr(p), N.ptr(pj), len(pj), N.ptr(pq), pq.nbytes, N.ptr(pt),
                                 pt.nbytes, out.ctypes.data, N.ptr(stats)))
        ref, _ = O.ext_batch(p, jobs, b.qseq, b.tseq)
        assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]
    ctx.close()


def test_job_outside_its_slice_falls_back(built):
    """Jobs in sequence order except one early job whose query and target are the last
    job's: the streamed path finds it past its slice's uploaded bytes, drains, and hands
    the batch to the path that places each job by its sequences.  Single band against the
    oracle; the bwa-mem2 policy and the learned band against the unsliced call."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, band_model as B, synth
    from oracle import ksw_oracle as O
    b = synth.workload_ext_1m(120_000, seed=78)
    jobs = b.jobs.copy()
    for f in ("q_off", "qlen", "t_off", "tlen"):
        jobs[5][f] = jobs[-1][f]
    p = fa.BandedPairWiseSW().to_struct()
    keep = []
    tj, pj = pinned(jobs)
    tq, pq = pinned(b.qseq)
    tt, pt = pinned(b.tseq)
    to, out = pinned(np.zeros(len(jobs), N.EXT_RESULT_DT))
    keep += [tj, tq, tt, to]
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    model = B.BandModel.load()
    with fa.Context(0) as ctx:
        ctx.set_slices(1, 1)
        want_bwa = fa.extend_batch(p, jobs, b.qseq, b.tseq, policy=bwa, ctx=ctx)[0].copy()
        want_learned = B.extend_batch_learned(p, jobs, b.qseq, b.tseq, model, ctx=ctx)[0].copy()
        ctx.set_slices(-1, -1)
        fa.extend_batch(p, pj, pq, pt, ctx=ctx, out=out)
        ref, _ = O.ext_batch(p, jobs, b.qseq, b.tseq)
        assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]
        fa.extend_batch(p, pj, pq, pt, policy=bwa, ctx=ctx, out=out)
        assert np.array_equal(out, want_bwa)
        B.extend_batch_learned(p, pj, pq, pt, model, ctx=ctx, out=out)
        assert np.array_equal(out, want_learned)
