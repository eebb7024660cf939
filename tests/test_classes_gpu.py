"""Length-class launches with the int32 work on a side stream.

A whole-batch call sorts its jobs longest first and launches once per capacity class of
32 query columns.  With several classes, each two-row launch's overflow pass (jobs whose
h0 + qlen * max passes 255, every query past 254 columns among them) and every class past
the two-row kernel's columns run on a second stream, with one overflow list and count per
class, joined back before the policy step or the call's end.  These batches put many
jobs on that path -- reads up to 300 bases, seeds anywhere in the read, and a = 3 scoring
-- and compare every entry point that launches classes with the oracle: the host call
under the single-band and bwa-mem2 policies, its recorded-graph form (first call and
replay), and the device-resident call.
"""
import ctypes

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu


def diff_report(a, b):
    bad = np.nonzero(a != b)[0]
    return f"{len(bad)} mismatches, first {bad[:5]}: gpu={a[bad[:3]]} oracle={b[bad[:3]]}"


@pytest.fixture(scope="module")
def batch(built):
    ref_seq = synth.reference(8_000_000, seed=81, n_rate=0.002, repeat_frac=0.05)
    return synth.ext_jobs(ref_seq, 40_000, seed=82, read_len=(50, 300), seed_at_start=False, seed_len=(10, 60))


SCORINGS = {
    "bwa": fa.BandedPairWiseSW(),
    "a3": fa.BandedPairWiseSW(o_del=5, e_del=2, o_ins=3, e_ins=1, mat=fa.bwa_fill_scmat(3, 2, 0), zdrop=30),
}


def overflow_share(p, jobs):
    a = int(np.asarray(p["mat"]).max())
    return float(((jobs["h0"] + a * jobs["qlen"] > 255) | (jobs["qlen"] > 254)).mean())


@pytest.mark.parametrize("kernel", [N.FA_KERNEL_AUTO, N.FA_KERNEL_ROWS2])
@pytest.mark.parametrize("scoring", sorted(SCORINGS))
def test_single_band_classes_bit_exact(ctx, batch, kernel, scoring):
    p = SCORINGS[scoring].to_struct()
    assert overflow_share(p, batch.jobs) > 0.01        # the side stream has work
    assert len(np.unique((batch.jobs["qlen"] + 31) // 32)) >= 8
    ctx.set_kernel(kernel)
    ctx.set_slices(1, 1)
    try:
        out, st, _ = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, ctx=ctx)
    finally:
        ctx.set_slices(-1, -1)
        ctx.set_kernel(N.FA_KERNEL_AUTO)
    ref, tr = O.ext_batch(p, batch.jobs, batch.qseq, batch.tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert st["cells"] == tr["cells"].sum()


@pytest.mark.parametrize("kernel", [N.FA_KERNEL_AUTO, N.FA_KERNEL_ROWS2])
def test_bwa_policy_classes_match_oracle(ctx, batch, kernel):
    p = SCORINGS["bwa"].to_struct()
    pol = fa.make_policy(N.FA_POLICY_BWA, 2)
    ctx.set_kernel(kernel)
    ctx.set_slices(1, 1)
    try:
        out, st, wfin = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, policy=pol, ctx=ctx)
    finally:
        ctx.set_slices(-1, -1)
        ctx.set_kernel(N.FA_KERNEL_AUTO)
    ref, rwfin, rtries, _ = O.ext_batch_policy(p, pol, batch.jobs, batch.qseq, batch.tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert np.array_equal(wfin, rwfin)
    assert st["retries"] == (rtries - 1).sum()


@pytest.mark.parametrize("policy", ["single", "bwa"])
def test_graph_classes_first_call_and_replay(batch, policy):
    p = SCORINGS["bwa"].to_struct()
    pol = fa.make_policy(N.FA_POLICY_BWA, 2) if policy == "bwa" else None
    if pol is None:
        ref, _ = O.ext_batch(p, batch.jobs, batch.qseq, batch.tseq)
    else:
        ref, _, _, _ = O.ext_batch_policy(p, pol, batch.jobs, batch.qseq, batch.tseq)
    with fa.Context(0) as g:
        g.set_graph(True)
        g.set_kernel(N.FA_KERNEL_ROWS2)
        for _ in range(2):                      # records the graph, then replays it
            out, _, _ = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, policy=pol, ctx=g)
            assert np.array_equal(out, ref), diff_report(out, ref)


@pytest.mark.parametrize("scoring", sorted(SCORINGS))
def test_device_entry_classes_bit_exact(batch, scoring):
    import torch
    p = SCORINGS[scoring].to_struct()
    dev = torch.device("cuda", 0)
    d_jobs = torch.from_numpy(batch.jobs.view(np.uint8)).to(dev)
    d_q = torch.from_numpy(batch.qseq).to(dev)
    d_t = torch.from_numpy(batch.tseq).to(dev)
    n = len(batch.jobs)
    d_out = torch.zeros(n * 6, dtype=torch.int32, device=dev)
    lib = N.load()
    with fa.Context(0) as c:
        c.set_kernel(N.FA_KERNEL_ROWS2)
        torch.cuda.synchronize()
        N.check(lib.fa_ext_batch_device(c.handle, N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                        None, d_out.data_ptr(), ctypes.c_void_p(0)))
        N.check(lib.fa_ctx_sync(c.handle))
    out = d_out.cpu().numpy().view(N.EXT_RESULT_DT)
    ref, _ = O.ext_batch(p, batch.jobs, batch.qseq, batch.tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)


@pytest.mark.parametrize("graph", [False, True])
def test_learned_rounds_with_side_streams_match_oracle(batch, graph):
    """Learned rounds: each band group's int32 jobs and the retry rounds' start on side
    streams while the two-row launches skip them; same results, decisions and cells as the
    oracle's policy run."""
    p = SCORINGS["bwa"].to_struct()
    rng = np.random.default_rng(83)
    wf = rng.choice([2, 3, 4, 8, 16, 32, 48], size=len(batch.jobs)).astype(np.int32)
    with fa.Context(0) as c:
        c.set_graph(graph)
        c.set_kernel(N.FA_KERNEL_ROWS2)
        c.set_slices(1, 1)
        for judge in (N.FA_JUDGE_BOUND, N.FA_JUDGE_BOUND | N.FA_JUDGE_ONCE | N.FA_JUDGE_HINT):
            pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, judge, 1)
            ref, rwfin, _, rcells = O.ext_batch_policy(p, pol, batch.jobs, batch.qseq, batch.tseq, wf)
            for _ in range(2 if graph else 1):
                out, st, wfin = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, policy=pol, w_first=wf, ctx=c)
                assert np.array_equal(out, ref), diff_report(out, ref)
                assert np.array_equal(wfin, rwfin)
                assert st["cells_executed"] == rcells.sum()


def test_whole_batch_features_in_length_order(batch):
    """The whole-batch learned call computes the band features with its threads walking the
    length order; the first bands it predicts equal the sliced call's, whose features run in
    input order, and so do the results."""
    from ferrousalign_b200 import band_model as B
    p = SCORINGS["bwa"].to_struct()
    model = B.BandModel.load(B.UNEVEN_MODEL if B.UNEVEN_MODEL.exists() else B.DEFAULT_MODEL)
    hints = B.hints_from_info(batch.info)
    res = {}
    with fa.Context(0) as c:
        for slices in (1, 3):
            c.set_slices(slices, slices)
            res[slices] = B.extend_batch_learned(p, batch.jobs, batch.qseq, batch.tseq, model, hints=hints, ctx=c)
    (o1, _, wf1, wfin1), (o3, _, wf3, wfin3) = res[1], res[3]
    assert len(np.unique(wf1)) > 3
    assert np.array_equal(wf1, wf3)
    assert np.array_equal(wfin1, wfin3)
    assert np.array_equal(o1, o3), diff_report(o1, o3)
