"""Graph mode: a policy or learned batch recorded as one CUDA graph and replayed gives
the same results, final bands and cell counts as the round-by-round path."""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import band_model as B
from ferrousalign_b200 import synth

pytestmark = pytest.mark.gpu


def test_graph_replays_match_round_by_round(ctx):
    p = fa.BandedPairWiseSW().to_struct()
    b1 = synth.workload_ext_1m(40_000, seed=501)
    b2 = synth.workload_ext_uneven(20_000, seed=502, ref_len=3_000_000)
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    ref1, st1, wf1 = fa.extend_batch(p, b1.jobs, b1.qseq, b1.tseq, policy=bwa, ctx=ctx)
    ref2, st2, wf2 = fa.extend_batch(p, b2.jobs, b2.qseq, b2.tseq, policy=bwa, ctx=ctx)
    g = N.Context(0)
    g.set_graph(True)
    try:
        # record, replay, another shape (re-record), and the first shape again
        for batch, ref, st, wf in ((b1, ref1, st1, wf1), (b1, ref1, st1, wf1), (b2, ref2, st2, wf2),
                                   (b1, ref1, st1, wf1)):
            out, gst, gwf = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, policy=bwa, ctx=g)
            assert np.array_equal(out, ref)
            assert np.array_equal(gwf, wf)
            assert gst["cells_executed"] == st["cells_executed"] and gst["retries"] == st["retries"]
    finally:
        g.close()


def test_graph_learned_matches(ctx):
    if not B.DEFAULT_MODEL.exists():
        pytest.skip("no trained model file")
    p = fa.BandedPairWiseSW().to_struct()
    b = synth.workload_ext_1m(50_000, seed=503)
    hints = B.hints_from_info(b.info)
    m = B.BandModel.load()
    ref, st, wf, wfin = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, ctx=ctx)
    g = N.Context(0)
    g.set_graph(True)
    try:
        for _ in range(2):
            out, gst, gwf, gwfin = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, ctx=g)
            assert np.array_equal(out, ref)
            assert np.array_equal(gwf, wf) and np.array_equal(gwfin, wfin)
            assert gst["cells_executed"] == st["cells_executed"]
            assert gst["retries"] == st["retries"] and gst["misses"] == st["misses"]
        # a different margin changes the recorded constants: re-recorded, still exact
        out2, _, _, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, margin=0.5, ctx=g)
        plain, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
        assert np.array_equal(out2, plain)
    finally:
        g.close()
