"""fa_pair_batch: one submission of a batch's seed extensions and mate-rescue SW jobs gives
the results of the separate calls (fa_ext_batch_policy / fa_ext_batch_learned and
fa_mate_sw_batch), both halves bit-exact against the oracle on a small case."""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import band_model as B
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def work():
    b = synth.workload_ext_1m(40_000, seed=5)
    m = synth.workload_mate(8_000, seed=6)
    return b, m


@pytest.mark.parametrize("mode", [N.FA_POLICY_SINGLE, N.FA_POLICY_BWA])
def test_plain_pair_batch_equals_separate_calls(ctx, work, mode):
    b, m = work
    p = fa.BandedPairWiseSW().to_struct()
    mp = fa.make_mate_params()
    pol = fa.make_policy(mode, 2)
    ext, mate, st, mst = fa.pair_batch(p, b.jobs, b.qseq, b.tseq, mp, m.jobs, m.qseq, m.tseq, policy=pol, ctx=ctx)
    ext_ref, est, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, ctx=ctx)
    mate_ref, mst_ref = fa.mate_sw_batch(mp, m.jobs, m.qseq, m.tseq, ctx=ctx)
    assert np.array_equal(ext, ext_ref)
    assert np.array_equal(mate, mate_ref)
    assert st["cells"] == est["cells"] and mst["cells"] == mst_ref["cells"]
    assert mst["jobs"] == len(m.jobs) and mst["kernel_ms"] > 0


def test_pair_batch_bit_exact_against_oracle(ctx, work):
    b, m = work
    p = fa.BandedPairWiseSW().to_struct()
    mp = fa.make_mate_params()
    sel = slice(0, 3000)
    jobs, mjobs = b.jobs[sel], m.jobs[:1500]
    ext, mate, _, _ = fa.pair_batch(p, jobs, b.qseq, b.tseq, mp, mjobs, m.qseq, m.tseq, ctx=ctx)
    ref, _ = O.ext_batch(p, jobs, b.qseq, b.tseq)
    assert np.array_equal(ext, ref)
    mref, _ = O.mate_batch(mp, mjobs, m.qseq, m.tseq)
    assert np.array_equal(mate, mref)


def test_learned_pair_batch_equals_separate_calls(ctx, work):
    b, m = work
    p = fa.BandedPairWiseSW().to_struct()
    mp = fa.make_mate_params()
    model = B.BandModel.load()
    hints = B.hints_from_info(b.info)
    ext, mate, st, _ = fa.pair_batch(p, b.jobs, b.qseq, b.tseq, mp, m.jobs, m.qseq, m.tseq, model=model,
                                     hints=hints, ctx=ctx)
    ext_ref, est, _, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, model, hints=hints, ctx=ctx)
    plain, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    assert np.array_equal(ext, ext_ref)
    assert np.array_equal(ext, plain)
    mate_ref, _ = fa.mate_sw_batch(mp, m.jobs, m.qseq, m.tseq, ctx=ctx)
    assert np.array_equal(mate, mate_ref)


def test_empty_halves_and_policy_errors(ctx, work):
    b, m = work
    p = fa.BandedPairWiseSW().to_struct()
    mp = fa.make_mate_params()
    ext, mate, _, mst = fa.pair_batch(p, b.jobs[:0], b.qseq, b.tseq, mp, m.jobs[:100], m.qseq, m.tseq, ctx=ctx)
    assert len(ext) == 0 and mst["jobs"] == 100
    assert np.array_equal(mate, fa.mate_sw_batch(mp, m.jobs[:100], m.qseq, m.tseq, ctx=ctx)[0])
    ext, mate, st, _ = fa.pair_batch(p, b.jobs[:500], b.qseq, b.tseq, mp, m.jobs[:0], m.qseq, m.tseq, ctx=ctx)
    assert len(mate) == 0 and st["jobs"] == 500
    with pytest.raises(N.NativeError):
        fa.pair_batch(p, b.jobs[:10], b.qseq, b.tseq, mp, m.jobs[:10], m.qseq, m.tseq,
                      policy=fa.make_policy(N.FA_POLICY_LEARNED, 2), ctx=ctx)
    # the context stays usable after the rejected call
    ext, _, _, _ = fa.pair_batch(p, b.jobs[:10], b.qseq, b.tseq, mp, m.jobs[:10], m.qseq, m.tseq, ctx=ctx)
    assert np.array_equal(ext, fa.extend_batch(p, b.jobs[:10], b.qseq, b.tseq, ctx=ctx)[0])


def test_sliced_mate_half(ctx, work):
    """A mate half of 32,768 jobs or more runs in job-index slices on its own streams: the
    results and cell count equal the unsliced separate call's, and a bad mate job in the last
    slice fails the call, named by its index."""
    b, _ = work
    m = synth.workload_mate(60_000, seed=16)
    p = fa.BandedPairWiseSW().to_struct()
    mp = fa.make_mate_params()
    with fa.Context(0) as c1:
        c1.set_slices(1, 1)
        mate_ref, mst_ref = fa.mate_sw_batch(mp, m.jobs, m.qseq, m.tseq, ctx=c1)
    ext, mate, _, mst = fa.pair_batch(p, b.jobs, b.qseq, b.tseq, mp, m.jobs, m.qseq, m.tseq, ctx=ctx)
    assert np.array_equal(mate, mate_ref)
    assert mst["cells"] == mst_ref["cells"]
    assert np.array_equal(ext, fa.extend_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)[0])
    bad = m.jobs.copy()
    bad["qlen"][59_001] = 0
    with pytest.raises(N.NativeError) as e:
        fa.pair_batch(p, b.jobs, b.qseq, b.tseq, mp, bad, m.qseq, m.tseq, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG and "59001" in str(e.value)
