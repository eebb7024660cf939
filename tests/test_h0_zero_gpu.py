"""h0 = 0 under FA_PARAM_H0_ZERO: the reference's job collection gives every right job h0 = 0
(src/pipelines/linear/batch_extension/collect_soa.rs:206), which ksw_extend2 asserts against
(src/core/alignment/ksw_affine_gap.rs:968).  With the flag the library runs the recurrence as
written; a batch collected exactly as the reference collects it goes through fa_ext_batch and
matches the oracle run with the same flag, for every kernel kind and for the pipelined host
path.  Without the flag the same batch is FA_ERR_ARG."""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def collected(built):
    from ferrousalign_b200 import collect as K, synth
    ref, reads, off, chains, seeds = synth.workload_chains(4000, ref_len=2_000_000)
    pac, l_pac = K.pack_reference(ref)
    return K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds)


@pytest.mark.parametrize("kernel", [N.FA_KERNEL_AUTO, N.FA_KERNEL_INT32, N.FA_KERNEL_ROWS2, N.FA_KERNEL_INT16X2])
def test_reference_right_jobs_run_as_written(collected, kernel):
    got = collected
    assert (got.right_jobs["h0"] == 0).all() and len(got.right_jobs) > 1000
    p = fa.BandedPairWiseSW(allow_h0_zero=True).to_struct()
    # the right jobs as collected, and the left and right jobs of the batch together
    both = np.concatenate([got.right_jobs, got.left_jobs])
    with fa.Context(0) as ctx:
        ctx.set_kernel(kernel)
        for jobs in (got.right_jobs, both):
            out, stats, _ = fa.extend_batch(p, jobs, got.qbuf, got.tbuf, ctx=ctx)
            ref, tr = O.ext_batch(p, jobs, got.qbuf, got.tbuf)
            assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]
            assert int(stats["cells"]) == int(tr["cells"].sum())
        # under the bwa-mem2 retry policy too (score 0 equals the previous try's h0: one run)
        pol = fa.make_policy(N.FA_POLICY_BWA, 2)
        out, _, _ = fa.extend_batch(p, both, got.qbuf, got.tbuf, policy=pol, ctx=ctx)
        ref, _, _, _ = O.ext_batch_policy(p, pol, both, got.qbuf, got.tbuf)
        assert np.array_equal(out, ref)


def test_pipelined_host_batch_with_h0_zero(built):
    """>= 32768 jobs take the pipelined host path (device-side validation)."""
    from ferrousalign_b200 import synth
    b = synth.workload_ext_1m(60_000, seed=21)
    jobs = b.jobs.copy()
    jobs["h0"][::3] = 0
    p0 = fa.BandedPairWiseSW().to_struct()
    p = fa.BandedPairWiseSW(allow_h0_zero=True).to_struct()
    with fa.Context(0) as ctx:
        with pytest.raises(N.NativeError) as e:
            fa.extend_batch(p0, jobs, b.qseq, b.tseq, ctx=ctx)
        assert e.value.code == N.FA_ERR_ARG
        out, _, _ = fa.extend_batch(p, jobs, b.qseq, b.tseq, ctx=ctx)
    ref, _ = O.ext_batch(p, jobs, b.qseq, b.tseq)
    assert np.array_equal(out, ref)
    assert (out["score"][::3] == 0).all()


def test_negative_h0_rejected_with_the_flag(built):
    from ferrousalign_b200 import synth
    b = synth.workload_ext_plain(100)
    jobs = b.jobs.copy()
    jobs["h0"][7] = -1
    p = fa.BandedPairWiseSW(allow_h0_zero=True).to_struct()
    with fa.Context(0) as ctx:
        with pytest.raises(N.NativeError) as e:
            fa.extend_batch(p, jobs, b.qseq, b.tseq, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG
