"""The allocation-free extension entry point against the regular device entry point.

fa_ext_batch_device_noalloc serves callers that cannot let the library allocate
device memory (their memory is owned by a pool allocator, held to a fixed budget, or
the call sits on an allocation-free latency path); it keeps its scratch in a static
device array instead.  Every call shares that array, so the cases here are the ones
where it behaves differently from a context's own buffers: a single job, the largest
batch the array holds, a small call after a large one, and batches with invalid jobs
(which must be reported without any write past the output buffer).  This file is
collected last so that a run stopping at the first failure has run every other test
before it.
"""
import ctypes

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu
GUARD = 4096          # result words after the output that no call may touch
SENTINEL = -7


@pytest.fixture(scope="module")
def dev_batch(built):
    """The largest batch the array holds, on the device, with a guarded output buffer."""
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    b = synth.workload_ext_1m(N.FA_NOALLOC_MAX_JOBS, seed=77)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        d_jobs = torch.from_numpy(b.jobs.view(np.uint8)).to(dev)
        d_q = torch.from_numpy(b.qseq).to(dev)
        d_t = torch.from_numpy(b.tseq).to(dev)
        d_out = torch.full((len(b.jobs) * 6 + GUARD,), SENTINEL, dtype=torch.int32, device=dev)
    stream.synchronize()
    return b, d_jobs, d_q, d_t, d_out, stream


def regular(lib, p, d_jobs, n, d_q, d_t, stream):
    """fa_ext_batch_device's results for the first n jobs."""
    import torch
    d_ref = torch.zeros(n * 6, dtype=torch.int32, device=d_jobs.device)
    h = ctypes.c_void_p(stream.cuda_stream)
    with fa.Context(0) as ctx:
        N.check(lib.fa_ext_batch_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                        None, d_ref.data_ptr(), h))
        N.check(lib.fa_ctx_sync(ctx.handle))
    stream.synchronize()
    return d_ref.cpu()


def noalloc(lib, p, d_jobs, n, d_q, d_t, d_out, stream):
    d_out.fill_(SENTINEL)
    stream.synchronize()
    return lib.fa_ext_batch_device_noalloc(N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                           d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))


def guard_ok(d_out, n):
    return bool((d_out[n * 6:].cpu() == SENTINEL).all())


@pytest.mark.parametrize("n", [60_000, 1, N.FA_NOALLOC_MAX_JOBS])
def test_no_alloc_matches_device_entry_point(dev_batch, n):
    b, d_jobs, d_q, d_t, d_out, stream = dev_batch
    lib = N.load()
    p = fa.BandedPairWiseSW().to_struct()
    ref = regular(lib, p, d_jobs, n, d_q, d_t, stream)
    # two calls in a row: the second reuses the static scratch left by the first
    for _ in range(2):
        N.check(noalloc(lib, p, d_jobs, n, d_q, d_t, d_out, stream))
        got = d_out[:n * 6].cpu()
        assert (got == ref).all(), f"{int((got != ref).sum())} result words differ"
        assert guard_ok(d_out, n)
    if n <= 20_000:
        want, _ = O.ext_batch(p, b.jobs[:n], b.qseq, b.tseq)
        assert np.array_equal(got.numpy().view(N.EXT_RESULT_DT), want)


def test_small_call_after_a_large_one(dev_batch):
    """A 5,000-job call after the largest one: only indices below 5,000 may be processed
    (the scratch still holds the large call's order past them)."""
    b, d_jobs, d_q, d_t, d_out, stream = dev_batch
    lib = N.load()
    p = fa.BandedPairWiseSW().to_struct()
    N.check(noalloc(lib, p, d_jobs, N.FA_NOALLOC_MAX_JOBS, d_q, d_t, d_out, stream))
    n = 5000
    N.check(noalloc(lib, p, d_jobs, n, d_q, d_t, d_out, stream))
    want, _ = O.ext_batch(p, b.jobs[:n], b.qseq, b.tseq)
    assert np.array_equal(d_out[:n * 6].cpu().numpy().view(N.EXT_RESULT_DT), want)
    assert (d_out[n * 6:].cpu() == SENTINEL).all()


@pytest.mark.parametrize("field,value", [("qlen", -1), ("qlen", 0), ("h0", 0), ("h0", -3), ("tlen", -2)])
def test_invalid_jobs_are_reported(dev_batch, field, value):
    """A batch with invalid jobs (the reference panics on them) after a larger valid call:
    FA_ERR_ARG from both device entry points, no write past the output, and the next valid
    call is correct."""
    import torch
    b, d_jobs, d_q, d_t, d_out, stream = dev_batch
    lib = N.load()
    p = fa.BandedPairWiseSW().to_struct()
    N.check(noalloc(lib, p, d_jobs, 100_000, d_q, d_t, d_out, stream))
    n = 20_000
    jobs = b.jobs[:n].copy()
    bad = np.arange(3, n, 997)
    jobs[field][bad] = value
    d_bad = torch.from_numpy(jobs.view(np.uint8)).to(d_jobs.device)
    torch.cuda.synchronize()
    assert noalloc(lib, p, d_bad, n, d_q, d_t, d_out, stream) == N.FA_ERR_ARG
    assert guard_ok(d_out, n)
    h = ctypes.c_void_p(stream.cuda_stream)
    d_ref = torch.full((n * 6 + GUARD,), SENTINEL, dtype=torch.int32, device=d_jobs.device)
    with fa.Context(0) as ctx:
        N.check(lib.fa_ext_batch_device(ctx.handle, N.ptr(p), d_bad.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                        None, d_ref.data_ptr(), h))
        assert lib.fa_ctx_sync(ctx.handle) == N.FA_ERR_ARG
    assert bool((d_ref[n * 6:].cpu() == SENTINEL).all())
    N.check(noalloc(lib, p, d_jobs, n, d_q, d_t, d_out, stream))
    want, _ = O.ext_batch(p, b.jobs[:n], b.qseq, b.tseq)
    assert np.array_equal(d_out[:n * 6].cpu().numpy().view(N.EXT_RESULT_DT), want)


def test_no_alloc_rejects_oversized_batches(built):
    lib = N.load()
    p = fa.BandedPairWiseSW().to_struct()
    one = ctypes.c_void_p(8)   # never dereferenced: the size check comes first
    rc = lib.fa_ext_batch_device_noalloc(N.ptr(p), one, N.FA_NOALLOC_MAX_JOBS + 1, one, one, one, None)
    assert rc == N.FA_ERR_CAPACITY
    assert b"exceed the limit" in lib.fa_last_error()
