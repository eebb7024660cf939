"""The allocation-free extension entry point against the regular device entry point.

fa_ext_batch_device_noalloc serves callers that cannot let the library allocate
device memory (their memory is owned by a pool allocator, held to a fixed budget, or
the call sits on an allocation-free latency path); it keeps its scratch in a static
device array instead.  This file is collected last so that a run stopping at the first
failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth

pytestmark = pytest.mark.gpu


def test_no_alloc_matches_device_entry_point(built):
    import torch
    lib = N.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    b = synth.workload_ext_1m(60_000, seed=77)
    p = fa.BandedPairWiseSW().to_struct()
    n = len(b.jobs)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        d_jobs = torch.from_numpy(b.jobs.view(np.uint8)).to(dev)
        d_q = torch.from_numpy(b.qseq).to(dev)
        d_t = torch.from_numpy(b.tseq).to(dev)
        d_ref = torch.zeros(n * 6, dtype=torch.int32, device=dev)
        d_out = torch.full((n * 6,), -7, dtype=torch.int32, device=dev)
    stream.synchronize()
    h = ctypes.c_void_p(stream.cuda_stream)

    with fa.Context(0) as ctx:
        N.check(lib.fa_ext_batch_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                        None, d_ref.data_ptr(), h))
        N.check(lib.fa_ctx_sync(ctx.handle))
    stream.synchronize()
    ref = d_ref.cpu()

    # two calls in a row: the second reuses the static scratch left by the first
    for _ in range(2):
        d_out.fill_(-7)
        stream.synchronize()
        N.check(lib.fa_ext_batch_device_noalloc(N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                                d_out.data_ptr(), h))
        got = d_out.cpu()
        assert torch.equal(got, ref), f"{int((got != ref).sum())} result words differ"


def test_no_alloc_rejects_oversized_batches(built):
    lib = N.load()
    p = fa.BandedPairWiseSW().to_struct()
    one = ctypes.c_void_p(8)   # never dereferenced: the size check comes first
    rc = lib.fa_ext_batch_device_noalloc(N.ptr(p), one, N.FA_NOALLOC_MAX_JOBS + 1, one, one, one, None)
    assert rc == N.FA_ERR_CAPACITY
    assert b"exceed the limit" in lib.fa_last_error()
