"""One device-resident extension batch of the bench workload, for ncu captures.

Usage: python -m ferrousalign_b200.profile_run [n_jobs] [probe|uneven|-] [kernel: 0 auto, 1 int32, 2 int16x2, 3 rows2]
       [reps] [threads per block]   (uneven: the 50-300 bp mixed left/right workload)
       python -m ferrousalign_b200.profile_run learned [n_jobs] [reps] [kernel] [uneven]
       python -m ferrousalign_b200.profile_run learned [n_jobs] [reps] [kernel]   (learned-band path)
       python -m ferrousalign_b200.profile_run bands [n_jobs]            (single runs at fixed bands)
       python -m ferrousalign_b200.profile_run mate [n_jobs] [reps]      (mate-rescue SW, device-resident)
       python -m ferrousalign_b200.profile_run regions [n_chains] [reps] (region merge, device-resident)
       python -m ferrousalign_b200.profile_run collect [n_reads] [reps]  (extension jobs from chains)
       python -m ferrousalign_b200.profile_run cigar [n_jobs] [reps]     (CIGAR regeneration)
       python -m ferrousalign_b200.profile_run rescue [n_pairs] [reps]   (mate-rescue jobs from anchors)
"""
import ctypes
import sys

import numpy as np
import torch

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N, synth

if len(sys.argv) > 1 and sys.argv[1] == "mate":
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 500_000
    m = synth.workload_mate(n)
    mp = fa.make_mate_params()
    ctx = fa.Context(0)
    lib = N.load()
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream(dev)
    with torch.cuda.stream(st):
        d_jobs = torch.from_numpy(m.jobs.view(np.uint8)).to(dev)
        d_q = torch.from_numpy(m.qseq).to(dev)
        d_t = torch.from_numpy(m.tseq).to(dev)
        d_out = torch.empty(n * 7, dtype=torch.int32, device=dev)
        for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            N.check(lib.fa_mate_sw_batch_device(ctx.handle, N.ptr(mp), d_jobs.data_ptr(), n, d_q.data_ptr(),
                                                d_t.data_ptr(), d_out.data_ptr(), ctypes.c_void_p(st.cuda_stream)))
            e1.record(st)
            st.synchronize()
            N.check(lib.fa_ctx_sync(ctx.handle))
            print("mate batch ms", e0.elapsed_time(e1))
    sys.exit(0)

if len(sys.argv) > 1 and sys.argv[1] == "rescue":
    from ferrousalign_b200 import mate_rescue as R
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 200_000
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(n)
    pac, l_pac = fa.pack_reference(ref)
    bounds = np.zeros(4, N.INSERT_BOUNDS_DT)
    bounds[:] = [(0, 0, 1, 0), (200, 600, 0, 0), (0, 0, 1, 0), (0, 0, 1, 0)]
    ctx = fa.Context(0)
    lib = N.load()
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
        got = R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, cands, bounds, ctx=ctx)
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        print("rescue collection kernel ms", k_ms.value, "jobs", len(got.jobs))
    sys.exit(0)

if len(sys.argv) > 1 and sys.argv[1] == "cigar":
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 200_000
    jobs, qseq, tseq = synth.workload_cigar(n)
    ctx = fa.Context(0)
    lib = N.load()
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    p = fa.BandedPairWiseSW().to_struct()
    for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
        got = fa.scalar_banded_swa_batch(p, jobs, qseq, tseq, ctx=ctx)
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        print("cigar kernel ms", k_ms.value, "cells", int(got.results["cells"].sum()))
    sys.exit(0)

if len(sys.argv) > 1 and sys.argv[1] == "collect":
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 500_000
    ref, reads, off, chains, seeds = synth.workload_chains(n, ref_len=100_000_000)
    pac, l_pac = fa.pack_reference(ref)
    ctx = fa.Context(0)
    lib = N.load()
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
        got = fa.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds, ctx=ctx)
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        print("collect kernel ms", k_ms.value, "jobs", len(got.left_jobs), len(got.right_jobs))
    sys.exit(0)

if len(sys.argv) > 1 and sys.argv[1] == "regions":
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 2_000_000
    first, qlen, seeds, left, right = synth.workload_regions(n)
    ctx = fa.Context(0)
    lib = N.load()
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream(dev)
    opt = fa.region_opts()
    t = lambda a: torch.from_numpy(a.view(np.uint8)).to(dev)  # noqa: E731
    d = [t(first), t(qlen), t(seeds), t(left), t(right)]
    d_out = torch.empty(n * N.REGION_DT.itemsize, dtype=torch.uint8, device=dev)
    for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        N.check(lib.fa_merge_regions_device(ctx.handle, N.ptr(opt), d[0].data_ptr(), n, d[1].data_ptr(),
                                            d[2].data_ptr(), len(seeds), d[3].data_ptr(), len(left), d[4].data_ptr(),
                                            len(right), d_out.data_ptr(), ctypes.c_void_p(st.cuda_stream)))
        e1.record(st)
        st.synchronize()
        N.check(lib.fa_ctx_sync(ctx.handle))
        print("region merge ms", e0.elapsed_time(e1))
    sys.exit(0)

if len(sys.argv) > 1 and sys.argv[1] in ("learned", "bands"):
    from ferrousalign_b200 import band_model as B
    mode = sys.argv[1]
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 1_000_000
    uneven = len(sys.argv) > 5 and sys.argv[5] == "uneven"   # the 50-300 bp batch, whole-batch launches
    b = synth.workload_ext_uneven(n) if uneven else synth.workload_ext_1m(n)
    p = fa.BandedPairWiseSW().to_struct()
    ctx = fa.Context(0)
    if len(sys.argv) > 4:               # fixed kernel choice (autotuning timings mean nothing under ncu)
        ctx.set_kernel(int(sys.argv[4]))
    if uneven:
        ctx.set_slices(1, 1)
    if mode == "learned":
        m = B.BandModel.load(B.UNEVEN_MODEL if uneven else B.DEFAULT_MODEL)
        hints = B.hints_from_info(b.info)
        for r in range(int(sys.argv[3]) if len(sys.argv) > 3 else 1):
            out, st, wf, wfin = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, ctx=ctx)
            print("learned kernel ms", float(st["kernel_ms"]), "cells", int(st["cells_executed"]),
                  "launches", int(st["kernel_launches"]), "retries", int(st["retries"]))
        vals, cnts = np.unique(wf, return_counts=True)
        print("first bands", {int(v): int(c) for v, c in zip(vals, cnts)})
    else:
        for w in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 64, 100):
            j = b.jobs.copy()
            j["w"] = np.minimum(j["w"], w)
            for r in range(2):
                out, st, _ = fa.extend_batch(p, j, b.qseq, b.tseq, ctx=ctx)
            print(f"band {w}: kernel ms {float(st['kernel_ms']):.3f} cells {int(st['cells_executed'])} "
                  f"Gcell/s {int(st['cells_executed']) / float(st['kernel_ms']) / 1e6:.1f}")
    sys.exit(0)

n = int(sys.argv[1]) if len(sys.argv) > 1 else 1_000_000
b = synth.workload_ext_uneven(n) if len(sys.argv) > 2 and sys.argv[2] == "uneven" else synth.workload_ext_1m(n)
p = fa.BandedPairWiseSW().to_struct()
ctx = fa.Context(0)
lib = N.load()
if len(sys.argv) > 3:
    ctx.set_kernel(int(sys.argv[3]))
if len(sys.argv) > 5:
    ctx.set_threads(int(sys.argv[5]))
reps = int(sys.argv[4]) if len(sys.argv) > 4 else 1
dev = torch.device("cuda", 0)
st = torch.cuda.Stream(dev)
with torch.cuda.stream(st):
    d_jobs = torch.from_numpy(b.jobs.view(np.uint8)).to(dev)
    d_q = torch.from_numpy(b.qseq).to(dev)
    d_t = torch.from_numpy(b.tseq).to(dev)
    d_out = torch.empty(n * 6, dtype=torch.int32, device=dev)
    for r in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        N.check(lib.fa_ext_batch_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(),
                                        d_t.data_ptr(), None, d_out.data_ptr(), ctypes.c_void_p(st.cuda_stream)))
        e1.record(st)
        st.synchronize()
        N.check(lib.fa_ctx_sync(ctx.handle))
        print("batch ms", e0.elapsed_time(e1))
if len(sys.argv) > 2 and sys.argv[2] == "probe":
    v, ms = ctypes.c_double(), ctypes.c_float()
    for k, name in enumerate(["viaddmax_s16x2_relu", "vimax3_s16x2_relu", "viaddmax_s32_relu", "vimax3_s32",
                              "add+max (2 instr)"]):
        N.check(lib.fa_probe_int_peak(ctx.handle, k, ctypes.byref(v), ctypes.byref(ms)))
        print(f"probe {name}: {v.value / 1e12:.2f} Tops/s")
