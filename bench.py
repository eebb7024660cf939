#!/usr/bin/env python3
"""Throughput of the batched banded seed extension on B200.

Workload (one step): 1,000,000 right extensions of 151-bp reads (per-read indel rate
from {0, 0.1%, 1%, 3%}, 1% substitutions, seed 19-51 bp at the read start, h0 = seed
length, target = suffix length + 100), scoring A=1 B=4 N=-1 O=6 E=1, w=100, zdrop=100,
end bonus 5 -- seeded synthetic data with the shapes of the reference's workload.
Results are bit-exact to the oracle (checked on a sample every run).

value   : alignments/s with inputs resident in HBM (device-resident C ABI call,
          longest-first device ordering inside the timed region).
e2e     : alignments/s through the host C ABI call fa_ext_batch from pinned host buffers,
          host->device copies of jobs and sequences and the device->host copy of the
          results inside the timed region.
GCUPS   : cells = sum over rows of the adaptive band width (end - beg), the oracle's count.

--impl reference times the reference's own CPU path for this step -- its SIMD batch kernels
(sw_kernel_i16, AVX-512BW or AVX2), restated in C++ because the Rust crate cannot be built
here -- on all host cores over the whole batch.  The line's cpu_baselines also time that path
in every width the CPU runs and the exact-semantics scalar port of ksw_extend2.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GCUPS & alignments/s @151bp, learned-band vs plain-band on B200, bit-exact"
N_JOBS = 1_000_000
CPU_SAMPLE = 200_000
MATE_JOBS = 500_000
# DRAM bytes per job of the extension kernels (ncu dram__bytes_read.sum + write.sum of one
# launch on the 151-bp workload; the algorithmic bytes are about 372 B per job):
# ext_packed_kernel (int32, 439,186 jobs): 248.1 MB + 11.2 MB;
# ext_rows2_kernel (two rows per thread, 175,709 jobs): 72.3 MB + 2.5 MB
EXT_KERNELS = {"int32": ("ext_packed_kernel", (248.106e6 + 11.161e6) / 439_186, "int32"),
               "rows2": ("ext_rows2_persist_kernel", (72.319e6 + 2.543e6) / 175_709, "int16x2"),
               "int16x2": ("ext_pair_kernel", None, "int16x2")}
UNEVEN_JOBS = 2_000_000
MATE_CPU_SAMPLE = 20_000
DPX_OPS_PER_CELL_PAIR = 9   # int16x2 ops per packed cell pair in the roofline model
# mate SW (u8 engine, unsaturated form): PRMT profile byte, max(hd + s, E, 0), max(., F), the
# shared gap term, E and F updates -- DPX 16x2 instructions per two cells of a segment
MATE_DPX_OPS_PER_CELL_PAIR = 6
# mate SW bytes per job: the algorithmic reads and writes (job record 32 B, query 151 B,
# window 551 B, result 28 B) and the DRAM traffic of one ncu capture of both kernels on
# 200,000 jobs of the same workload, per job
MATE_ALGO_PER_JOB = 32 + 151 + 551 + 28
MATE_DRAM_PER_JOB = (6.405e6 + 148.886e6 + 3.509e6 + 100.364e6 + 7.430e6) / 200_000


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def hbm_peak() -> tuple[float, str]:
    """HBM copy bandwidth (GB/s) for the HBM rooflines: the measured figure of this GPU pool
    (MEASURED_PEAKS.json hbm_gbs) when the file is there, else the pool's earlier measured
    6,650 GB/s."""
    try:
        v = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
        return v, f"of measured (MEASURED_PEAKS.json hbm_gbs = {v})"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "of fallback (6.65 TB/s, earlier measurement on this GPU pool)"


HBM_GBS, HBM_SOURCE = hbm_peak()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    from ferrousalign_b200.replicas import dist_env as env
    return env()


def make_workload(rank: int, n: int):
    from ferrousalign_b200 import synth
    from ferrousalign_b200.replicas import shard_seed
    t0 = time.time()
    b = synth.workload_ext_1m(n, seed=shard_seed(2, rank))
    log(f"[rank {rank}] generated {n} jobs in {time.time() - t0:.1f}s "
        f"(query {b.qseq.nbytes / 1e6:.0f} MB, target {b.tseq.nbytes / 1e6:.0f} MB)")
    return b


def cpu_oracle_rate(b, p, sample: int):
    """Oracle (restated ksw_extend2) on all host threads over the first `sample` jobs."""
    from oracle import ksw_oracle as O
    jobs = b.jobs[:sample]
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    out, tr = O.ext_batch(p, jobs, b.qseq, b.tseq, threads=threads)
    dt = time.perf_counter() - t0
    return out, tr, dt, threads


SIMD_PATH = {"avx512": "sw_kernel_i16 (banded_swa/kernel_i16.rs:44-272) with AVX-512BW, 32 int16 lanes",
             "avx2": "sw_kernel_i16 (banded_swa/kernel_i16.rs:44-272) with AVX2, 16 int16 lanes"}
KSWV_PATH = {"avx512": "batch_ksw_align (kswv_avx2.rs:93-641) with AVX-512BW, 64 u8 lanes",
             "avx2": "batch_ksw_align_avx2 (kswv_avx2.rs:93-641), 32 u8 lanes"}


def cpu_simd_rate(b, p, isa: str, reps: int = 1):
    """The reference's SIMD CPU path restated (oracle/simd_baseline.cpp): every job of the
    batch in chunks of the vector width, SoA transposes included, on all host threads.
    Returns (seconds per pass, threads)."""
    from oracle import simd_baseline as S
    threads = os.cpu_count() or 1
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        S.ext_batch(p, b.jobs, b.qseq, b.tseq, isa=isa, threads=threads)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best, threads


def cpu_baselines(b, p, cells: int | None):
    """CPU baselines on the host cores: the reference's SIMD path (every width the CPU runs)
    over the whole batch, and the exact-semantics scalar port over a 200k-job sample.
    `cells`: the batch's algorithmic cells (the GCUPS numerator of every line)."""
    from oracle import simd_baseline as S
    n = len(b.jobs)
    res = {}
    for isa in S.ISAS:
        if not S.cpu_has(isa):
            res[f"simd_{isa}"] = {"unavailable": f"host CPU lacks {isa}"}
            continue
        dt, threads = cpu_simd_rate(b, p, isa, reps=2)
        res[f"simd_{isa}"] = {"value": n / dt, "unit": "alignments/s", "cores": threads, "kind": "port",
                              "restates": SIMD_PATH[isa], "gcups": (cells / dt / 1e9) if cells else None,
                              "sample": f"all {n} jobs of the batch (chunks of the vector width), all host threads"}
    sample = min(CPU_SAMPLE, n)
    _, tr, dt, threads = cpu_oracle_rate(b, p, sample)
    res["scalar_ksw_extend2"] = {"value": sample / dt, "unit": "alignments/s", "cores": threads, "kind": "port",
                                 "restates": "ksw_extend2 (ksw_affine_gap.rs:952-1169), exact outputs",
                                 "gcups": float(tr["cells"].sum()) / dt / 1e9,
                                 "sample": f"first {sample} jobs of the batch, all host threads"}
    isa = S.best_isa()
    head = dict(res[f"simd_{isa}"])
    return head, res


def bench_learned(args, ctx, b, p):
    """Learned band vs plain band on the same 1M batch: the plain bwa-mem2 retry policy at
    w=100 against the learned path (GPU features + MLP first band, exit-bound certificate
    as the judge, one narrow try then the configured band), and the same policy without
    the network (every job starting at one fixed band); all through the host ABI with the
    whole batch uploaded before its kernels (slice count 1, so each kernel runs over the full
    batch), rates from the device time of their kernels, outputs compared with the plain
    path's.  The overlapped end-to-end forms are in the e2e_packed section."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from ferrousalign_b200 import band_model as B
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    model = B.BandModel.load()
    hints = B.hints_from_info(b.info)
    n = len(b.jobs)
    fixed_w = 24
    nonet_pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_LEARNED, 1)
    wf_fixed = np.full(n, fixed_w, np.int32)
    plain_ms, learned_ms, nonet_ms = [], [], []
    plain = learned = nonet = None
    ctx.set_slices(1, 1)
    for _ in range(max(3, args.steps // 10)):
        plain, pst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=bwa, ctx=ctx)
        plain_ms.append(float(pst["kernel_ms"]))
        learned, lst, wf, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, model, hints=hints, ctx=ctx)
        learned_ms.append(float(lst["kernel_ms"]))
        nonet, nst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=nonet_pol, w_first=wf_fixed, ctx=ctx)
        nonet_ms.append(float(nst["kernel_ms"]))
    ctx.set_slices(-1, -1)
    pm, lm, fm = float(np.median(plain_ms)), float(np.median(learned_ms)), float(np.median(nonet_ms))
    return {"plain": {"policy": "bwa-mem2 w=100 then 200", "value": n / (pm * 1e-3), "unit": "alignments/s",
                      "gcups": float(pst["cells_executed"]) / (pm * 1e-3) / 1e9,
                      "kernel_ms": pm, "cells_executed": int(pst["cells_executed"])},
            "learned": {"policy": "MLP first band (ladder 2,3,4,6,8,12,..; >= 2), exit-bound certificate judge "
                                  "(exact), one narrow try then w=100 plain policy",
                        "value": n / (lm * 1e-3), "unit": "alignments/s", "kernel_ms": lm,
                        "kernel_launches": int(lst["kernel_launches"]),
                        "cells_executed": int(lst["cells_executed"]),
                        "cells_saved_frac": 1.0 - float(lst["cells_executed"]) / float(pst["cells_executed"]),
                        "miss_rate": float(lst["misses"]) / n,
                        "wasted_cells": int(lst["cells_executed"]) - int(lst["cells"]),
                        "wasted_frac_of_executed": (float(lst["cells_executed"]) - float(lst["cells"]))
                        / float(lst["cells_executed"]),
                        "first_band_median": float(np.median(wf))},
            "no_network": {"policy": f"same policy, every job first at w={fixed_w} (best fixed first band on the "
                                     "held-out evaluation batch)",
                           "value": n / (fm * 1e-3), "unit": "alignments/s", "kernel_ms": fm,
                           "cells_executed": int(nst["cells_executed"]),
                           "identical_outputs": bool(np.array_equal(plain, nonet))},
            "speedup": pm / lm, "network_gain": fm / lm,
            "identical_outputs": bool(np.array_equal(plain, learned)),
            "identical_frac": float(np.mean(plain == learned))}


def pin_array(a):
    """A page-locked copy of a numpy array (same dtype and shape)."""
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.uint8).reshape(-1)).pin_memory().numpy().view(a.dtype).reshape(a.shape)


def bench_e2e_forms(args, ctx, b, p):
    """End to end through the host ABI, on the 1M-job batch: the call a user makes, from
    page-locked host buffers (jobs, sequences, hints) into a page-locked result buffer, with
    every copy inside the timed call, in wall-clock milliseconds (median over the steps).
    Forms: byte-code buffers (the drop-in for execute_batch_simd_scoring) and 2-bit packed
    buffers; the single-band call, the bwa-mem2 retry policy and the learned band.  Host-side
    packing is not timed (a packed caller holds packed sequences, as the reference's index
    holds its .pac)."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from ferrousalign_b200 import band_model as B
    n = len(b.jobs)
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    model = B.BandModel.load()
    hints = pin_array(B.hints_from_info(b.info))
    pj, pq, pt = pin_array(b.jobs), pin_array(b.qseq), pin_array(b.tseq)
    qp, tp = fa.pack(b.qseq).pinned(), fa.pack(b.tseq).pinned()
    out_h = pin_array(np.zeros(n, N.EXT_RESULT_DT))
    byte_in = int(pj.nbytes + pq.nbytes + pt.nbytes)
    pack_in = int(pj.nbytes + qp.nbytes + tp.nbytes)
    hint_in = int(hints.nbytes)
    o = {"ctx": ctx, "out": out_h, "bands": False}
    forms = {
        "bytes_single": (lambda: fa.extend_batch(p, pj, pq, pt, **o), byte_in),
        "packed_single": (lambda: fa.extend_batch_packed(p, pj, qp, tp, **o), pack_in),
        "bytes_bwa": (lambda: fa.extend_batch(p, pj, pq, pt, policy=bwa, **o), byte_in),
        "packed_bwa": (lambda: fa.extend_batch_packed(p, pj, qp, tp, policy=bwa, **o), pack_in),
        "bytes_learned": (lambda: B.extend_batch_learned(p, pj, pq, pt, model, hints=hints, **o), byte_in + hint_in),
        "packed_learned": (lambda: fa.extend_batch_learned_packed(p, pj, qp, tp, model, hints=hints, **o),
                           pack_in + hint_in),
    }
    res, outs = {}, {}
    for name, (fn, h2d) in forms.items():
        for _ in range(max(2, args.warmup)):
            fn()
        t = []
        for _ in range(max(5, args.steps // 2)):
            t0 = time.perf_counter()
            fn()
            t.append((time.perf_counter() - t0) * 1e3)
        outs[name] = out_h.copy()
        ms = float(np.median(t))
        res[name] = {"value": n / (ms * 1e-3), "unit": "alignments/s", "ms_per_step": ms,
                     "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * 24}
    res["identical_outputs"] = bool(all(np.array_equal(outs[k], outs["bytes_bwa"])
                                        for k in ("packed_bwa", "bytes_learned", "packed_learned")) and
                                    np.array_equal(outs["packed_single"], outs["bytes_single"]))
    res["learned_vs_bwa_packed"] = res["packed_bwa"]["ms_per_step"] / res["packed_learned"]["ms_per_step"]
    res["learned_vs_single_packed"] = res["packed_single"]["ms_per_step"] / res["packed_learned"]["ms_per_step"]
    res["learned_vs_bwa_bytes"] = res["bytes_bwa"]["ms_per_step"] / res["bytes_learned"]["ms_per_step"]
    return res


def bench_uneven(args, ctx, p):
    """Uneven-length batch: 2,000,000 mixed left and right extensions, reads 50-300 bp,
    seeds anywhere in the read, targets from a 100 Mbp reference with 5% low-complexity
    repeats.  Plain bwa-mem2 policy against the learned path (the model trained on this
    shape, band_model_uneven.bin, when present, else the 151-bp model; results stay exact
    whatever it predicts), both through the host ABI with whole-batch kernels (slice count
    1), device time of their kernels; outputs compared."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from ferrousalign_b200 import band_model as B
    from ferrousalign_b200 import synth
    t0 = time.time()
    u = synth.workload_ext_uneven(UNEVEN_JOBS)
    log(f"uneven workload: {UNEVEN_JOBS} jobs in {time.time() - t0:.1f}s")
    n = len(u.jobs)
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    model_path = B.UNEVEN_MODEL if B.UNEVEN_MODEL.exists() else B.DEFAULT_MODEL
    model = B.BandModel.load(model_path)
    hints = B.hints_from_info(u.info)
    pm, lm = [], []
    ctx.set_slices(1, 1)
    for _ in range(max(2, args.steps // 10)):
        plain, pst, _ = fa.extend_batch(p, u.jobs, u.qseq, u.tseq, policy=bwa, ctx=ctx)
        pm.append(float(pst["kernel_ms"]))
        learned, lst, wf, _ = B.extend_batch_learned(p, u.jobs, u.qseq, u.tseq, model, hints=hints, ctx=ctx)
        lm.append(float(lst["kernel_ms"]))
    # the kernel the learned call's plain-policy rounds ran (autotuned for the longest class)
    lc = ctx.kernel_choice()
    ctx.set_slices(-1, -1)
    pms, lms = float(np.median(pm)), float(np.median(lm))
    # the same two calls with the whole extend / check / retry loop recorded as one CUDA graph
    # per context (replayed after the first call of the shape)
    gp, gl = N.Context(0), N.Context(0)
    try:
        gp.set_graph(True)
        gl.set_graph(True)
        gpm, glm = [], []
        for r in range(1 + max(2, args.steps // 10)):
            gplain, gst, _ = fa.extend_batch(p, u.jobs, u.qseq, u.tseq, policy=bwa, ctx=gp)
            glearned, glst, _, _ = B.extend_batch_learned(p, u.jobs, u.qseq, u.tseq, model, hints=hints, ctx=gl)
            if r:
                gpm.append(float(gst["kernel_ms"]))
                glm.append(float(glst["kernel_ms"]))
    finally:
        gp.close()
        gl.close()
    gpms, glms = float(np.median(gpm)), float(np.median(glm))
    ql = u.jobs["qlen"]
    return {"workload": f"{n} mixed left/right extensions, reads 50-300 bp, 100 Mbp reference with 5% repeats",
            "qlen_mean": float(ql.mean()), "qlen_max": int(ql.max()), "model": model_path.name,
            "plain": {"value": n / (pms * 1e-3), "unit": "alignments/s", "kernel_ms": pms,
                      "gcups": float(pst["cells_executed"]) / (pms * 1e-3) / 1e9},
            "learned": {"value": n / (lms * 1e-3), "unit": "alignments/s", "kernel_ms": lms,
                        "cells_saved_frac": 1.0 - float(lst["cells_executed"]) / float(pst["cells_executed"]),
                        "miss_rate": float(lst["misses"]) / n,
                        "retry_kernel": {"kernel": lc["kernel"], "threads_per_block": lc["threads_per_block"]}},
            "speedup": pms / lms, "identical_outputs": bool(np.array_equal(plain, learned)),
            "graph": {"plain_kernel_ms": gpms, "learned_kernel_ms": glms,
                      "plain_value": n / (gpms * 1e-3), "learned_value": n / (glms * 1e-3),
                      "identical_outputs": bool(np.array_equal(gplain, plain) and np.array_equal(glearned, plain))}}


def bench_mixed(args, b, p):
    """Mixed batch: 500,000 mate-rescue pairs and the 1,000,000 seed extensions of one
    batch, submitted together through one host ABI call (fa_pair_batch: the mate SW runs on
    its own stream while the extension rounds run), inputs and results in pinned host
    memory, copies included.  Plain (bwa-mem2 policy) and learned-band forms; latency
    percentiles over the batches."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from ferrousalign_b200 import band_model as B
    from ferrousalign_b200 import synth
    m = synth.workload_mate(MATE_JOBS)
    mp = fa.make_mate_params()
    mj, mq, mt = pin_array(m.jobs), pin_array(m.qseq), pin_array(m.tseq)
    ej, eq, et = pin_array(b.jobs), pin_array(b.qseq), pin_array(b.tseq)
    hints = pin_array(B.hints_from_info(b.info))
    model = B.BandModel.load()
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)
    ctx = N.Context(0)
    res = {"workload": f"{MATE_JOBS} mate-rescue SW jobs (2x151 bp pairs, 551 bp windows) + {len(b.jobs)} "
                       "151-bp seed extensions per batch, one fa_pair_batch call, pinned buffers"}
    outs = {}
    try:
        for form in ("plain", "learned"):
            eo = pin_array(np.zeros(len(b.jobs), N.EXT_RESULT_DT))
            mo = pin_array(np.zeros(MATE_JOBS, N.KSWR_DT))
            lat, kern, mkern = [], [], []
            for it in range(args.warmup + max(5, args.steps // 3)):
                t0 = time.perf_counter()
                if form == "plain":
                    _, _, st, mst = fa.pair_batch(p, ej, eq, et, mp, mj, mq, mt, policy=bwa, ctx=ctx, out=eo,
                                                  mate_out=mo)
                else:
                    _, _, st, mst = fa.pair_batch(p, ej, eq, et, mp, mj, mq, mt, model=model, hints=hints,
                                                  ctx=ctx, out=eo, mate_out=mo)
                dt = (time.perf_counter() - t0) * 1e3
                if it >= args.warmup:
                    lat.append(dt)
                    kern.append(float(st["kernel_ms"]))
                    mkern.append(float(mst["kernel_ms"]))
            outs[form] = (eo.copy(), mo.copy())
            lat = np.array(lat)
            res[form] = {"batches": len(lat), "p50_ms": float(np.percentile(lat, 50)),
                         "p95_ms": float(np.percentile(lat, 95)), "p99_ms": float(np.percentile(lat, 99)),
                         "max_ms": float(lat.max()),
                         "ext_kernel_ms_p50": float(np.median(kern)), "mate_kernel_ms_p50": float(np.median(mkern)),
                         "alignments_per_s": (MATE_JOBS + len(b.jobs)) / (float(np.median(lat)) * 1e-3)}
        res["identical_outputs"] = bool(np.array_equal(outs["plain"][0], outs["learned"][0]) and
                                        np.array_equal(outs["plain"][1], outs["learned"][1]))
    finally:
        ctx.close()
    return res


def bench_mate(args, ctx, lib, dev, stream, flush, skip_cpu=False):
    """Mate-rescue local SW on 500,000 2x151 bp pairs (insert ~ N(400, 50), window 551 bp),
    device-resident, same step/warm-up counts as the extension line."""
    import ctypes
    import torch
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from ferrousalign_b200 import synth
    t0 = time.time()
    m = synth.workload_mate(MATE_JOBS)
    log(f"mate workload: {MATE_JOBS} jobs in {time.time() - t0:.1f}s")
    mp = fa.make_mate_params()
    with torch.cuda.stream(stream):
        d_jobs = torch.from_numpy(m.jobs.view(np.uint8)).to(dev)
        d_q = torch.from_numpy(m.qseq).to(dev)
        d_t = torch.from_numpy(m.tseq).to(dev)
        d_out = torch.empty(MATE_JOBS * 7, dtype=torch.int32, device=dev)
    stream.synchronize()
    k_ms, k_n, cells = ctypes.c_float(), ctypes.c_int(), ctypes.c_ulonglong()

    def step():
        N.check(lib.fa_mate_sw_batch_device(ctx.handle, N.ptr(mp), d_jobs.data_ptr(), MATE_JOBS, d_q.data_ptr(),
                                            d_t.data_ptr(), d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            step()
    N.check(lib.fa_ctx_sync(ctx.handle))
    times, ktimes, launches = [], [], 0
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.steps // 3)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
            ktimes.append(k_ms.value)
            launches += k_n.value
    N.check(lib.fa_ctx_sync(ctx.handle))
    N.check(lib.fa_ctx_last_cells(ctx.handle, ctypes.byref(cells)))
    ms = float(np.mean(times))
    kms = float(np.mean(ktimes))
    out = d_out.cpu().numpy().view(N.KSWR_DT).reshape(-1)
    from oracle import ksw_oracle as O
    chk = np.arange(0, MATE_JOBS, max(1, MATE_JOBS // 2000))
    ref, _ = O.mate_batch(mp, m.jobs[chk], m.qseq, m.tseq)
    # roofline: the u8 engine's unsaturated form issues MATE_DPX_OPS_PER_CELL_PAIR DPX 16x2
    # instructions per two cells of a segment update; the peak is the measured DPX issue rate
    v, pms = ctypes.c_double(), ctypes.c_float()
    N.check(lib.fa_probe_int_peak(ctx.handle, 0, ctypes.byref(v), ctypes.byref(pms)))
    peak_gcups = v.value * 2 / MATE_DPX_OPS_PER_CELL_PAIR / 1e9
    achieved = cells.value / (kms * 1e-3) / 1e9
    res = {"workload": "500k 2x151bp pairs, insert N(400,50), 551 bp window, ksw_align2 u8 + XSTART",
           "value": MATE_JOBS / (ms * 1e-3), "unit": "alignments/s", "ms_per_step": ms,
           "gcups": achieved, "kernel_ms_per_step": kms,
           "cells_per_step": int(cells.value), "bit_exact_sample": bool(np.array_equal(out[chk], ref)),
           "gpu_launches": launches,
           "roofline": {"bound": "dpx", "achieved": achieved, "peak": peak_gcups, "unit": "Gcell/s",
                        "frac": achieved / peak_gcups, "kernel": "mate_sw_kernel_u8x2 + mate_rev_kernel_u8x2",
                        "cells": "ksw_align2's cells (forward pass and every KSW_XSTART pass it runs, those "
                                 "skipped as unable to reach the score included)",
                        "traffic": None if MATE_DRAM_PER_JOB is None else MATE_DRAM_PER_JOB * MATE_JOBS,
                        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per job of both "
                                          "kernels, scaled",
                        "algorithmic_bytes": MATE_ALGO_PER_JOB * MATE_JOBS,
                        "peak_source": f"measured __viaddmax_s16x2_relu rate {v.value / 1e12:.2f} Tops/s x2/"
                                       f"{MATE_DPX_OPS_PER_CELL_PAIR}"}}
    # end to end through the host entries, pinned buffers, copies in the timed call: byte codes
    # and 2-bit packed bases
    mj, mq, mt = pin_array(m.jobs), pin_array(m.qseq), pin_array(m.tseq)
    qp, tp = fa.pack(m.qseq).pinned(), fa.pack(m.tseq).pinned()
    mo = pin_array(np.zeros(MATE_JOBS, N.KSWR_DT))
    forms = {"bytes": (lambda: fa.mate_sw_batch(mp, mj, mq, mt, ctx=ctx, out=mo),
                       int(mj.nbytes + mq.nbytes + mt.nbytes)),
             "packed": (lambda: fa.mate_sw_batch_packed(mp, mj, qp, tp, ctx=ctx, out=mo),
                        int(mj.nbytes + qp.nbytes + tp.nbytes))}
    e2e = {}
    for name, (fn, h2d) in forms.items():
        fn()
        wall = []
        for _ in range(3):
            t0 = time.perf_counter()
            o, _ = fn()
            wall.append((time.perf_counter() - t0) * 1e3)
        e2e[name] = {"value": MATE_JOBS / (float(np.median(wall)) * 1e-3), "unit": "alignments/s",
                     "ms_per_step": float(np.median(wall)), "h2d_bytes_per_step": h2d,
                     "d2h_bytes_per_step": MATE_JOBS * 28, "identical": bool(np.array_equal(o[chk], ref))}
    res["e2e"] = e2e
    if not skip_cpu:
        from oracle import simd_baseline as S
        base = {}
        for isa in S.ISAS:
            if not S.cpu_has(isa):
                continue
            t0 = time.perf_counter()
            S.kswv_batch(m.jobs, m.qseq, m.tseq, isa=isa, threads=os.cpu_count() or 1)
            dt = time.perf_counter() - t0
            base[f"kswv_{isa}"] = {"value": MATE_JOBS / dt, "unit": "alignments/s", "cores": os.cpu_count(),
                                   "kind": "port", "restates": KSWV_PATH[isa],
                                   "gcups": cells.value / dt / 1e9,
                                   "sample": f"all {MATE_JOBS} jobs, all host threads (score/te exact; tb/qb "
                                             "estimated and score2 on every other lane, as the reference's kernel)"}
        sample = m.jobs[:MATE_CPU_SAMPLE]
        t0 = time.perf_counter()
        _, cc = O.mate_batch(mp, sample, m.qseq, m.tseq, threads=os.cpu_count() or 1)
        dt = time.perf_counter() - t0
        base["scalar_ksw_align2"] = {"value": MATE_CPU_SAMPLE / dt, "unit": "alignments/s",
                                     "cores": os.cpu_count(), "kind": "port",
                                     "restates": "ksw_align2 (ksw_affine_gap.rs:773-861), exact outputs",
                                     "gcups": float(cc.sum()) / dt / 1e9,
                                     "sample": f"first {MATE_CPU_SAMPLE} jobs, all host threads"}
        res["cpu_baseline"] = dict(base.get(f"kswv_{S.best_isa()}", base["scalar_ksw_align2"]))
        res["cpu_baselines"] = base
    return res


def bench_regions(args, ctx, lib, dev, stream, flush):
    """Region merge (merge_scores_to_regions) over the results of an extension batch:
    2M chains of 1-8 seeds (9M seeds, one left and one right result each), device
    resident, timed with CUDA events; HBM-bound, so reported against the measured copy
    bandwidth.  Algorithmic bytes per chain: its bounds and read length (8 B), its seed
    records (24 B each), the left and right results they index (2 x 24 B each) and the
    region written (48 B)."""
    import ctypes
    import torch
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    from oracle import region_oracle as R
    from ferrousalign_b200 import synth
    first, qlen, seeds, left, right = synth.workload_regions(2_000_000)
    n_chains, ns = len(qlen), len(seeds)
    res = [left, right]
    opt = fa.region_opts()
    t = lambda a: torch.from_numpy(a.view(np.uint8)).to(dev)  # noqa: E731
    d_first, d_qlen, d_seeds, d_left, d_right = t(first), t(qlen), t(seeds), t(res[0]), t(res[1])
    d_out = torch.empty(n_chains * N.REGION_DT.itemsize, dtype=torch.uint8, device=dev)

    def step():
        N.check(lib.fa_merge_regions_device(ctx.handle, N.ptr(opt), d_first.data_ptr(), n_chains, d_qlen.data_ptr(),
                                            d_seeds.data_ptr(), ns, d_left.data_ptr(), ns, d_right.data_ptr(), ns,
                                            d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))

    times = []
    with torch.cuda.stream(stream):
        for it in range(args.warmup + 10):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            if it >= args.warmup:
                times.append(e0.elapsed_time(e1))
    N.check(lib.fa_ctx_sync(ctx.handle))
    ms = float(np.median(times))
    out = d_out.cpu().numpy().view(N.REGION_DT)
    k = 3000
    o = {f: int(opt[f][0]) for f in ("a", "pen_clip5", "pen_clip3", "w")}
    ref = R.merge_regions(o, first[:k + 1], qlen[:k], seeds, res[0], res[1])
    algo = n_chains * (8 + 48) + ns * (24 + 2 * 24)
    return {"workload": f"{n_chains} chains, {ns} seeds (1-8 per chain), one left and one right result per seed",
            "kernel": "merge_regions_kernel", "kernel_ms": ms, "chains_per_s": n_chains / (ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": algo / (ms * 1e-3) / 1e9, "peak": HBM_GBS, "unit": "GB/s",
                         "frac": algo / (ms * 1e-3) / 1e9 / HBM_GBS, "algorithmic_bytes": algo,
                         "peak_source": HBM_SOURCE},
            "bit_exact_sample": bool(np.array_equal(out[:k], ref)), "sample": f"first {k} chains against the oracle"}


def bench_collect(args, ctx, lib):
    """Extension-job collection (collect_extension_jobs_batch_soa) from chains of seeds over
    a 100 Mbp reference held 2-bit packed on the GPU: 500k 151-bp reads from both strands,
    1-3 chains of 1-4 seeds each.  Timed through the host ABI (`e2e`: the packed reference
    resident on the device as a loaded index is, page-locked reads, chains and seeds, every
    copy in and out inside the call, outputs into reusable page-locked buffers, as a caller
    collecting batch after batch holds them) and on the device (the kernels, with the one
    read of the totals between plan and fill).
    Algorithmic bytes: reads, chains, seeds and the windows' packed bases in; both copies
    of every read and window, the jobs, the seed table and the chain windows out."""
    import ctypes
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, synth
    from oracle import collect_oracle as C
    ref, reads, off, chains, seeds = synth.workload_chains(500_000, ref_len=100_000_000)
    pac, l_pac = fa.pack_reference(ref)
    p_reads, p_off = pin_array(reads), pin_array(off)
    p_chains, p_seeds = pin_array(chains), pin_array(seeds)
    bufs, pbufs = fa.CollectBuffers(pinned=True), fa.CollectBuffers(pinned=True)
    ctx.set_reference(pac, l_pac)   # the index is loaded once; batches bring reads, chains and seeds
    p_pac = None
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    wall, kern = [], []
    got = None
    for it in range(args.warmup + 5):
        t0 = time.perf_counter()
        got = fa.collect_extension_jobs(p_pac, l_pac, p_reads, p_off, p_chains, p_seeds, ctx=ctx, bufs=bufs)
        t1 = time.perf_counter()
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        if it >= args.warmup:
            wall.append((t1 - t0) * 1e3)
            kern.append(k_ms.value)
    win = got.chain_win.astype(np.int64)
    wlen = int(np.maximum(win[:, 1] - win[:, 0], 0).sum())
    n_jobs = len(got.left_jobs) + len(got.right_jobs)
    algo = (len(reads) + 16 * (len(chains) + len(seeds)) + wlen // 4 + 2 * len(reads) + 2 * wlen + 40 * n_jobs
            + 24 * len(got.seed_ext) + 20 * len(chains))
    km = float(np.median(kern))
    # the packed form: same jobs, qbuf / tbuf packed on the device (a quarter of their bytes back)
    pwall, pkern = [], []
    pk = None
    for it in range(args.warmup + 5):
        t0 = time.perf_counter()
        pk = fa.collect_extension_jobs_packed(p_pac, l_pac, p_reads, p_off, p_chains, p_seeds, ctx=ctx, bufs=pbufs)
        t1 = time.perf_counter()
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        if it >= args.warmup:
            pwall.append((t1 - t0) * 1e3)
            pkern.append(k_ms.value)
    packed_same = bool(np.array_equal(pk.left_jobs, got.left_jobs) and np.array_equal(pk.right_jobs, got.right_jobs)
                       and np.array_equal(fa.unpack(pk.tbuf)[:1 << 20], got.tbuf[:1 << 20]))
    # the first chains' jobs and seed table against the oracle (job numbers start at 0 there too)
    k = 1500
    o = {f: int(v) for f, v in zip(("a", "o_del", "e_del", "o_ins", "e_ins", "w"), (1, 6, 1, 6, 1, 100))}
    rl = [list(reads[int(off[r]):int(off[r + 1])]) for r in range(int(chains["read"][k - 1]) + 1)]
    ch = [{f: int(c[f]) for f in ("read", "seed_first", "n_seeds", "kept")} for c in chains[:k]]
    ns = int(chains["seed_first"][k - 1] + chains["n_seeds"][k - 1])
    sd = [{"ref_pos": int(s["ref_pos"]), "query_pos": int(s["query_pos"]), "len": int(s["len"])} for s in seeds[:ns]]
    want = C.collect(o, pac, l_pac, rl, ch, sd)
    same = all(list(got.qbuf[int(j["q_off"]):int(j["q_off"]) + int(j["qlen"])]) == q and
               list(got.tbuf[int(j["t_off"]):int(j["t_off"]) + int(j["tlen"])]) == t and int(j["h0"]) == h0
               for jobs, side in ((got.left_jobs, "left"), (got.right_jobs, "right"))
               for j, (q, t, h0, _, _) in zip(jobs, want[side]))
    same = same and [int(x) for x in got.chain_first[:k + 1]] == want["chain_first"]
    return {"workload": f"{len(off) - 1} reads of 151 bp, {len(chains)} chains, {len(seeds)} seeds, "
                        f"100 Mbp reference (2-bit packed, {len(pac)} B)",
            "jobs": {"left": len(got.left_jobs), "right": len(got.right_jobs)},
            "kernel_ms": km, "e2e_ms": float(np.median(wall)), "kernel_launches": int(k_n.value),
            "roofline": {"bound": "hbm", "achieved": algo / (km * 1e-3) / 1e9, "peak": HBM_GBS, "unit": "GB/s",
                         "frac": algo / (km * 1e-3) / 1e9 / HBM_GBS, "algorithmic_bytes": algo,
                         "peak_source": HBM_SOURCE},
            "bit_exact_sample": bool(same), "sample": f"first {k} chains against the oracle",
            "packed": {"e2e_ms": float(np.median(pwall)), "kernel_ms": float(np.median(pkern)),
                       "d2h_sequence_bytes": int(pk.qbuf.nbytes + pk.tbuf.nbytes),
                       "byte_form_sequence_bytes": int(len(got.qbuf) + len(got.tbuf)),
                       "same_jobs_and_bases": packed_same}}


def bench_cigar(args, ctx, lib):
    """CIGAR regeneration (scalar_banded_swa, h0 = 0) for 200k regions of 151-bp reads (the
    read against its reference span, bands of the length difference plus 5-30): kernel time
    with CUDA events, cells from the kernel's own count.  One thread per alignment runs the
    scalar int32 recurrence with a two-bit traceback written to HBM and read back along the
    path; reported against the copy bandwidth for its bytes (sequences in, traceback out
    and back, results out) and as cells per second.  `e2e_ms`: the host ABI call from
    page-locked inputs into reusable page-locked outputs, copies inside."""
    import ctypes
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, synth
    from oracle import cigar_oracle as C
    jobs, qseq, tseq = synth.workload_cigar(200_000)
    p = fa.BandedPairWiseSW().to_struct()
    p_jobs, p_q, p_t = pin_array(jobs), pin_array(qseq), pin_array(tseq)
    bufs = fa.HostBuffers(pinned=True)   # outputs reused call after call, as a batch loop holds them
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    kern, wall = [], []
    got = None
    for it in range(args.warmup + 5):
        t0 = time.perf_counter()
        got = fa.scalar_banded_swa_batch(p, p_jobs, p_q, p_t, ctx=ctx, bufs=bufs)
        t1 = time.perf_counter()
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        if it >= args.warmup:
            kern.append(k_ms.value)
            wall.append((t1 - t0) * 1e3)
    km = float(np.median(kern))
    n = len(jobs)
    cells = int(got.results["cells"].sum())
    seq_bytes = int(jobs["qlen"].sum() + jobs["tlen"].sum())
    out_bytes = n * 40 + 4 * int(got.results["n_cigar"].sum()) + int(got.results["n_ref"].sum() +
                                                                         got.results["n_query"].sum())
    algo = seq_bytes + cells // 4 + out_bytes + n * 32
    op = {"mat": [int(x) for x in p["mat"][0]], "o_del": 6, "e_del": 1, "o_ins": 6, "e_ins": 1, "zdrop": 100,
          "pen_clip3": 5}
    k = 300
    same = True
    for i in range(k):
        j = jobs[i]
        q = list(qseq[int(j["q_off"]):int(j["q_off"]) + int(j["qlen"])])
        t = list(tseq[int(j["t_off"]):int(j["t_off"]) + int(j["tlen"])])
        out, cig, ra, qa = C.banded_swa(op, q, t, int(j["w"]), int(j["h0"]))
        same = same and {f: int(got.results[i][f]) for f in out} == out and got.cigar_of(i) == cig
    return {"workload": f"{n} regions of 151-bp reads (read vs its reference span, h0 = 0, bands |dlen| + 5-30)",
            "kernel": "cigar_kernel", "kernel_ms": km, "alignments_per_s": n / (km * 1e-3),
            "gcups": cells / (km * 1e-3) / 1e9, "cells": cells, "e2e_ms": float(np.median(wall)),
            "roofline": {"bound": "alu", "hbm_achieved_gbs": algo / (km * 1e-3) / 1e9, "hbm_peak_gbs": HBM_GBS,
                         "hbm_frac": algo / (km * 1e-3) / 1e9 / HBM_GBS, "algorithmic_bytes": algo,
                         "note": "scalar int32 cells with a 2-bit traceback; one thread per alignment"},
            "bit_exact_sample": bool(same), "sample": f"first {k} alignments against the oracle"}


def bench_rescue_collect(args, ctx, lib):
    """Mate-rescue job collection (collect_rescue_jobs_for_read_soa) for 200k attempts of
    2x151-bp pairs (fragments N(400, 50), FR bounds [200, 600], the other orientations failed)
    over a 20 Mbp reference of six sequences held 2-bit packed on the GPU; device time of the
    plan, scan and fill kernels.  Algorithmic bytes: attempts, the rescued reads' alignments
    and bases in, the windows' packed bases in, jobs, origins, reads and windows out."""
    import ctypes
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, mate_rescue as R, synth
    from oracle import mate_collect_oracle as M
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(200_000)
    pac, l_pac = fa.pack_reference(ref)
    bounds = np.zeros(4, N.INSERT_BOUNDS_DT)
    bounds[:] = [(0, 0, 1, 0), (200, 600, 0, 0), (0, 0, 1, 0), (0, 0, 1, 0)]
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()
    kern, wall = [], []
    got = None
    p_reads, p_off, p_alns, p_cands = pin_array(reads), pin_array(off), pin_array(alns), pin_array(cands)
    bufs = fa.HostBuffers(pinned=True)   # outputs reused call after call, as a batch loop holds them
    ctx.set_reference(pac, l_pac)        # the index is loaded once
    p_pac = None
    for it in range(args.warmup + 5):
        t0 = time.perf_counter()
        got = R.collect_rescue_jobs(p_pac, l_pac, chr_off, chr_len, p_reads, p_off, p_alns, p_cands, bounds, ctx=ctx,
                                    bufs=bufs)
        t1 = time.perf_counter()
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        if it >= args.warmup:
            kern.append(k_ms.value)
            wall.append((t1 - t0) * 1e3)
    km = float(np.median(kern))
    # insert-size statistics of the attempts' pairs (anchor, the read's first alignment)
    l2 = np.int64(l_pac) * 2
    def fm(a):   # noqa: E306
        g = chr_off[a["ref_id"]].astype(np.int64) + a["pos"]
        return np.where(a["is_rev"] != 0, l2 - 1 - (g + a["ref_len"] - 1), g)
    pairs = np.stack([fm(cands["anchor"]), fm(alns[cands["aln_first"]])], 1).astype(np.int64)
    st_ms = []
    for it in range(args.warmup + 5):
        stats = R.calculate_insert_size_stats(l_pac, pairs, ctx=ctx)
        N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
        if it >= args.warmup:
            st_ms.append(k_ms.value)
    wl = int(got.info["adj_re"].sum() - got.info["adj_rb"].sum())
    algo = (cands.nbytes + alns.nbytes + len(reads) + wl // 4 + got.jobs.nbytes + got.info.nbytes +
            len(got.qbuf) + len(got.tbuf))
    k = 2000
    o = {"pen_unpaired": 17, "max_matesw": 50, "min_seed_len": 19, "match_score": 1}
    rd = lambda x, dt: {f: (rd(x[f], dt[f]) if dt[f].names else int(x[f])) for f in dt.names}  # noqa: E731
    rl = [list(reads[int(off[r]):int(off[r + 1])]) for r in range(k)]
    want = M.collect(o, [rd(b, bounds.dtype) for b in bounds], pac, l_pac, [int(x) for x in chr_off],
                     [int(x) for x in chr_len], rl, [rd(a, alns.dtype) for a in alns],
                     [rd(c, cands.dtype) for c in cands[:k]])
    same = len(want) <= len(got.jobs) and all(
        int(got.info["cand"][i]) == w["cand"] and int(got.info["orientation"][i]) == w["orientation"] and
        list(got.tbuf[int(got.jobs["t_off"][i]):int(got.jobs["t_off"][i]) + int(got.jobs["tlen"][i])]) == w["target"]
        for i, w in enumerate(want))
    return {"workload": f"{len(cands)} rescue attempts of 2x151-bp pairs, 20 Mbp reference (6 sequences, 2-bit packed)",
            "jobs": len(got.jobs), "kernel_ms": km, "e2e_ms": float(np.median(wall)),
            "kernel_launches": int(k_n.value),
            "roofline": {"bound": "hbm", "achieved": algo / (km * 1e-3) / 1e9, "peak": HBM_GBS, "unit": "GB/s",
                         "frac": algo / (km * 1e-3) / 1e9 / HBM_GBS, "algorithmic_bytes": algo,
                         "peak_source": HBM_SOURCE},
            "bit_exact_sample": bool(same), "sample": f"first {k} attempts against the oracle",
            "insert_size_stats": {"pairs": len(pairs), "kernel_ms": float(np.median(st_ms)),
                                  "fr": {f: float(stats[1][f]) for f in ("avg", "std", "low", "high", "failed")}}}


def run_reference(args):
    """The reference's own CPU implementation of the path, on the host cores: its SIMD batch
    kernels (sw_kernel_i16 in the widest vector width the CPU runs, fed chunk by chunk as the
    reference's dispatcher intends), restated in C++ in oracle/simd_baseline.cpp because the
    Rust crate cannot be built here.  One step = the whole 1M-job batch."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import ferrousalign_b200 as fa
    from oracle import ksw_oracle as O
    from oracle import simd_baseline as S
    b = make_workload(0, N_JOBS)
    p = fa.BandedPairWiseSW().to_struct()
    isa = S.best_isa()
    for _ in range(args.warmup):
        cpu_simd_rate(b, p, isa)
    times = []
    threads = os.cpu_count() or 1
    for _ in range(args.steps):
        dt, threads = cpu_simd_rate(b, p, isa)
        times.append(dt)
    dt = sum(times) / len(times)
    aln = N_JOBS / dt
    # GCUPS numerator: the batch's algorithmic cells (the scalar port's count, untimed)
    _, tr = O.ext_batch(p, b.jobs, b.qseq, b.tseq, threads=threads)
    cells = int(tr["cells"].sum())
    line = {
        "impl": "reference", "metric": METRIC, "value": aln, "unit": "alignments/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
        "config": {"workload": "1M right extensions, 151 bp reads, indel rate {0,0.1,1,3}%, w=100",
                   "jobs_per_step": N_JOBS, "w": 100, "zdrop": 100, "end_bonus": 5},
        "gcups": cells / dt / 1e9,
        "cpu_baseline": {"value": aln, "unit": "alignments/s", "cores": threads, "kind": "port",
                         "restates": SIMD_PATH[isa],
                         "sample": f"all {N_JOBS} jobs per step, chunks of the vector width, all host threads"},
        "e2e": {"value": aln, "unit": "alignments/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--jobs", type=int, default=N_JOBS)
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline leg")
    ap.add_argument("--skip-mate", action="store_true", help="omit the mate-rescue section")
    ap.add_argument("--skip-learned", action="store_true", help="omit the learned-band section")
    ap.add_argument("--skip-mixed", action="store_true", help="omit the mixed mate + extension batch section")
    ap.add_argument("--skip-uneven", action="store_true", help="omit the uneven-length batch section")
    ap.add_argument("--skip-regions", action="store_true", help="omit the region-merge section")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    n = args.jobs
    b = make_workload(rank, n)
    sw = fa.BandedPairWiseSW()
    p = sw.to_struct()
    ctx = fa.Context(local)
    lib = N.load()

    # ---- device-resident inputs -------------------------------------------------
    d_jobs = torch.from_numpy(b.jobs.view(np.uint8)).to(dev)
    d_q = torch.from_numpy(b.qseq).to(dev)
    d_t = torch.from_numpy(b.tseq).to(dev)
    d_out = torch.empty(n * 6, dtype=torch.int32, device=dev)
    # every launch of the timed region goes to one non-default stream, so the events
    # recorded on it bracket the library's kernels
    stream = torch.cuda.Stream(dev)
    # L2 flush buffer (inputs are > L2 already; flushing keeps every step cold)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    N.check(lib.fa_ctx_set_timing(ctx.handle, 1))
    import ctypes
    k_ms, k_n = ctypes.c_float(), ctypes.c_int()

    def step_device():
        N.check(lib.fa_ext_batch_device(ctx.handle, N.ptr(p), d_jobs.data_ptr(), n, d_q.data_ptr(), d_t.data_ptr(),
                                        None, d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            step_device()
    N.check(lib.fa_ctx_sync(ctx.handle))
    stream.synchronize()

    # ---- timed: device-resident ------------------------------------------------
    times, ktimes = [], []
    launches = 0
    with ClockSampler(local) as clk:
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step_device()
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                N.check(lib.fa_ctx_last_timing(ctx.handle, ctypes.byref(k_ms), ctypes.byref(k_n)))
                ktimes.append(k_ms.value)
                launches += k_n.value
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
    N.check(lib.fa_ctx_sync(ctx.handle))
    clocks = clk.summary()
    from ferrousalign_b200.replicas import max_over_ranks
    ms_step = max_over_ranks(float(np.mean(times)), dev)
    kernel_ms = float(np.mean(ktimes))

    # correctness on the timed outputs: a sample against the oracle, plus the cell count
    out = d_out.view(torch.int32).cpu().numpy().view(N.EXT_RESULT_DT).reshape(-1)
    from oracle import ksw_oracle as O
    chk = np.arange(0, n, max(1, n // 20000))
    sub = b.jobs[chk]
    ref_out, ref_tr = O.ext_batch(p, sub, b.qseq, b.tseq)
    exact = bool(np.array_equal(out[chk], ref_out))

    tune_dev = ctx.kernel_choice()   # autotuned kernel of the device-resident runs above
    # per-batch stats (cells, kernel time) from the host API run, also the e2e timing
    pin_jobs = torch.from_numpy(b.jobs.view(np.uint8)).pin_memory().numpy().view(N.JOB_DT)
    pin_q = torch.from_numpy(b.qseq).pin_memory().numpy()
    pin_t = torch.from_numpy(b.tseq).pin_memory().numpy()
    out_h = torch.empty(n * 24, dtype=torch.uint8).pin_memory().numpy().view(N.EXT_RESULT_DT)
    stats = np.zeros(1, N.STATS_DT)

    def step_host(st=None):
        N.check(lib.fa_ext_batch(ctx.handle, N.ptr(p), N.ptr(pin_jobs), n, N.ptr(pin_q), pin_q.nbytes,
                                 N.ptr(pin_t), pin_t.nbytes, out_h.ctypes.data, N.ptr(st)))

    step_host(stats)            # cells and kernel time of one batch (untimed)
    for _ in range(max(1, args.warmup) - 1):
        step_host()
    e2e_times = []
    if ws > 1:
        torch.distributed.barrier()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step_host()
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.mean(e2e_times)), dev)
    cells = int(stats[0]["cells"])
    exact = exact and np.array_equal(out_h[chk], ref_out)

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0

    # roofline: DPX int16x2 issue rate measured on this GPU
    v = ctypes.c_double()
    ms = ctypes.c_float()
    N.check(lib.fa_probe_int_peak(ctx.handle, 0, ctypes.byref(v), ctypes.byref(ms)))
    peak_ops = v.value
    N.check(lib.fa_probe_int_peak(ctx.handle, 2, ctypes.byref(v), ctypes.byref(ms)))
    peak_s32 = v.value
    peak_gcups = peak_ops * 2 / DPX_OPS_PER_CELL_PAIR / 1e9
    achieved_gcups = cells / (kernel_ms * 1e-3) / 1e9
    total_aln = n * ws
    value = total_aln / (ms_step * 1e-3)
    gcups_step = cells * ws / (ms_step * 1e-3) / 1e9
    bytes_in = int(b.jobs.nbytes + b.qseq.nbytes + b.tseq.nbytes)
    bytes_out = n * 24
    kname, kbytes, kdtype = EXT_KERNELS.get(tune_dev["kernel"], ("ext_packed_kernel", None, "int32"))
    line = {
        "metric": METRIC, "value": value, "unit": "alignments/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": kdtype, "data": "synthetic",
        "config": {"workload": "1M right extensions, 151 bp reads, indel rate {0,0.1,1,3}%, w=100",
                   "jobs_per_gpu": n, "w": 100, "zdrop": 100, "end_bonus": 5, "scoring": "A1 B4 N-1 O6 E1",
                   "l2": "inputs (%d MB) larger than L2; 256 MB flush between steps" % (bytes_in // 10**6),
                   "parallelism": f"replicas x{ws}"},
        "gcups": gcups_step,
        "bit_exact_sample": exact,
        "roofline": {"bound": "dpx", "achieved": achieved_gcups, "peak": peak_gcups, "unit": "Gcell/s",
                     "kernel": kname, "kernel_ms_per_step": kernel_ms,
                     "launches_per_step": launches / max(1, args.steps),
                     "frac": achieved_gcups / peak_gcups,
                     # DRAM bytes of one step's extension launches: the per-job read + write
                     # traffic of one ncu capture of that kernel (profiles/) times the step's jobs
                     "traffic": kbytes * n if kbytes else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per job, scaled",
                     "peak_source": f"measured __viaddmax_s16x2_relu rate {peak_ops / 1e12:.2f} Tops/s x2/"
                                    f"{DPX_OPS_PER_CELL_PAIR}; s32 DPX {peak_s32 / 1e12:.2f} Tops/s",
                     "hbm": {"achieved_gbs": (bytes_in + bytes_out) / (kernel_ms * 1e-3) / 1e9,
                             "peak_gbs": HBM_GBS, "peak_source": HBM_SOURCE}},
        "e2e": {"value": total_aln / (e2e_ms * 1e-3), "unit": "alignments/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": bytes_in + n * 4, "d2h_bytes_per_step": bytes_out},
        "gpu_launches": launches,
        "clocks": clocks,
        "autotune": tune_dev,
    }
    if not args.skip_learned:
        line["learned_band"] = bench_learned(args, ctx, b, p)
        forms = bench_e2e_forms(args, ctx, b, p)
        line["learned_band"]["e2e"] = forms
        line["e2e_packed"] = dict(forms["packed_single"], entry="fa_ext_batch_packed (2-bit packed host buffers)")
    if not args.skip_mate:
        line["mate_rescue"] = bench_mate(args, ctx, lib, dev, stream, flush, skip_cpu=args.skip_cpu)
    if not args.skip_mate and not args.skip_learned and not args.skip_mixed:
        line["mixed_batch"] = bench_mixed(args, b, p)
    if not args.skip_learned and not args.skip_uneven:
        line["uneven"] = bench_uneven(args, ctx, p)
    if not args.skip_regions:
        line["region_merge"] = bench_regions(args, ctx, lib, dev, stream, flush)
        line["job_collection"] = bench_collect(args, ctx, lib)
        line["cigar"] = bench_cigar(args, ctx, lib)
        line["rescue_collection"] = bench_rescue_collect(args, ctx, lib)
    if not args.skip_cpu:
        line["cpu_baseline"], line["cpu_baselines"] = cpu_baselines(b, p, cells)
    print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
