"""Trains the band predictor on the GPU and evaluates it on a held-out batch.

Training set: 5,000,000 right extensions of the 151-bp generator with per-read indel
rates {0, 0.1, 1, 3}% (seed 4).  Label: the smallest band of the doubling ladders from 2
and 3 whose run the exit-bound certificate proves equal to the configured-band run (the
configured band when none does).  One model is trained per pinball quantile tau and
evaluated with three retry rules (doubling; one narrow try then the configured band; one
narrow try, one retry at the band the certificate's shortfall suggests, then the configured
band);
the pair with the shortest extension time on a validation batch (seed 6) is kept.  Evaluation on
a fresh 1,000,000-job batch from disjoint generator seeds: the plain bwa-mem2 policy
against the learned path (outputs must be identical), miss rate, executed and saved
cells, kernel time, and the same policy without the network (every job starting at one
fixed band).

    python -m ferrousalign_b200.train_band_model --out band_model_151bp.bin [--train N] [--eval N]

With --shape uneven the three batches come from the uneven generator instead: mixed left and
right extensions of 50-300 bp reads, seeds anywhere in the read, a reference with 5%
low-complexity repeats (training seed 14, validation 16, evaluation 19; the bench's uneven
batch uses seed 3), and the model goes to band_model_uneven.bin.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

import ferrousalign_b200 as fa
from . import _native as N
from . import band_model as B
from . import synth

FIXED_FIRST = (2, 3, 4, 6, 8, 12, 16, 24, 32)


def uneven_batch(n: int, seed: int) -> synth.ExtBatch:
    """The uneven shape (synth.workload_ext_uneven) on a 20 Mbp reference of its own seed."""
    ref = synth.reference(20_000_000, seed=seed, n_rate=0.001, repeat_frac=0.05)
    return synth.ext_jobs(ref, n, seed=seed + 100, read_len=(50, 300), seed_at_start=False, indel_rates=(0.001,))


# generators per shape: (training, validation, evaluation) batches
SHAPES = {
    "151": (lambda n: synth.workload_ext_train(n, seed=4), lambda n: synth.workload_ext_1m(n, seed=6),
            lambda n: synth.workload_ext_1m(n, seed=2 + 7919)),
    "uneven": (lambda n: uneven_batch(n, 14), lambda n: uneven_batch(n, 16), lambda n: uneven_batch(n, 19)),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def run_learned(p, batch, model, w_min, ctx, reps=2, judge=None):
    """Learned path, best kernel time of `reps` runs (outputs of the last)."""
    hints = B.hints_from_info(batch.info)
    judge = B.JUDGE_EXACT if judge is None else judge
    best = None
    for _ in range(reps):
        out, st, wf, wfin = B.extend_batch_learned(p, batch.jobs, batch.qseq, batch.tseq, model, hints=hints,
                                                   judge=judge, w_min=w_min, ctx=ctx)
        if best is None or st["kernel_ms"] < best[1]["kernel_ms"]:
            best = (out, st, wf, wfin)
    return best


def run_fixed(p, batch, w0, ctx, reps=2, judge=None):
    wf = np.full(len(batch.jobs), w0, np.int32)
    pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_EXACT if judge is None else judge, 1)
    best = None
    for _ in range(reps):
        out, st, _ = fa.extend_batch(p, batch.jobs, batch.qseq, batch.tseq, policy=pol, w_first=wf, ctx=ctx)
        if best is None or st["kernel_ms"] < best[1]["kernel_ms"]:
            best = (out, st)
    return best


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--shape", choices=sorted(SHAPES), default="151")
    ap.add_argument("--train", type=int, default=5_000_000)
    ap.add_argument("--val", type=int, default=500_000)
    ap.add_argument("--eval", type=int, default=1_000_000)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--taus", default="0.5,0.6,0.7,0.8")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--w-min", type=int, default=2)
    args = ap.parse_args(argv)
    if args.out is None:
        args.out = str(B.DEFAULT_MODEL if args.shape == "151" else B.UNEVEN_MODEL)
    gen_train, gen_val, gen_eval = SHAPES[args.shape]
    ctx = N.default_context()
    ctx.set_slices(1, 1)   # kernel times of whole-batch runs
    p = fa.BandedPairWiseSW().to_struct()
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)

    t0 = time.time()
    tr = gen_train(args.train)
    log(f"train set {args.train} jobs in {time.time() - t0:.1f}s")
    t0 = time.time()
    label, ladder_cells = B.make_labels(p, tr.jobs, tr.qseq, tr.tseq, ctx=ctx)
    hist = {int(k): int(v) for k, v in zip(*np.unique(label, return_counts=True))}
    log(f"labels in {time.time() - t0:.1f}s; histogram {hist}")
    x = B.features(p, tr.jobs, tr.qseq, tr.tseq, B.hints_from_info(tr.info), ctx=ctx)
    target = np.log2(label.astype(np.float32))
    del tr

    val = gen_val(args.val)
    val_plain, _, _ = fa.extend_batch(p, val.jobs, val.qseq, val.tseq, policy=bwa, ctx=ctx)
    best = None
    sweep = {}
    for tau in (float(t) for t in args.taus.split(",")):
        model = B.BandModel.create(seed=11)
        model.fit_norm(x)
        t0 = time.time()
        losses = model.train(x, target, epochs=args.epochs, batch=8192, lr=args.lr, tau=tau, ctx=ctx)
        for rule, judge in (("double", B.JUDGE_EXACT), ("once", B.JUDGE_EXACT | N.FA_JUDGE_ONCE),
                            ("hint", B.JUDGE_EXACT | N.FA_JUDGE_ONCE | N.FA_JUDGE_HINT)):
            out, st, wf, _ = run_learned(p, val, model, args.w_min, ctx, judge=judge)
            if not np.array_equal(out, val_plain):
                raise RuntimeError(f"tau {tau}: learned path differs from the plain path on the validation batch")
            key = f"{tau}/{rule}"
            sweep[key] = {"val_kernel_ms": float(st["kernel_ms"]), "val_cells_executed": int(st["cells_executed"]),
                          "val_miss_rate": float(st["misses"]) / len(val.jobs), "final_loss": float(losses[-1])}
            log(f"tau {key}: trained in {time.time() - t0:.1f}s, {sweep[key]}")
            if best is None or st["kernel_ms"] < best[1]:
                best = (tau, float(st["kernel_ms"]), model, losses, judge, rule)
    tau, _, model, losses, judge, rule = best
    model.save(args.out)
    del x, val

    # held-out evaluation (disjoint generator seeds)
    ev = gen_eval(args.eval)
    plain, pst, _ = fa.extend_batch(p, ev.jobs, ev.qseq, ev.tseq, policy=bwa, ctx=ctx)
    out, st, wf, wfin = run_learned(p, ev, model, args.w_min, ctx, judge=judge)
    res = {"shape": args.shape, "w_min": args.w_min, "train_jobs": args.train, "eval_jobs": args.eval, "epochs": args.epochs,
           "tau": tau, "retry_rule": rule, "judge": judge, "tau_sweep": sweep, "train_loss": [float(v) for v in losses], "label_hist": hist,
           "plain": {"cells_executed": int(pst["cells_executed"]), "kernel_ms": float(pst["kernel_ms"])},
           "learned": {"identical_all": bool(np.array_equal(out, plain)),
                       "miss_rate": float(st["misses"]) / args.eval,
                       "cells_executed": int(st["cells_executed"]),
                       "cells_saved_frac": 1.0 - float(st["cells_executed"]) / float(pst["cells_executed"]),
                       "kernel_ms": float(st["kernel_ms"]), "w_first_median": float(np.median(wf)),
                       "retries": int(st["retries"])}}
    # the same policy without the network: every job starts at one fixed band
    fixed = {}
    for w0 in FIXED_FIRST:
        o, s = run_fixed(p, ev, w0, ctx, judge=judge)
        fixed[w0] = {"identical_all": bool(np.array_equal(o, plain)), "miss_rate": float(s["misses"]) / args.eval,
                     "cells_executed": int(s["cells_executed"]), "kernel_ms": float(s["kernel_ms"])}
    res["fixed_first_band"] = fixed
    best_fixed = min(fixed, key=lambda k: fixed[k]["kernel_ms"])
    res["network_gain"] = {"best_fixed_first_band": best_fixed,
                           "kernel_time_ratio": fixed[best_fixed]["kernel_ms"] / res["learned"]["kernel_ms"],
                           "cells_ratio": fixed[best_fixed]["cells_executed"] / res["learned"]["cells_executed"]}
    res["speedup_vs_plain"] = res["plain"]["kernel_ms"] / res["learned"]["kernel_ms"]
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
