"""Trains the band predictor on the GPU and evaluates it on a held-out batch.

Training set: 5,000,000 right extensions of the 151-bp generator with per-read indel
rates {0, 0.1, 1, 3}% (seed 4); labels: the smallest band of the ladder 4..64 whose
single run reproduces the plain bwa-mem2 policy's result and passes the acceptance
judge (else the configured band).  Evaluation: a fresh 1,000,000-job batch from
disjoint generator seeds, plain policy vs learned path: identical outputs, miss rate,
executed and saved cells, kernel time.

    python -m ferrousalign_b200.train_band_model --out band_model_151bp.bin [--train N] [--eval N]
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


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(B.DEFAULT_MODEL))
    ap.add_argument("--train", type=int, default=5_000_000)
    ap.add_argument("--eval", type=int, default=1_000_000)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--tau", type=float, default=0.6)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--margin", type=float, default=0.0)
    ap.add_argument("--w-min", type=int, default=16)
    args = ap.parse_args(argv)
    ctx = N.default_context()
    p = fa.BandedPairWiseSW().to_struct()
    bwa = fa.make_policy(N.FA_POLICY_BWA, 2)

    t0 = time.time()
    tr = synth.workload_ext_train(args.train, seed=4)
    log(f"train set {args.train} jobs in {time.time() - t0:.1f}s")
    plain, pst, _ = fa.extend_batch(p, tr.jobs, tr.qseq, tr.tseq, policy=bwa, ctx=ctx)
    t0 = time.time()
    label, ladder_cells = B.make_labels(p, tr.jobs, tr.qseq, tr.tseq, plain, ctx=ctx)
    log(f"labels in {time.time() - t0:.1f}s; histogram {dict(zip(*np.unique(label, return_counts=True)))}")
    hints = B.hints_from_info(tr.info)
    x = B.features(p, tr.jobs, tr.qseq, tr.tseq, hints, ctx=ctx)
    target = np.log2(label.astype(np.float32))
    model = B.BandModel.create(seed=11)
    model.fit_norm(x)
    t0 = time.time()
    losses = model.train(x, target, epochs=args.epochs, batch=8192, lr=args.lr, tau=args.tau, ctx=ctx)
    log(f"trained {args.epochs} epochs in {time.time() - t0:.1f}s; loss {losses.tolist()}")
    model.save(args.out)
    del tr, x, plain

    # held-out evaluation (disjoint generator seeds)
    ev = synth.workload_ext_1m(args.eval, seed=2 + 7919)
    ev_hints = B.hints_from_info(ev.info)
    plain, pst, _ = fa.extend_batch(p, ev.jobs, ev.qseq, ev.tseq, policy=bwa, ctx=ctx)
    res = {"w_min": args.w_min, "train_jobs": args.train, "eval_jobs": args.eval, "epochs": args.epochs, "tau": args.tau,
           "train_loss": [float(v) for v in losses],
           "label_hist": {int(k): int(v) for k, v in zip(*np.unique(label, return_counts=True))},
           "plain": {"cells_executed": int(pst["cells_executed"]), "kernel_ms": float(pst["kernel_ms"])}}
    for name, judge in (("fast", B.JUDGE_FAST),):
        out, st, wf, wfin = B.extend_batch_learned(p, ev.jobs, ev.qseq, ev.tseq, model, hints=ev_hints, judge=judge,
                                                   margin=args.margin, w_min=args.w_min, ctx=ctx)
        ident = bool(np.array_equal(out, plain))
        res[name] = {"identical_all": ident, "identical_frac": float(np.mean(out == plain)),
                     "miss_rate": float(st["misses"]) / args.eval,
                     "cells_executed": int(st["cells_executed"]),
                     "cells_saved_frac": 1.0 - float(st["cells_executed"]) / float(pst["cells_executed"]),
                     "kernel_ms": float(st["kernel_ms"]),
                     "w_first_median": float(np.median(wf)), "retries": int(st["retries"])}
    # the method without the network: every job starts at a fixed narrow band
    for w0 in (16, 24, 32):
        wf = np.full(args.eval, w0, np.int32)
        out, st, _ = fa.extend_batch(p, ev.jobs, ev.qseq, ev.tseq,
                                     policy=fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_FAST, 1), w_first=wf,
                                     ctx=ctx)
        res[f"fixed_w{w0}"] = {"identical_all": bool(np.array_equal(out, plain)),
                               "miss_rate": float(st["misses"]) / args.eval,
                               "cells_executed": int(st["cells_executed"]), "kernel_ms": float(st["kernel_ms"])}
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
