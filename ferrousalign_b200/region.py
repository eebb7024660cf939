"""Alignment regions from extension results: the host mirror of merge_scores_to_regions
(src/pipelines/linear/region.rs:737-890).

For each chain, every seed's region from its left and right extension results (bwa-mem2's
clip decision per side, region.rs:792-835), its total score, true score and seed
coverage, and the region of the chain's first seed with the strictly highest total score.
The merge runs as one CUDA kernel over all chains of a batch (csrc/region_kernel.cu);
reference positions stay in FM-index space, as in the reference before its coordinate
conversion (coordinates.rs), which needs the index and stays with the caller.
"""
from __future__ import annotations

from typing import Iterable, Sequence

import numpy as np

from . import _native as N

REGION_DT = N.REGION_DT
SEED_EXT_DT = N.SEED_EXT_DT


def region_opts(a: int = 1, pen_clip5: int = 5, pen_clip3: int = 5, w: int = 100) -> np.ndarray:
    """MemOpt's fields the merge reads (mem_opt.rs: a, pen_clip5, pen_clip3, w)."""
    o = np.zeros(1, N.REGION_OPTS_DT)
    o["a"], o["pen_clip5"], o["pen_clip3"], o["w"] = a, pen_clip5, pen_clip3, w
    return o


def chain_seed_table(chains: Iterable[Sequence[tuple]], mapping_order: bool = True):
    """(chain_first, seeds) from per-chain lists of (ref_pos, query_pos, len, left_job,
    right_job) in chain order.  mapping_order: list each chain's seeds last to first, the
    order the reference builds its SeedExtensionMapping list in (region.rs:397), which
    decides ties between equal totals."""
    first = [0]
    rows = []
    for ch in chains:
        seq = list(ch)[::-1] if mapping_order else list(ch)
        rows.extend(seq)
        first.append(len(rows))
    seeds = np.zeros(len(rows), SEED_EXT_DT)
    for k, (rp, qp, ln, lj, rj) in enumerate(rows):
        seeds[k] = (rp, qp, ln, -1 if lj is None else lj, -1 if rj is None else rj)
    return np.asarray(first, np.uint32), seeds


def merge_scores_to_regions(chain_first: np.ndarray, query_len: np.ndarray, seeds: np.ndarray,
                            left_scores: np.ndarray, right_scores: np.ndarray, opts: np.ndarray | None = None,
                            ctx: N.Context | None = None) -> np.ndarray:
    """One region per chain (REGION_DT; seed = index into `seeds`, -1 for a chain without
    seeds).  left_scores/right_scores are the EXT_RESULT_DT outputs of the left and right
    extension batches, indexed by the seeds' left_job/right_job."""
    lib = N.load()
    ctx = ctx or N.default_context()
    opts = region_opts() if opts is None else opts
    chain_first = np.ascontiguousarray(chain_first, np.uint32)
    n = len(chain_first) - 1
    query_len = np.ascontiguousarray(query_len, np.int32)
    if len(query_len) != n:
        raise ValueError("query_len needs one entry per chain")
    seeds = np.ascontiguousarray(seeds, SEED_EXT_DT)
    left = np.ascontiguousarray(left_scores, N.EXT_RESULT_DT)
    right = np.ascontiguousarray(right_scores, N.EXT_RESULT_DT)
    out = np.zeros(max(n, 0), REGION_DT)
    if n <= 0:
        return out
    N.check(lib.fa_merge_regions(ctx.handle, N.ptr(opts), N.ptr(chain_first), n, N.ptr(query_len),
                                 N.ptr(seeds) if len(seeds) else None, len(seeds),
                                 N.ptr(left) if len(left) else None, len(left),
                                 N.ptr(right) if len(right) else None, len(right), N.ptr(out)))
    return out
