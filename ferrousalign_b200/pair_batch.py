"""One submission of a paired-end batch's two kinds of GPU work: seed extensions
(execute_batch_simd_scoring, src/pipelines/linear/batch_extension/dispatch.rs:31-86) and
mate-rescue local SW (execute_mate_rescue_batch_with_engine,
src/pipelines/linear/paired/mate_rescue.rs:595-685), through fa_pair_batch: the mate kernels
run on their own stream while the extension rounds run on the context's main stream."""
from __future__ import annotations

import numpy as np

from . import _native as N


def pair_batch(params: np.ndarray, jobs: np.ndarray, qseq: np.ndarray, tseq: np.ndarray,
               mate_params: np.ndarray, mate_jobs: np.ndarray, mate_qseq: np.ndarray, mate_tseq: np.ndarray,
               policy: np.ndarray | None = None, model=None, hints: np.ndarray | None = None,
               margin: float = 0.0, ctx: N.Context | None = None, out: np.ndarray | None = None,
               mate_out: np.ndarray | None = None):
    """Returns (extension results, mate kswr records, extension stats, mate stats).  With
    `model` (a BandModel) the extensions take the learned first band and `policy` must be a
    FA_POLICY_LEARNED policy (the default then); otherwise `policy` defaults to the
    single-band policy.  `out` / `mate_out` may be (pinned) result buffers to fill; pinned
    input arrays let both uploads run asynchronously."""
    from .batch_extension import make_policy
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, dtype=N.JOB_DT)
    qseq = np.ascontiguousarray(qseq, dtype=np.uint8)
    tseq = np.ascontiguousarray(tseq, dtype=np.uint8)
    mate_jobs = np.ascontiguousarray(mate_jobs, dtype=N.MATE_JOB_DT)
    mate_qseq = np.ascontiguousarray(mate_qseq, dtype=np.uint8)
    mate_tseq = np.ascontiguousarray(mate_tseq, dtype=np.uint8)
    if policy is None and model is not None:
        from .band_model import JUDGE_LEARNED
        policy = make_policy(N.FA_POLICY_LEARNED, 2, JUDGE_LEARNED, 2)
    n, mn = len(jobs), len(mate_jobs)
    out = np.zeros(n, dtype=N.EXT_RESULT_DT) if out is None else out
    mate_out = np.zeros(mn, dtype=N.KSWR_DT) if mate_out is None else mate_out
    st = np.zeros(1, dtype=N.STATS_DT)
    mst = np.zeros(1, dtype=N.STATS_DT)
    from .band_model import HINT_DT
    h = None if hints is None else np.ascontiguousarray(hints, HINT_DT)
    N.check(lib.fa_pair_batch(ctx.handle, N.ptr(params), N.ptr(policy), None if model is None else model.handle,
                              margin, N.ptr(jobs), n, N.ptr(qseq), qseq.nbytes, N.ptr(tseq), tseq.nbytes,
                              N.ptr(h), N.ptr(out), N.ptr(mate_params), N.ptr(mate_jobs), mn, N.ptr(mate_qseq),
                              mate_qseq.nbytes, N.ptr(mate_tseq), mate_tseq.nbytes, N.ptr(mate_out),
                              N.ptr(st), N.ptr(mst)))
    return out, mate_out, st[0], mst[0]
