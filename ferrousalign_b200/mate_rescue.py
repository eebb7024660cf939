"""Mate-rescue local Smith-Waterman over the B200 kernels.

Mirrors ``execute_mate_rescue_batch_with_engine``
(src/pipelines/linear/paired/mate_rescue.rs:595-685): one ``ksw_align2`` per job with
the reference's flags (XSUBO | XSTART | XBYTE when mate_len * match_score < 250, and
min_seed_len * match_score as the sub-optimal threshold), the rescue scoring matrix
(mate_rescue.rs:116-122: match 1, mismatch -4, N 0) and gaps 6/1.  Results are
``Kswr`` records (src/core/alignment/ksw_affine_gap.rs:51-61) in job order.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .hostbuf import HostBuffers, out_array

MATE_RESCUE_SCORING_MATRIX = np.array([
    1, -4, -4, -4, 0,
    -4, 1, -4, -4, 0,
    -4, -4, 1, -4, 0,
    -4, -4, -4, 1, 0,
    0, 0, 0, 0, 0], dtype=np.int8)


@dataclass
class Kswr:
    score: int
    te: int
    qe: int
    score2: int
    te2: int
    tb: int
    qb: int


@dataclass
class MateRescueJob:
    """The fields of mate_rescue.rs:37-64 that the SW call consumes."""
    query_seq: bytes
    ref_seq: bytes
    mate_len: int
    min_seed_len: int = 19
    match_score: int = 1
    pair_index: int = 0
    extra: dict = field(default_factory=dict)


@dataclass
class MateRescueResult:
    job_index: int
    aln: Kswr


def mate_xtra(mate_len: int, match_score: int, min_seed_len: int) -> int:
    """mate_rescue.rs:314-321"""
    x = N.KSW_XSUBO | N.KSW_XSTART
    if mate_len * match_score < 250:
        x |= N.KSW_XBYTE
    return x | (min_seed_len * match_score)


def make_mate_params(mat=MATE_RESCUE_SCORING_MATRIX, o_del=6, e_del=1, o_ins=6, e_ins=1) -> np.ndarray:
    p = np.zeros(1, dtype=N.MATE_PARAMS_DT)
    p["mat"][0] = np.asarray(mat, dtype=np.int8).reshape(25)
    p["m"] = 5
    p["o_del"], p["e_del"], p["o_ins"], p["e_ins"] = o_del, e_del, o_ins, e_ins
    return p


def mate_sw_batch(params: np.ndarray, jobs: np.ndarray, qseq: np.ndarray, tseq: np.ndarray,
                  ctx: N.Context | None = None, out: np.ndarray | None = None):
    """Array-level call of fa_mate_sw_batch.  Returns (kswr records, stats); `out` may be a
    (page-locked) result buffer to fill."""
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, dtype=N.MATE_JOB_DT)
    qseq = np.ascontiguousarray(qseq, dtype=np.uint8)
    tseq = np.ascontiguousarray(tseq, dtype=np.uint8)
    out = np.zeros(len(jobs), dtype=N.KSWR_DT) if out is None else out
    stats = np.zeros(1, dtype=N.STATS_DT)
    N.check(lib.fa_mate_sw_batch(ctx.handle, N.ptr(params), N.ptr(jobs), len(jobs), N.ptr(qseq), qseq.nbytes,
                                 N.ptr(tseq), tseq.nbytes, N.ptr(out), N.ptr(stats)))
    return out, stats[0]


def mate_sw_batch_packed(params: np.ndarray, jobs: np.ndarray, qseq, tseq, ctx: N.Context | None = None,
                         out: np.ndarray | None = None):
    """fa_mate_sw_batch_packed on PackedSeq buffers (packed.pack).  Returns (kswr records,
    stats), those of mate_sw_batch on the same bases; `out` as for mate_sw_batch."""
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, dtype=N.MATE_JOB_DT)
    out = np.zeros(len(jobs), dtype=N.KSWR_DT) if out is None else out
    stats = np.zeros(1, dtype=N.STATS_DT)
    qs, ts = qseq.struct(), tseq.struct()
    N.check(lib.fa_mate_sw_batch_packed(ctx.handle, N.ptr(params), N.ptr(jobs), len(jobs), N.ptr(qs), N.ptr(ts),
                                        N.ptr(out), N.ptr(stats)))
    return out, stats[0]


def execute_mate_rescue_batch_with_engine(jobs: list[MateRescueJob], engine=None) -> list[MateRescueResult]:
    """mate_rescue.rs:595-637.  ``engine`` is accepted for signature compatibility."""
    if not jobs:
        return []
    arr = np.zeros(len(jobs), dtype=N.MATE_JOB_DT)
    qb, tb = bytearray(), bytearray()
    for i, j in enumerate(jobs):
        q, t = bytes(bytearray(j.query_seq)), bytes(bytearray(j.ref_seq))
        arr[i] = (len(qb), len(tb), j.mate_len, len(t), mate_xtra(j.mate_len, j.match_score, j.min_seed_len), 0)
        qb += q[:j.mate_len]
        tb += t
    q = np.frombuffer(bytes(qb), dtype=np.uint8) if qb else np.zeros(1, np.uint8)
    t = np.frombuffer(bytes(tb), dtype=np.uint8) if tb else np.zeros(1, np.uint8)
    out, _ = mate_sw_batch(make_mate_params(), arr, q, t)
    return [MateRescueResult(i, Kswr(*(int(v) for v in o))) for i, o in enumerate(out)]


# ---- rescue jobs from anchors (collect_rescue_jobs_for_read_soa, mate_rescue.rs:1804-2045)

def rescue_opts(pen_unpaired: int = 17, max_matesw: int = 50, min_seed_len: int = 19,
                match_score: int = 1) -> np.ndarray:
    """MemOpt's pen_unpaired and max_matesw, the index's min_seed_len, the match score."""
    o = np.zeros(1, N.RESCUE_OPTS_DT)
    o["pen_unpaired"], o["max_matesw"], o["min_seed_len"], o["match_score"] = (pen_unpaired, max_matesw,
                                                                               min_seed_len, match_score)
    return o


@dataclass
class RescueJobs:
    jobs: np.ndarray     # MATE_JOB_DT, for mate_sw_batch with qbuf / tbuf
    info: np.ndarray     # RESCUE_JOB_INFO_DT: attempt, orientation, strand, window
    qbuf: np.ndarray
    tbuf: np.ndarray


def collect_rescue_jobs(pac: np.ndarray, l_pac: int, chr_off: np.ndarray, chr_len: np.ndarray,
                        reads: np.ndarray, read_off: np.ndarray, alns: np.ndarray, cands: np.ndarray,
                        bounds: np.ndarray, opts: np.ndarray | None = None,
                        ctx: N.Context | None = None, bufs: HostBuffers | None = None) -> RescueJobs:
    """Mate-rescue jobs of every attempt (RESCUE_CAND_DT) on the GPU; bounds is
    INSERT_BOUNDS_DT[4] (FF, FR, RF, RR: low, high, failed).  pac=None reads the reference the
    context keeps (Context.set_reference).  With `bufs` the outputs land in those reusable
    (page-locked) buffers and the result views them."""
    lib = N.load()
    ctx = ctx or N.default_context()
    opts = rescue_opts() if opts is None else opts
    pac = None if pac is None else np.ascontiguousarray(pac, np.uint8)   # None: the context's resident reference
    chr_off = np.ascontiguousarray(chr_off, np.uint64)
    chr_len = np.ascontiguousarray(chr_len, np.uint64)
    reads = np.ascontiguousarray(reads, np.uint8)
    read_off = np.ascontiguousarray(read_off, np.uint64)
    alns = np.ascontiguousarray(alns, N.RESCUE_ALN_DT)
    cands = np.ascontiguousarray(cands, N.RESCUE_CAND_DT)
    bounds = np.ascontiguousarray(bounds, N.INSERT_BOUNDS_DT)
    n = len(cands)
    # written in full up to the returned counts; uninitialised, so untouched pages stay unmapped
    jobs = out_array(bufs, "jobs", 4 * n, N.MATE_JOB_DT)
    info = out_array(bufs, "info", 4 * n, N.RESCUE_JOB_INFO_DT)
    counts = np.zeros(1, N.COLLECT_COUNTS_DT)
    qlen = np.diff(read_off.astype(np.int64))
    qcap = int(4 * qlen[cands["read"]].sum()) if n else 0
    span = int(np.maximum(bounds["high"] - bounds["low"], 0).max()) if len(bounds) else 0
    tcap = int(4 * (qlen[cands["read"]] + span + 1).sum()) if n else 0
    for _ in range(2):
        qbuf = out_array(bufs, "qbuf", max(qcap, 1), np.uint8)
        tbuf = out_array(bufs, "tbuf", max(tcap, 1), np.uint8)
        rc = lib.fa_collect_mate_jobs(ctx.handle, N.ptr(opts), N.ptr(bounds), N.ptr(pac), l_pac, N.ptr(chr_off),
                                      N.ptr(chr_len), len(chr_off), N.ptr(reads), N.ptr(read_off),
                                      len(read_off) - 1, N.ptr(alns), len(alns), N.ptr(cands), n, N.ptr(jobs),
                                      N.ptr(info), N.ptr(qbuf), qcap, N.ptr(tbuf), tcap, N.ptr(counts))
        c = counts[0]
        if rc == N.FA_ERR_CAPACITY and (int(c["qbuf_len"]) > qcap or int(c["tbuf_len"]) > tcap):
            qcap, tcap = max(qcap, int(c["qbuf_len"])), max(tcap, int(c["tbuf_len"]))
            continue
        N.check(rc)
        break
    k = int(counts[0]["n_left"])
    return RescueJobs(jobs[:k], info[:k], qbuf[:int(counts[0]["qbuf_len"])],
                      tbuf[:int(counts[0]["tbuf_len"])])


def calculate_insert_size_stats(l_pac: int, pairs: np.ndarray, ctx: N.Context | None = None) -> np.ndarray:
    """InsertSizeStats of the four orientations (FF, FR, RF, RR) from pairs of FM-index
    positions (n x 2 int64: read 1, read 2), on the GPU (insert_size.rs:73-243)."""
    lib = N.load()
    ctx = ctx or N.default_context()
    pairs = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
    out = np.zeros(4, N.INSERT_STATS_DT)
    N.check(lib.fa_insert_size_stats(ctx.handle, l_pac, N.ptr(pairs) if len(pairs) else None, len(pairs),
                                     N.ptr(out)))
    return out


def insert_bounds(stats: np.ndarray) -> np.ndarray:
    """The bounds the rescue-job collection reads, from InsertSizeStats."""
    b = np.zeros(4, N.INSERT_BOUNDS_DT)
    b["low"], b["high"], b["failed"] = stats["low"], stats["high"], stats["failed"]
    return b
