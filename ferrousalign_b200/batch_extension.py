"""Batched seed extension: the reference's batch-extension interface over the B200 kernels.

Mirrors src/pipelines/linear/batch_extension/{types.rs,dispatch.rs}:
``ExtensionJobBatch.add_job`` (types.rs:124-159) collects jobs into contiguous
query/reference buffers, ``execute_batch_simd_scoring`` (dispatch.rs:31-86) scores
them and returns one ``BatchExtensionResult`` per job in job order.  Scores follow
``ksw_extend2`` (src/core/alignment/ksw_affine_gap.rs:952-1169) exactly.

Errors: the reference panics where ksw_extend2 asserts (h0 <= 0) or a slice is out of
range; here those raise ``NativeError`` with code FA_ERR_ARG.  With
``BandedPairWiseSW(allow_h0_zero=True)`` jobs with h0 == 0 run the recurrence as written.  An empty batch returns
an empty list (dispatch.rs:36-38).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass

import numpy as np

from . import _native as N


class ExtensionDirection(enum.IntEnum):
    """types.rs:13-17"""
    Left = N.FA_DIR_LEFT
    Right = N.FA_DIR_RIGHT


def bwa_fill_scmat(match_score: int, mismatch_penalty: int, ambig_penalty: int = -1) -> np.ndarray:
    """5x5 scoring matrix, A C G T N (src/core/alignment/banded_swa/scoring.rs:2-27)."""
    mat = np.full((5, 5), ambig_penalty, dtype=np.int8)
    for i in range(4):
        for j in range(4):
            mat[i, j] = match_score if i == j else -mismatch_penalty
    return mat.reshape(25)


@dataclass
class BandedPairWiseSW:
    """Scoring parameters (src/core/alignment/banded_swa/types.rs:106-160)."""
    o_del: int = 6
    e_del: int = 1
    o_ins: int = 6
    e_ins: int = 1
    zdrop: int = 100
    end_bonus: int = 5
    pen_clip5: int = 5
    pen_clip3: int = 5
    mat: np.ndarray | None = None
    w_match: int = 1
    w_mismatch: int = -4
    # FA_PARAM_H0_ZERO: jobs with h0 == 0 (the reference's right jobs, collect_soa.rs:206)
    # run the recurrence as written instead of failing like ksw_extend2's assert
    allow_h0_zero: bool = False

    def __post_init__(self):
        if self.mat is None:
            self.mat = bwa_fill_scmat(self.w_match, -self.w_mismatch, -1)
        self.mat = np.asarray(self.mat, dtype=np.int8).reshape(25)

    def to_struct(self) -> np.ndarray:
        p = np.zeros(1, dtype=N.PARAMS_DT)
        p["mat"][0] = self.mat
        p["m"] = 5
        for k in ("o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus", "pen_clip5", "pen_clip3"):
            p[k] = getattr(self, k)
        p["flags"] = N.FA_PARAM_H0_ZERO if self.allow_h0_zero else 0
        return p


@dataclass
class BatchedExtensionJob:
    """types.rs:20-41"""
    read_idx: int
    chain_idx: int
    seed_idx: int
    direction: ExtensionDirection
    query_len: int
    ref_len: int
    h0: int
    band_width: int
    query_offset: int
    ref_offset: int


@dataclass
class BatchExtensionResult:
    """types.rs:45-66"""
    read_idx: int
    chain_idx: int
    seed_idx: int
    direction: ExtensionDirection
    score: int
    query_end: int
    ref_end: int
    gscore: int
    gref_end: int
    max_off: int


class ExtensionJobBatch:
    """Jobs plus contiguous query/reference code buffers (types.rs:74-183)."""

    def __init__(self, job_capacity: int = 1024, seq_capacity: int = 65536):
        self.jobs: list[BatchedExtensionJob] = []
        self._q = bytearray()
        self._r = bytearray()
        self.query_offset = 0
        self.ref_offset = 0

    def add_job(self, read_idx, chain_idx, seed_idx, direction, query_seq, ref_seq, h0, band_width):
        q = bytes(bytearray(query_seq))
        r = bytes(bytearray(ref_seq))
        self.jobs.append(BatchedExtensionJob(read_idx, chain_idx, seed_idx, ExtensionDirection(direction),
                                             len(q), len(r), int(h0), int(band_width),
                                             self.query_offset, self.ref_offset))
        self._q += q
        self._r += r
        self.query_offset += len(q)
        self.ref_offset += len(r)

    def get_query_seq(self, i: int) -> bytes:
        j = self.jobs[i]
        return bytes(self._q[j.query_offset:j.query_offset + j.query_len])

    def get_ref_seq(self, i: int) -> bytes:
        j = self.jobs[i]
        return bytes(self._r[j.ref_offset:j.ref_offset + j.ref_len])

    def __len__(self) -> int:
        return len(self.jobs)

    def is_empty(self) -> bool:
        return not self.jobs

    def clear(self) -> None:
        self.__init__()

    def to_arrays(self):
        jobs = np.zeros(len(self.jobs), dtype=N.JOB_DT)
        for i, j in enumerate(self.jobs):
            jobs[i] = (j.query_offset, j.ref_offset, j.query_len, j.ref_len, j.h0, j.band_width,
                       int(j.direction), 0)
        q = np.frombuffer(bytes(self._q), dtype=np.uint8) if self._q else np.zeros(1, np.uint8)
        r = np.frombuffer(bytes(self._r), dtype=np.uint8) if self._r else np.zeros(1, np.uint8)
        return jobs, q, r


def make_policy(mode: int = N.FA_POLICY_SINGLE, max_tries: int = 2, judge: int = N.FA_JUDGE_CERT,
                w_min: int = 1) -> np.ndarray:
    p = np.zeros(1, dtype=N.POLICY_DT)
    p["mode"], p["max_tries"], p["judge"], p["w_min"] = mode, max_tries, judge, w_min
    return p


def extend_batch(params: np.ndarray, jobs: np.ndarray, qseq: np.ndarray, tseq: np.ndarray,
                 policy: np.ndarray | None = None, w_first: np.ndarray | None = None,
                 ctx: N.Context | None = None, out: np.ndarray | None = None, bands: bool = True):
    """Array-level call of fa_ext_batch_policy.  Returns (results, stats, w_final); `out`
    may be a (pinned) result buffer to fill; bands=False asks for no final bands (None)."""
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, dtype=N.JOB_DT)
    qseq = np.ascontiguousarray(qseq, dtype=np.uint8)
    tseq = np.ascontiguousarray(tseq, dtype=np.uint8)
    n = len(jobs)
    out = np.zeros(n, dtype=N.EXT_RESULT_DT) if out is None else out
    stats = np.zeros(1, dtype=N.STATS_DT)
    w_final = np.zeros(n, dtype=np.int32) if bands else None
    wf = None if w_first is None else np.ascontiguousarray(w_first, dtype=np.int32)
    N.check(lib.fa_ext_batch_policy(ctx.handle, N.ptr(params), N.ptr(policy), N.ptr(jobs), n,
                                    N.ptr(qseq), qseq.nbytes, N.ptr(tseq), tseq.nbytes, N.ptr(wf),
                                    N.ptr(out), N.ptr(w_final), N.ptr(stats)))
    return out, stats[0], w_final


def execute_batch_simd_scoring(sw_params: BandedPairWiseSW, batch: ExtensionJobBatch,
                               engine=None) -> list[BatchExtensionResult]:
    """dispatch.rs:31-86.  ``engine`` is accepted for signature compatibility."""
    if batch.is_empty():
        return []
    jobs, q, r = batch.to_arrays()
    out, _, _ = extend_batch(sw_params.to_struct(), jobs, q, r)
    res = []
    for j, o in zip(batch.jobs, out):
        res.append(BatchExtensionResult(j.read_idx, j.chain_idx, j.seed_idx, j.direction, int(o["score"]),
                                        int(o["qle"]), int(o["tle"]), int(o["gscore"]), int(o["gtle"]),
                                        int(o["max_off"])))
    return res
