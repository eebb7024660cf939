"""CIGAR regeneration: the host mirror of scalar_banded_swa
(src/core/alignment/banded_swa/scalar/implementation.rs:5-440) as a batch on the GPU
(csrc/cigar_kernel.cu), and infer_band_width (src/pipelines/linear/region.rs:1277-1316),
which picks each job's band.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .hostbuf import HostBuffers, out_array

CIGAR_JOB_DT = N.CIGAR_JOB_DT
CIGAR_RESULT_DT = N.CIGAR_RESULT_DT
CIGAR_OPS = "MIDNS"   # op codes 0-4 of the packed CIGAR words (len << 4 | op)


def infer_band_width(l_query: int, l_ref: int, score: int, a: int, o_del: int, e_del: int, o_ins: int,
                     e_ins: int, cmd_w: int, region_w: int) -> int:
    """Band for regenerating a region's CIGAR (bwamem.cpp:1752-1756 in the reference's
    port): from the score lost to gaps on either axis, at least the length difference,
    the region's own band when above the command-line one, at most four times that."""
    def side(o: int, e: int) -> int:
        if l_query == l_ref and l_query * a - score < (o + e - a) * 2:
            return 0
        x = float(min(l_query, l_ref) * a - score - o)
        q = x / e if e else (math.inf if x > 0 else -math.inf if x < 0 else math.nan)
        q += 2.0
        v = 0 if math.isnan(q) else (2**31 - 1 if q >= 2**31 - 1 else -2**31 if q <= -2**31 else int(q))
        return max(v, abs(l_query - l_ref))
    w = max(side(o_del, e_del), side(o_ins, e_ins))
    if w > cmd_w:
        w = min(w, region_w)
    return min(w, cmd_w * 4)


def _excl_cumsum(v: np.ndarray) -> np.ndarray:
    o = np.zeros(len(v), np.int64)
    if len(v) > 1:
        np.cumsum(v[:-1], out=o[1:])
    return o


@dataclass
class CigarBatch:
    results: np.ndarray        # CIGAR_RESULT_DT: OutScore fields and output lengths
    cigar: np.ndarray          # u32 words, job k's at cigar_off[k]
    ref_aligned: np.ndarray    # u8, job k's at ref_off[k]
    query_aligned: np.ndarray  # u8, job k's at qry_off[k]
    jobs: np.ndarray           # the batch's CIGAR_JOB_DT records: the offsets derive from them, so
                               # they stay as they were while the offsets are read
    first: np.ndarray | None = None   # the packed form's CIGAR offsets; slots of qlen + tlen + 2 without

    # per-job offsets, computed on first use (a caller reading only the results never pays)
    @property
    def cigar_off(self) -> np.ndarray:
        if self.first is None:
            self.first = _excl_cumsum(self.jobs["qlen"].astype(np.int64) + self.jobs["tlen"] + 2)
        return self.first

    @property
    def ref_off(self) -> np.ndarray:
        if getattr(self, "_ref_off", None) is None:
            self._ref_off = _excl_cumsum(self.jobs["tlen"])
        return self._ref_off

    @property
    def qry_off(self) -> np.ndarray:
        if getattr(self, "_qry_off", None) is None:
            self._qry_off = _excl_cumsum(self.jobs["qlen"])
        return self._qry_off

    def cigar_of(self, k: int) -> list[tuple[str, int]]:
        n = int(self.results["n_cigar"][k])
        words = self.cigar[int(self.cigar_off[k]):int(self.cigar_off[k]) + n]
        return [(CIGAR_OPS[int(x) & 15], int(x) >> 4) for x in words]

    def ref_aligned_of(self, k: int) -> np.ndarray:
        return self.ref_aligned[int(self.ref_off[k]):int(self.ref_off[k]) + int(self.results["n_ref"][k])]

    def query_aligned_of(self, k: int) -> np.ndarray:
        return self.query_aligned[int(self.qry_off[k]):int(self.qry_off[k]) + int(self.results["n_query"][k])]


def scalar_banded_swa_batch(params: np.ndarray, jobs: np.ndarray, qseq: np.ndarray, tseq: np.ndarray,
                            ctx: N.Context | None = None, packed: bool = True,
                            bufs: HostBuffers | None = None) -> CigarBatch:
    """scalar_banded_swa for every job (CIGAR_JOB_DT: offsets, lengths, band, h0).  packed:
    the CIGAR words come back back to back (fa_cigar_batch_packed), otherwise in slots of
    qlen + tlen + 2 words per job (fa_cigar_batch).  With `bufs` the outputs land in those
    reusable (page-locked) buffers and the batch views them."""
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, CIGAR_JOB_DT)
    qseq = np.ascontiguousarray(qseq, np.uint8)
    tseq = np.ascontiguousarray(tseq, np.uint8)
    n = len(jobs)
    t_sum = int(jobs["tlen"].sum(dtype=np.int64))
    q_sum = int(jobs["qlen"].sum(dtype=np.int64))
    cig_total = q_sum + t_sum + 2 * n
    res = out_array(bufs, "res", n, CIGAR_RESULT_DT, zero=True)
    ra = out_array(bufs, "ref_al", max(t_sum, 1), np.uint8)
    qa = out_array(bufs, "qry_al", max(q_sum, 1), np.uint8)
    if packed:
        # capacity for every slot, of which only the used words' pages are ever touched
        cig = out_array(bufs, "cigar", max(cig_total, 1), np.uint32)
        first = out_array(bufs, "first", max(n, 1), np.uint64, zero=True)
        if n:
            N.check(lib.fa_cigar_batch_packed(ctx.handle, N.ptr(params), N.ptr(jobs), n, N.ptr(qseq), len(qseq),
                                              N.ptr(tseq), len(tseq), N.ptr(res), N.ptr(cig), len(cig),
                                              N.ptr(first), N.ptr(ra), N.ptr(qa)))
        total = int(res["n_cigar"].sum()) if n else 0
        return CigarBatch(res, cig[:total], ra, qa, jobs, first[:n])
    cig = np.zeros(max(cig_total, 1), np.uint32)
    if n:
        N.check(lib.fa_cigar_batch(ctx.handle, N.ptr(params), N.ptr(jobs), n, N.ptr(qseq), len(qseq), N.ptr(tseq),
                                   len(tseq), N.ptr(res), N.ptr(cig), N.ptr(ra), N.ptr(qa)))
    return CigarBatch(res, cig, ra, qa, jobs)
