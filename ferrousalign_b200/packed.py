"""2-bit packed sequence buffers (fa_packed_seq) and the packed extension entry points.

A packed buffer stores four bases per byte -- base k in bits 2*(k % 4) .. 2*(k % 4) + 1 of
byte k / 4, codes A0 C1 G2 T3 -- and lists its N bases (code 4) as sorted runs, the form of
the reference's index (a 2-bit .pac beside its ambiguous stretches,
src/pipelines/linear/index/bntseq.rs:451-535).  Packing a byte-code buffer keeps every
position, so the jobs of a byte-code batch address the packed one unchanged (offsets and
lengths count bases either way).
"""
from __future__ import annotations

import numpy as np

from . import _native as N


class PackedSeq:
    """A packed host buffer: `bases` (uint8, (n + 3) // 4 bytes) and `runs` (NRUN_DT)."""

    def __init__(self, bases: np.ndarray, n_bases: int, runs: np.ndarray):
        self.bases = np.ascontiguousarray(bases, np.uint8)
        self.n_bases = int(n_bases)
        self.runs = np.ascontiguousarray(runs, N.NRUN_DT)
        if len(self.bases) < (self.n_bases + 3) // 4:
            raise ValueError("packed buffer shorter than its base count")

    @property
    def nbytes(self) -> int:
        """Bytes a transfer of this buffer moves (bases and N runs)."""
        return (self.n_bases + 3) // 4 + self.runs.nbytes

    def struct(self) -> np.ndarray:
        """The fa_packed_seq record (pointers into this object's arrays: keep it alive)."""
        s = np.zeros(1, N.PACKED_SEQ_DT)
        s["bases"] = self.bases.ctypes.data if len(self.bases) else 0
        s["n_bases"] = self.n_bases
        s["n_runs"] = self.runs.ctypes.data if len(self.runs) else 0
        s["n_nruns"] = len(self.runs)
        return s

    def pinned(self) -> "PackedSeq":
        """A copy in page-locked host memory (for overlapped uploads)."""
        import torch
        b = torch.from_numpy(self.bases).pin_memory().numpy()
        r = torch.from_numpy(self.runs.view(np.uint8)).pin_memory().numpy().view(N.NRUN_DT) if len(self.runs) \
            else self.runs
        return PackedSeq(b, self.n_bases, r)

    def unpack(self) -> np.ndarray:
        return unpack(self)


def n_runs_of(codes: np.ndarray) -> np.ndarray:
    """Sorted runs (pos, len) of the N (code 4) positions of a byte-code array."""
    isn = np.concatenate([[False], np.asarray(codes) == 4, [False]])
    d = np.diff(isn.astype(np.int8))
    starts = np.nonzero(d == 1)[0]
    ends = np.nonzero(d == -1)[0]
    runs = np.zeros(len(starts), N.NRUN_DT)
    runs["pos"] = starts
    runs["len"] = ends - starts
    return runs


def pack(codes: np.ndarray) -> PackedSeq:
    """Byte codes 0-4 to a packed buffer (N positions stored as 0 and listed as runs)."""
    c = np.ascontiguousarray(codes, np.uint8)
    if len(c) and int(c.max()) > 4:
        raise ValueError("codes must be 0-4")
    n = len(c)
    nb = (n + 3) // 4
    c4 = np.zeros(nb * 4 + 4, np.uint8)   # 4 bytes of slack past the last base word
    c4[:n] = np.where(c == 4, 0, c)
    c4 = c4[: nb * 4].reshape(-1, 4)
    bases = np.zeros(nb + 4, np.uint8)
    bases[:nb] = c4[:, 0] | (c4[:, 1] << 2) | (c4[:, 2] << 4) | (c4[:, 3] << 6)
    return PackedSeq(bases, n, n_runs_of(c))


def unpack(ps: PackedSeq) -> np.ndarray:
    b = ps.bases[: (ps.n_bases + 3) // 4]
    c = np.stack([b & 3, (b >> 2) & 3, (b >> 4) & 3, (b >> 6) & 3], axis=1).reshape(-1)[: ps.n_bases].copy()
    for r in ps.runs:
        c[int(r["pos"]):int(r["pos"]) + int(r["len"])] = 4
    return c


def extend_batch_packed(params: np.ndarray, jobs: np.ndarray, qseq: PackedSeq, tseq: PackedSeq,
                        policy: np.ndarray | None = None, w_first: np.ndarray | None = None,
                        ctx: N.Context | None = None, out: np.ndarray | None = None, bands: bool = True):
    """fa_ext_batch_packed.  Returns (results, stats, w_final); `out` may be a (pinned)
    result buffer to fill; bands=False asks for no final bands (None)."""
    lib = N.load()
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, N.JOB_DT)
    n = len(jobs)
    out = np.zeros(n, N.EXT_RESULT_DT) if out is None else out
    stats = np.zeros(1, N.STATS_DT)
    w_final = np.zeros(n, np.int32) if bands else None
    wf = None if w_first is None else np.ascontiguousarray(w_first, np.int32)
    qs, ts = qseq.struct(), tseq.struct()
    N.check(lib.fa_ext_batch_packed(ctx.handle, N.ptr(params), N.ptr(policy), N.ptr(jobs), n, N.ptr(qs), N.ptr(ts),
                                    N.ptr(wf), N.ptr(out), N.ptr(w_final), N.ptr(stats)))
    return out, stats[0], w_final


def extend_batch_learned_packed(params: np.ndarray, jobs: np.ndarray, qseq: PackedSeq, tseq: PackedSeq, model,
                                hints: np.ndarray | None = None, judge: int | None = None, margin: float = 0.0,
                                w_min: int = 2, max_tries: int = 2, ctx: N.Context | None = None,
                                out: np.ndarray | None = None, bands: bool = True):
    """fa_ext_batch_learned_packed.  Returns (results, stats, w_first, w_final); bands=False
    asks for neither band array (None, None)."""
    from .band_model import HINT_DT, JUDGE_LEARNED
    from .batch_extension import make_policy
    ctx = ctx or N.default_context()
    jobs = np.ascontiguousarray(jobs, N.JOB_DT)
    n = len(jobs)
    out = np.zeros(n, N.EXT_RESULT_DT) if out is None else out
    stats = np.zeros(1, N.STATS_DT)
    wf = np.zeros(n, np.int32) if bands else None
    wfin = np.zeros(n, np.int32) if bands else None
    pol = make_policy(N.FA_POLICY_LEARNED, max_tries, JUDGE_LEARNED if judge is None else judge, w_min)
    h = None if hints is None else np.ascontiguousarray(hints, HINT_DT)
    qs, ts = qseq.struct(), tseq.struct()
    N.check(N.load().fa_ext_batch_learned_packed(ctx.handle, N.ptr(params), N.ptr(pol), model.handle, margin,
                                                 jobs.ctypes.data, n, N.ptr(qs), N.ptr(ts), N.ptr(h),
                                                 out.ctypes.data, N.ptr(wf), N.ptr(wfin), stats.ctypes.data))
    return out, stats[0], wf, wfin
