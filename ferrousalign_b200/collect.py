"""Extension jobs from chains: the host mirror of collect_extension_jobs_batch_soa
(src/pipelines/linear/batch_extension/collect_soa.rs:28-230).

For each kept chain with seeds, the reference window its seeds can reach, read on the GPU
out of the 2-bit packed reference, and per seed (last to first) a left and a right
extension job, ready for `extend_batch` (queries in `qbuf`, targets in `tbuf`), plus the
seed table `merge_scores_to_regions` reads (csrc/collect_kernel.cu).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .hostbuf import HostBuffers, capacity, out_array

CHAIN_DT = N.CHAIN_DT
SEED_DT = N.SEED_DT


def collect_opts(a: int = 1, o_del: int = 6, e_del: int = 1, o_ins: int = 6, e_ins: int = 1,
                 w: int = 100) -> np.ndarray:
    """MemOpt's fields the collection reads (mem_opt.rs defaults)."""
    o = np.zeros(1, N.COLLECT_OPTS_DT)
    o["a"], o["o_del"], o["e_del"], o["o_ins"], o["e_ins"], o["w"] = a, o_del, e_del, o_ins, e_ins, w
    return o


def pack_reference(codes: np.ndarray) -> tuple[np.ndarray, int]:
    """The .pac layout of a forward reference: two bits per base, base k in bits 7-6 of byte
    k/4 when k % 4 == 0 down to bits 1-0 when k % 4 == 3 (bntseq.rs:564-575).  N (code 4)
    has no 2-bit code; like bwa's indexer, which stores a random base for it, this stores
    code & 3."""
    c = np.asarray(codes, np.uint8) & 3
    n = len(c)
    pad = np.zeros((n + 3) // 4 * 4, np.uint8)
    pad[:n] = c
    q = pad.reshape(-1, 4)
    pac = (q[:, 0] << 6) | (q[:, 1] << 4) | (q[:, 2] << 2) | q[:, 3]
    return pac.astype(np.uint8), n


# Reusable output buffers of the collection calls (hostbuf.HostBuffers).
CollectBuffers = HostBuffers
_out = out_array


@dataclass
class CollectedJobs:
    left_jobs: np.ndarray      # JOB_DT, the reference's left batch order
    right_jobs: np.ndarray     # JOB_DT, the reference's right batch order
    qbuf: np.ndarray           # u8: every read forward then reversed, at twice its offset
    tbuf: np.ndarray           # u8: every chain window forward then reversed
    seed_ext: np.ndarray       # SEED_EXT_DT, chains' seeds last to first, global job indices
    chain_first: np.ndarray    # u32[n_chains + 1]
    chain_win: np.ndarray      # u64[n_chains, 2]: [rmax0, rmax1), (0, 0) without jobs


def collect_extension_jobs(pac: np.ndarray, l_pac: int, reads: np.ndarray, read_off: np.ndarray,
                           chains: np.ndarray, seeds: np.ndarray, opts: np.ndarray | None = None,
                           ctx: N.Context | None = None, bufs: HostBuffers | None = None) -> CollectedJobs:
    """fa_collect_ext_jobs.  pac=None reads the reference the context keeps
    (Context.set_reference).  With `bufs` the outputs land in those reusable (page-locked)
    buffers and the result views them; without, in fresh arrays."""
    lib = N.load()
    ctx = ctx or N.default_context()
    opts = collect_opts() if opts is None else opts
    pac = None if pac is None else np.ascontiguousarray(pac, np.uint8)   # None: the context's resident reference
    reads = np.ascontiguousarray(reads, np.uint8)
    read_off = np.ascontiguousarray(read_off, np.uint64)
    chains = np.ascontiguousarray(chains, CHAIN_DT)
    seeds = np.ascontiguousarray(seeds, SEED_DT)
    n_reads, n_chains, n_seeds = len(read_off) - 1, len(chains), len(seeds)
    read_bytes = int(read_off[-1]) if n_reads >= 0 and len(read_off) else 0
    # outputs the library writes in full up to the returned counts: left uninitialised, so
    # only the pages the copies reach are ever touched
    left = _out(bufs, "left", n_seeds, N.JOB_DT)
    right = _out(bufs, "right", n_seeds, N.JOB_DT)
    qbuf = _out(bufs, "qbuf", max(2 * read_bytes, 1), np.uint8)
    ext = _out(bufs, "ext", n_seeds, N.SEED_EXT_DT)
    first = _out(bufs, "first", n_chains + 1, np.uint32)
    win = _out(bufs, "win", 2 * n_chains, np.uint64).reshape(n_chains, 2)
    counts = np.zeros(1, N.COLLECT_COUNTS_DT)
    # target capacity: what reused buffers hold (the call reports the length it needs when
    # that is short), else every chain's widest window
    cap = capacity(bufs, "tbuf", np.uint8)
    if cap == 0 and n_chains:
        qlen = np.diff(read_off.astype(np.int64))
        cap = int(2 * (qlen[chains["read"]] + 4 * int(opts["w"][0]) + 64).sum())
    for _ in range(2):
        tbuf = _out(bufs, "tbuf", max(cap, 1), np.uint8)
        rc = lib.fa_collect_ext_jobs(ctx.handle, N.ptr(opts), N.ptr(pac), l_pac, N.ptr(reads), N.ptr(read_off),
                                     n_reads, N.ptr(chains), n_chains, N.ptr(seeds), n_seeds, N.ptr(left),
                                     N.ptr(right), N.ptr(qbuf), N.ptr(tbuf), cap, N.ptr(ext), N.ptr(first),
                                     N.ptr(win), N.ptr(counts))
        if rc == N.FA_ERR_CAPACITY and int(counts["tbuf_len"][0]) > cap:
            cap = int(counts["tbuf_len"][0])
            continue
        N.check(rc)
        break
    c = counts[0]
    return CollectedJobs(left[:c["n_left"]], right[:c["n_right"]], qbuf[:c["qbuf_len"]],
                         tbuf[:c["tbuf_len"]], ext[:c["n_seed_ext"]], first, win)


def collect_extension_jobs_packed(pac: np.ndarray, l_pac: int, reads: np.ndarray, read_off: np.ndarray,
                                  chains: np.ndarray, seeds: np.ndarray, opts: np.ndarray | None = None,
                                  ctx: N.Context | None = None, bufs: HostBuffers | None = None) -> CollectedJobs:
    """fa_collect_ext_jobs_packed: the same jobs and seed table, with `qbuf` and `tbuf` as
    2-bit packed buffers (PackedSeq, N runs listed), packed on the device -- ready for
    extend_batch_packed.  `bufs` as for collect_extension_jobs."""
    from .packed import PackedSeq
    lib = N.load()
    ctx = ctx or N.default_context()
    opts = collect_opts() if opts is None else opts
    pac = None if pac is None else np.ascontiguousarray(pac, np.uint8)   # None: the context's resident reference
    reads = np.ascontiguousarray(reads, np.uint8)
    read_off = np.ascontiguousarray(read_off, np.uint64)
    chains = np.ascontiguousarray(chains, CHAIN_DT)
    seeds = np.ascontiguousarray(seeds, SEED_DT)
    n_reads, n_chains, n_seeds = len(read_off) - 1, len(chains), len(seeds)
    read_bytes = int(read_off[-1]) if len(read_off) else 0
    left = _out(bufs, "left", n_seeds, N.JOB_DT)
    right = _out(bufs, "right", n_seeds, N.JOB_DT)
    qb = _out(bufs, "qbuf", (2 * read_bytes + 3) // 4 + 4, np.uint8, zero=True)   # 4 bytes of slack, as pack() leaves
    ext = _out(bufs, "ext", n_seeds, N.SEED_EXT_DT)
    first = _out(bufs, "first", n_chains + 1, np.uint32)
    win = _out(bufs, "win", 2 * n_chains, np.uint64).reshape(n_chains, 2)
    counts = np.zeros(1, N.COLLECT_COUNTS_DT)
    n_runs = np.zeros(2, np.uint64)
    # capacities: what reused buffers hold (the call reports what it needs when that is
    # short), else every chain's widest window and a run per 64 / 256 bases
    cap = 4 * max(capacity(bufs, "tbuf", np.uint8) - 4, 0)
    if cap == 0 and n_chains:
        qlen = np.diff(read_off.astype(np.int64))
        cap = int(2 * (qlen[chains["read"]] + 4 * int(opts["w"][0]) + 64).sum())
    qcap = max(1024, 2 * read_bytes // 64, capacity(bufs, "qruns", N.NRUN_DT))
    tcap = max(1024, cap // 256, capacity(bufs, "truns", N.NRUN_DT))
    for _ in range(3):
        tb = _out(bufs, "tbuf", (cap + 3) // 4 + 4, np.uint8, zero=True)
        qr = _out(bufs, "qruns", qcap, N.NRUN_DT)
        tr = _out(bufs, "truns", tcap, N.NRUN_DT)
        rc = lib.fa_collect_ext_jobs_packed(ctx.handle, N.ptr(opts), N.ptr(pac), l_pac, N.ptr(reads),
                                            N.ptr(read_off), n_reads, N.ptr(chains), n_chains, N.ptr(seeds),
                                            n_seeds, N.ptr(left), N.ptr(right), N.ptr(qb), N.ptr(qr), qcap,
                                            N.ptr(tb), len(tb) - 4, N.ptr(tr), tcap, N.ptr(ext), N.ptr(first),
                                            N.ptr(win), N.ptr(counts), N.ptr(n_runs))
        if rc == N.FA_ERR_CAPACITY:
            cap = max(cap, int(counts["tbuf_len"][0]))
            qcap, tcap = max(qcap, int(n_runs[0])), max(tcap, int(n_runs[1]))
            continue
        N.check(rc)
        break
    c = counts[0]
    qs = PackedSeq(qb[:(int(c["qbuf_len"]) + 3) // 4 + 4], int(c["qbuf_len"]), qr[:int(n_runs[0])].copy())
    ts = PackedSeq(tb[:(int(c["tbuf_len"]) + 3) // 4 + 4], int(c["tbuf_len"]), tr[:int(n_runs[1])].copy())
    return CollectedJobs(left[:c["n_left"]], right[:c["n_right"]], qs, ts, ext[:c["n_seed_ext"]], first, win)
