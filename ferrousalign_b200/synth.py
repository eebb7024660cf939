"""Seeded synthetic workloads (ctypes binding of libfa_synth.so).

Named workloads:
  ext_plain        10,000 right extensions: 1 Mbp i.i.d. reference with 0.1% N, 151 bp reads,
                   1% substitutions, 0.1% indels (geometric, mean 2), seed 19-51 bp at the
                   read start, h0 = seed length, target = suffix length + w, w = 100.
  ext_1m           1,000,000 right extensions from the same generator, per-read indel rate
                   drawn from {0, 0.1%, 1%, 3%}.
  ext_uneven       2,000,000 mixed left+right extensions, reads 50-300 bp, seed position
                   uniform, 100 Mbp reference with 5% dinucleotide-repeat tracts.
  ext_train        the ext_1m generator with a 3% indel-rate mixture (band-model training).
  mate_rescue      500,000 2x151 bp pairs, insert ~ N(400, 50); the mate's window covers
                   mean +- 4 sd plus the read length (551 bp).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native as N

LIB_PATH = Path(__file__).resolve().parent / "libfa_synth.so"

EXT_INFO_DT = np.dtype([("seed_len", "<i4"), ("diag_spread", "<i4"), ("has_partner", "<i4"),
                        ("read_idx", "<i4"), ("indel_rate_ppm", "<i4"), ("_pad", "<i4")])


class ExtCfg(C.Structure):
    _fields_ = [("read_len_min", C.c_int32), ("read_len_max", C.c_int32),
                ("seed_len_min", C.c_int32), ("seed_len_max", C.c_int32),
                ("seed_at_start", C.c_int32), ("w", C.c_int32), ("match_score", C.c_int32),
                ("n_indel_rates", C.c_int32), ("indel_rates", C.c_double * 4),
                ("sub_rate", C.c_double), ("indel_mean", C.c_double)]


class MateCfg(C.Structure):
    _fields_ = [("read_len", C.c_int32), ("match_score", C.c_int32), ("min_seed_len", C.c_int32),
                ("_pad", C.c_int32), ("insert_mean", C.c_double), ("insert_sd", C.c_double),
                ("sub_rate", C.c_double), ("indel_rate", C.c_double)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: run ferrousalign_b200.build.build_all()")
        lib = C.CDLL(str(LIB_PATH))
        lib.fa_synth_reference.restype = C.c_int
        lib.fa_synth_reference.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_void_p]
        lib.fa_synth_ext_jobs.restype = C.c_int64
        lib.fa_synth_ext_jobs.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(ExtCfg), C.c_uint32,
                                          C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                          C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        lib.fa_synth_mate_jobs.restype = C.c_int64
        lib.fa_synth_mate_jobs.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(MateCfg), C.c_uint32,
                                           C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        _lib = lib
    return _lib


def reference(length: int, seed: int = 1, n_rate: float = 0.001, repeat_frac: float = 0.0) -> np.ndarray:
    out = np.empty(length, dtype=np.uint8)
    rc = _load().fa_synth_reference(seed, length, n_rate, repeat_frac, out.ctypes.data)
    if rc:
        raise RuntimeError(f"fa_synth_reference failed ({rc})")
    return out


@dataclass
class ExtBatch:
    jobs: np.ndarray     # JOB_DT
    qseq: np.ndarray     # uint8 codes
    tseq: np.ndarray
    info: np.ndarray     # EXT_INFO_DT


def ext_jobs(ref: np.ndarray, n: int, seed: int = 7, read_len=(151, 151), seed_len=(19, 51),
             seed_at_start=True, w=100, match_score=1, indel_rates=(0.001,), sub_rate=0.01,
             indel_mean=2.0, threads: int = 0) -> ExtBatch:
    cfg = ExtCfg()
    cfg.read_len_min, cfg.read_len_max = read_len
    cfg.seed_len_min, cfg.seed_len_max = seed_len
    cfg.seed_at_start = int(seed_at_start)
    cfg.w, cfg.match_score = w, match_score
    cfg.n_indel_rates = len(indel_rates)
    for i, r in enumerate(indel_rates):
        cfg.indel_rates[i] = r
    cfg.sub_rate, cfg.indel_mean = sub_rate, indel_mean
    jobs = np.zeros(n, dtype=N.JOB_DT)
    info = np.zeros(n, dtype=EXT_INFO_DT)
    qcap = n * read_len[1]
    tcap = n * (read_len[1] + w)
    q = np.empty(max(qcap, 1), dtype=np.uint8)
    t = np.empty(max(tcap, 1), dtype=np.uint8)
    qu, tu = C.c_uint64(), C.c_uint64()
    got = _load().fa_synth_ext_jobs(ref.ctypes.data, len(ref), seed, C.byref(cfg), n, threads, jobs.ctypes.data,
                                    info.ctypes.data, q.ctypes.data, qcap, t.ctypes.data, tcap, C.byref(qu),
                                    C.byref(tu))
    if got != n:
        raise RuntimeError(f"fa_synth_ext_jobs produced {got} of {n} jobs")
    return ExtBatch(jobs, q[:max(qu.value, 1)].copy(), t[:max(tu.value, 1)].copy(), info)


@dataclass
class MateBatch:
    jobs: np.ndarray     # MATE_JOB_DT
    qseq: np.ndarray
    tseq: np.ndarray


def mate_jobs(ref: np.ndarray, n: int, seed: int = 11, read_len=151, insert_mean=400.0, insert_sd=50.0,
              sub_rate=0.01, indel_rate=0.001, match_score=1, min_seed_len=19, threads: int = 0) -> MateBatch:
    cfg = MateCfg()
    cfg.read_len, cfg.match_score, cfg.min_seed_len = read_len, match_score, min_seed_len
    cfg.insert_mean, cfg.insert_sd, cfg.sub_rate, cfg.indel_rate = insert_mean, insert_sd, sub_rate, indel_rate
    tcap_one = int(8 * insert_sd) + read_len + 8
    jobs = np.zeros(n, dtype=N.MATE_JOB_DT)
    q = np.empty(max(n * read_len, 1), dtype=np.uint8)
    t = np.empty(max(n * tcap_one, 1), dtype=np.uint8)
    qu, tu = C.c_uint64(), C.c_uint64()
    got = _load().fa_synth_mate_jobs(ref.ctypes.data, len(ref), seed, C.byref(cfg), n, threads, jobs.ctypes.data,
                                     q.ctypes.data, q.nbytes, t.ctypes.data, t.nbytes, C.byref(qu), C.byref(tu))
    if got != n:
        raise RuntimeError(f"fa_synth_mate_jobs produced {got} of {n} jobs")
    return MateBatch(jobs, q[:max(qu.value, 1)].copy(), t[:max(tu.value, 1)].copy())


# ---- named workloads --------------------------------------------------------

def workload_ext_plain(n: int = 10_000, seed: int = 1) -> ExtBatch:
    ref = reference(1_000_000, seed=seed, n_rate=0.001)
    return ext_jobs(ref, n, seed=seed + 100, indel_rates=(0.001,))


def workload_ext_1m(n: int = 1_000_000, seed: int = 2, ref_len: int = 1_000_000) -> ExtBatch:
    ref = reference(ref_len, seed=seed, n_rate=0.001)
    return ext_jobs(ref, n, seed=seed + 100, indel_rates=(0.0, 0.001, 0.01, 0.03))


def workload_ext_uneven(n: int = 2_000_000, seed: int = 3, ref_len: int = 100_000_000) -> ExtBatch:
    ref = reference(ref_len, seed=seed, n_rate=0.001, repeat_frac=0.05)
    return ext_jobs(ref, n, seed=seed + 100, read_len=(50, 300), seed_at_start=False,
                    indel_rates=(0.001,))


def workload_ext_train(n: int = 5_000_000, seed: int = 4) -> ExtBatch:
    ref = reference(1_000_000, seed=seed, n_rate=0.001)
    return ext_jobs(ref, n, seed=seed + 100, indel_rates=(0.0, 0.001, 0.01, 0.03))


def workload_mate(n: int = 500_000, seed: int = 5, ref_len: int = 10_000_000) -> MateBatch:
    ref = reference(ref_len, seed=seed, n_rate=0.001)
    return mate_jobs(ref, n, seed=seed + 100)


def workload_regions(n_chains: int = 2_000_000, seed: int = 17):
    """Region-merge input shaped like an extension batch's consumer: chains of 1-8 seeds
    (19-51 bp, nearby reference positions per chain, so seeds cover one another), one left
    and one right result per seed with scores, ends and end-to-end scores around the clip
    threshold.  Returns (chain_first, query_len, seeds, left_results, right_results)."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(1, 9, n_chains)
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    ns = int(first[-1])
    seeds = np.zeros(ns, N.SEED_EXT_DT)
    ci = np.repeat(np.arange(n_chains, dtype=np.uint64), counts)
    seeds["ref_pos"] = np.uint64(1 << 20) + ci * np.uint64(4096) + rng.integers(0, 200, ns).astype(np.uint64)
    seeds["query_pos"] = rng.integers(0, 100, ns)
    seeds["len"] = rng.integers(19, 52, ns)
    seeds["left_job"] = np.arange(ns)
    seeds["right_job"] = np.arange(ns)
    res = []
    for _ in range(2):
        r = np.zeros(ns, N.EXT_RESULT_DT)
        r["score"] = rng.integers(20, 160, ns)
        r["qle"] = rng.integers(0, 100, ns)
        r["tle"] = rng.integers(0, 120, ns)
        r["gtle"] = rng.integers(0, 120, ns)
        r["gscore"] = r["score"] - rng.integers(-3, 30, ns)
        res.append(r)
    return first, np.full(n_chains, 151, np.int32), seeds, res[0], res[1]


def workload_chains(n_reads: int = 100_000, seed: int = 21, ref_len: int = 10_000_000, read_len: int = 151,
                    w: int = 100):
    """Chains of seeds for the job collection: reads sampled from either strand of a seeded
    reference (1% substitutions), 1-3 chains per read, each of 1-4 exact seeds of 19-40 bp
    along the read's true diagonal (occasionally shifted by a small indel-like offset), a
    tenth of the chains placed at a random position instead, and one chain in twenty marked
    as not kept.  Positions are in FM-index space: forward [0, l_pac), reverse strand
    [l_pac, 2 l_pac).  Returns (ref_codes, reads, read_off, chains, seeds)."""
    rng = np.random.default_rng(seed)
    ref = reference(ref_len, seed=seed, n_rate=0.0, repeat_frac=0.02)
    l_pac = len(ref)
    reads = np.empty(n_reads * read_len, np.uint8)
    read_off = np.arange(n_reads + 1, dtype=np.uint64) * read_len
    starts = rng.integers(0, l_pac - read_len, n_reads)
    strand = rng.random(n_reads) < 0.5
    for r in range(n_reads):
        s = ref[starts[r]:starts[r] + read_len] & 3
        if strand[r]:
            s = (3 - s)[::-1]
        reads[r * read_len:(r + 1) * read_len] = s
    sub = rng.random(len(reads)) < 0.01
    reads[sub] = (reads[sub] + rng.integers(1, 4, int(sub.sum()))) & 3
    # FM coordinate of read position 0: forward start, or the reverse-strand image
    origin = np.where(strand, 2 * l_pac - (starts + read_len), starts).astype(np.int64)
    n_ch = rng.integers(1, 4, n_reads)
    chain_read = np.repeat(np.arange(n_reads), n_ch)
    nc = len(chain_read)
    n_sd = rng.integers(1, 5, nc)
    chains = np.zeros(nc, N.CHAIN_DT)
    chains["read"] = chain_read
    chains["n_seeds"] = n_sd
    chains["seed_first"] = np.concatenate([[0], np.cumsum(n_sd)[:-1]])
    chains["kept"] = (rng.random(nc) >= 0.05).astype(np.int32)
    ns = int(n_sd.sum())
    seeds = np.zeros(ns, N.SEED_DT)
    ci = np.repeat(np.arange(nc), n_sd)
    ln = rng.integers(19, 41, ns)
    qp = rng.integers(0, read_len - ln + 1)
    base = origin[chain_read[ci]]
    rand_chain = rng.random(nc) < 0.1
    strand_c = strand[chain_read]
    rand_origin = np.where(strand_c, l_pac + rng.integers(0, l_pac - 2 * read_len, nc),
                           rng.integers(0, l_pac - 2 * read_len, nc))
    base = np.where(rand_chain[ci], rand_origin[ci], base)
    shift = np.where(rng.random(ns) < 0.1, rng.integers(-3, 4, ns), 0)
    rp = base + qp + shift
    lo = np.where(base >= l_pac, l_pac, 0)
    hi = np.where(base >= l_pac, 2 * l_pac, l_pac) - ln
    seeds["ref_pos"] = np.clip(rp, lo, hi).astype(np.uint64)
    seeds["query_pos"] = qp
    seeds["len"] = ln
    return ref, reads, read_off, chains, seeds


def workload_cigar(n: int = 200_000, seed: int = 31, ref_len: int = 10_000_000, read_len: int = 151):
    """CIGAR-regeneration jobs shaped like the regions of 151-bp reads: the whole read
    against the reference span it came from (1% substitutions, per-read indel rate drawn
    from {0, 0.1, 1, 3}%, so the span is the read length give or take the indels), h0 = 0,
    and a band of the length difference plus 5-30 (the range infer_band_width gives such
    regions).  Returns (jobs, qseq, tseq) with CIGAR_JOB_DT jobs."""
    rng = np.random.default_rng(seed)
    ref = reference(ref_len, seed=seed, n_rate=0.001)
    b = ext_jobs(ref, n, seed=seed + 100, read_len=(read_len, read_len), seed_len=(1, 1),
                 indel_rates=(0.0, 0.001, 0.01, 0.03), w=100)
    jobs = np.zeros(n, N.CIGAR_JOB_DT)
    jobs["q_off"], jobs["t_off"] = b.jobs["q_off"], b.jobs["t_off"]
    jobs["qlen"] = b.jobs["qlen"]
    jobs["tlen"] = np.minimum(b.jobs["tlen"], b.jobs["qlen"] + rng.integers(-3, 4, n))
    jobs["w"] = np.abs(jobs["qlen"] - jobs["tlen"]) + rng.integers(5, 31, n)
    return jobs, b.qseq, b.tseq


def workload_rescue(n_pairs: int = 100_000, seed: int = 41, ref_len: int = 20_000_000, n_chr: int = 6,
                    read_len: int = 151):
    """Mate-rescue attempts shaped like paired-end data: a reference cut into n_chr sequences,
    fragments of N(400, 50) bases, read 1 (the anchor) at one end of a fragment and read 2 at
    the other, either strand; read 2 carries 1-3 alignments of its own, half the time one of
    them at its true place (so that orientation is already paired) and the others anywhere.
    Returns (ref_codes, chr_off, chr_len, reads, read_off, alns, cands) with reads the
    rescued reads' codes."""
    rng = np.random.default_rng(seed)
    ref = reference(ref_len, seed=seed, n_rate=0.001)
    cuts = np.sort(rng.choice(np.arange(1, n_chr * 8) * (ref_len // (n_chr * 8)), n_chr - 1, replace=False))
    chr_off = np.concatenate([[0], cuts]).astype(np.uint64)
    chr_len = (np.concatenate([cuts, [ref_len]]) - chr_off.astype(np.int64)).astype(np.uint64)
    ins = np.clip(rng.normal(400, 50, n_pairs).astype(np.int64), read_len, 1000)
    rid = rng.integers(0, n_chr, n_pairs)
    span = chr_len[rid].astype(np.int64) - ins - 1
    p1 = chr_off[rid].astype(np.int64) + (rng.random(n_pairs) * span).astype(np.int64)
    flip = rng.random(n_pairs) < 0.5
    reads = np.empty(n_pairs * read_len, np.uint8)
    read_off = np.arange(n_pairs + 1, dtype=np.uint64) * read_len
    alns_l, cands = [], np.zeros(n_pairs, N.RESCUE_CAND_DT)
    for i in range(n_pairs):
        a_pos, m_pos = int(p1[i]), int(p1[i] + ins[i] - read_len)
        if flip[i]:
            a_pos, m_pos = m_pos, a_pos
        seg = ref[m_pos:m_pos + read_len] & 3
        # read 2 lies on the other strand from the anchor (FR pairs)
        mate_rev = not flip[i]
        reads[i * read_len:(i + 1) * read_len] = (3 - seg)[::-1] if mate_rev else seg
        off = int(chr_off[rid[i]])
        own = []
        if rng.random() < 0.5:
            own.append((m_pos - off, int(rid[i]), int(mate_rev), read_len, int(rng.integers(100, 152))))
        for _ in range(int(rng.integers(1 if not own else 0, 3))):
            r2 = int(rng.integers(0, n_chr))
            own.append((int(rng.integers(0, int(chr_len[r2]) - read_len)), r2, int(rng.integers(0, 2)), read_len,
                        int(rng.integers(20, 152))))
        first = len(alns_l)
        alns_l.extend(own)
        best = max(range(len(own)), key=lambda k: own[k][4])
        cands[i] = (i, first, len(own), first + best,
                    (a_pos - off, int(rid[i]), int(flip[i]), read_len, int(rng.integers(120, 152))))
    alns = np.array(alns_l, dtype=[("pos", "<i8"), ("ref_id", "<i4"), ("is_rev", "<i4"), ("ref_len", "<i4"),
                                   ("score", "<i4")]).astype(N.RESCUE_ALN_DT)
    return ref, chr_off, chr_len, reads, read_off, alns, cands
