"""ctypes binding of oracle/libsimd_baseline.so: the reference's SIMD CPU path restated.

Benchmark and test infrastructure only (the timed CPU baseline), never product code.
simd_baseline.cpp says which reference lines each kernel restates.  Outputs are the
reference SIMD kernels' OutScore fields (score, 0-based target end, 0-based query end) or
Kswr records, which by design differ from ksw_extend2's six fields.
"""
from __future__ import annotations

import ctypes as C
import functools
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsimd_baseline.so"
OUT3_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4")])
KSWR_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4"), ("score2", "<i4"),
                    ("te2", "<i4"), ("tb", "<i4"), ("qb", "<i4")])
ISAS = ("avx512", "avx2")


@functools.lru_cache(maxsize=None)
def load() -> C.CDLL:
    if not LIB_PATH.exists():
        from . import build_oracle
        build_oracle.build_simd()
    lib = C.CDLL(str(LIB_PATH))
    P, U, I = C.c_void_p, C.c_uint32, C.c_int
    for isa in ISAS:
        f = getattr(lib, f"simd_ext_batch_{isa}")
        f.restype, f.argtypes = I, [P, P, U, P, P, P, I, I]
        g = getattr(lib, f"simd_kswv_batch_{isa}")
        g.restype, g.argtypes = None, [P, U, P, P, P, I]
    lib.simd_ext_batch_port.restype = I
    lib.simd_ext_batch_port.argtypes = [P, P, U, P, P, P, I]
    lib.simd_i8_chunk_avx2.restype = I
    lib.simd_i8_chunk_avx2.argtypes = [P] * 6 + [I, I, I, P, P]
    return lib


def cpu_has(isa: str) -> bool:
    """Whether the host CPU runs the given build (flags from /proc/cpuinfo)."""
    try:
        flags = next(ln for ln in open("/proc/cpuinfo") if ln.startswith("flags")).split()
    except (OSError, StopIteration):
        return False
    need = {"avx2": ["avx2"], "avx512": ["avx512f", "avx512bw"]}[isa]
    return all(f in flags for f in need)


def best_isa() -> str:
    return next(i for i in ISAS if cpu_has(i))


def _p(a):
    return None if a is None else a.ctypes.data


def ext_batch(params, jobs, qseq, tseq, isa: str | None = None, threads: int = 0, force_i16: bool = False):
    """All jobs through the banded SIMD kernels (chunks of the vector width).  Returns the
    OutScore records and the kernel width used (8 = int8 lanes, 16 = int16 lanes)."""
    isa = isa or best_isa()
    n = len(jobs)
    out = np.zeros(n, OUT3_DT)
    lib = load()
    if isa == "port":
        bits = lib.simd_ext_batch_port(_p(params), _p(jobs), n, _p(qseq), _p(tseq), _p(out), threads)
    else:
        bits = getattr(lib, f"simd_ext_batch_{isa}")(_p(params), _p(jobs), n, _p(qseq), _p(tseq), _p(out), threads,
                                                     int(force_i16))
    return out, bits


def kswv_batch(jobs, qseq, tseq, isa: str | None = None, threads: int = 0):
    """Mate-rescue jobs through the u8 horizontal kernel (chunks of the vector width)."""
    isa = isa or best_isa()
    n = len(jobs)
    out = np.zeros(n, KSWR_DT)
    getattr(load(), f"simd_kswv_batch_{isa}")(_p(jobs), n, _p(qseq), _p(tseq), _p(out), threads)
    return out


def i8_chunk(q_soa, t_soa, qlen, tlen, h0, w, max_q, max_t, params):
    """One chunk of the int8 kernel on SoA inputs of stride len(qlen), as the reference's
    kernel tests call it; returns score, te, qe per lane."""
    lanes = len(qlen)
    a = [np.ascontiguousarray(x, np.int8) for x in (qlen, tlen, h0, w)]
    q = np.ascontiguousarray(q_soa, np.uint8)
    t = np.ascontiguousarray(t_soa, np.uint8)
    out = np.zeros(lanes, OUT3_DT)
    rc = load().simd_i8_chunk_avx2(_p(q), _p(t), *[_p(x) for x in a], lanes, max_q, max_t, _p(params), _p(out))
    if rc:
        raise ValueError("lanes exceed the AVX2 int8 width")
    return out


def threads_default() -> int:
    return os.cpu_count() or 1
