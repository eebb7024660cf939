"""ctypes binding of the CPU oracle (oracle/libksw_oracle.so).

Test infrastructure only: the parity checker for the CUDA kernels and the timed CPU
baseline.  See ksw_oracle.c for the reference lines each function restates.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libksw_oracle.so"

TRACE_DT = np.dtype([("cells", "<i8"), ("rows", "<i4"), ("clamped", "<i4"), ("label", "<i4"),
                     ("w_eff", "<i4"), ("bound_ok", "<i4"), ("init_reach", "<i4"), ("hint", "<i4"), ("_pad", "<i4")])
EXT_RESULT_DT = np.dtype([("score", "<i4"), ("qle", "<i4"), ("tle", "<i4"), ("gtle", "<i4"),
                          ("gscore", "<i4"), ("max_off", "<i4")])
KSWR_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4"), ("score2", "<i4"),
                    ("te2", "<i4"), ("tb", "<i4"), ("qb", "<i4")])

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build_oracle
            build_oracle.build()
        lib = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        lib.ora_ksw_extend2.restype = C.c_int
        lib.ora_ksw_extend2.argtypes = [C.c_int, P, C.c_int, P, C.c_int, P] + [C.c_int] * 8 + [P, P]
        lib.ora_ksw_extend2_flags.restype = C.c_int
        lib.ora_ksw_extend2_flags.argtypes = [C.c_int, P, C.c_int, P, C.c_int, P] + [C.c_int] * 8 + [C.c_uint, P, P]
        lib.ora_ksw_align2.restype = C.c_int
        lib.ora_ksw_align2.argtypes = [C.c_int, P, C.c_int, P, C.c_int, P] + [C.c_int] * 4 + [C.c_uint32, P, P]
        lib.ora_ext_batch.restype = C.c_int
        lib.ora_ext_batch.argtypes = [P, P, C.c_uint32, P, P, P, P, C.c_int]
        lib.ora_ext_batch_policy.restype = C.c_int
        lib.ora_ext_batch_policy.argtypes = [P, P, P, C.c_uint32, P, P, P, P, P, P, P, C.c_int]
        lib.ora_wide_clean.restype = C.c_int
        lib.ora_wide_clean.argtypes = [P, C.c_int, C.c_int, C.c_int]
        lib.ora_mate_batch.restype = C.c_int
        lib.ora_mate_batch.argtypes = [P, P, C.c_uint32, P, P, P, P, C.c_int]
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _codes(x):
    if isinstance(x, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(x), dtype=np.uint8)
    return np.ascontiguousarray(x, dtype=np.uint8)


def ksw_extend2(query, target, mat, o_del, e_del, o_ins, e_ins, w, end_bonus, zdrop, h0, flags: int = 0):
    """flags: fa_params.flags (1 = FA_PARAM_H0_ZERO: h0 == 0 runs as written)."""
    q, t = _codes(query), _codes(target)
    m = np.ascontiguousarray(mat, dtype=np.int8)
    out = np.zeros(1, EXT_RESULT_DT)
    tr = np.zeros(1, TRACE_DT)
    rc = load().ora_ksw_extend2_flags(len(q), _p(q), len(t), _p(t), 5, _p(m), o_del, e_del, o_ins, e_ins, w,
                                      end_bonus, zdrop, h0, flags, _p(out), _p(tr))
    if rc:
        raise ValueError(f"oracle ksw_extend2 rejected the input ({rc})")
    return out[0], tr[0]


def wide_clean(params, qlen: int, w: int, init_reach: int) -> bool:
    """Whether band w's first row covers every positive first-row cell."""
    return bool(load().ora_wide_clean(_p(params), qlen, w, init_reach))


def ksw_align2(query, target, mat, o_del, e_del, o_ins, e_ins, xtra):
    q, t = _codes(query), _codes(target)
    m = np.ascontiguousarray(mat, dtype=np.int8)
    out = np.zeros(1, KSWR_DT)
    cells = np.zeros(1, np.int64)
    rc = load().ora_ksw_align2(len(q), _p(q), len(t), _p(t), 5, _p(m), o_del, e_del, o_ins, e_ins, xtra,
                               _p(out), _p(cells))
    if rc:
        raise ValueError(f"oracle ksw_align2 rejected the input ({rc})")
    return out[0]


def ext_batch(params, jobs, qseq, tseq, threads: int = 0):
    n = len(jobs)
    out = np.zeros(n, EXT_RESULT_DT)
    tr = np.zeros(n, TRACE_DT)
    rc = load().ora_ext_batch(_p(params), _p(jobs), n, _p(qseq), _p(tseq), _p(out), _p(tr), threads)
    if rc:
        raise ValueError(f"oracle ext_batch failed ({rc})")
    return out, tr


def ext_batch_policy(params, policy, jobs, qseq, tseq, w_first=None, threads: int = 0):
    n = len(jobs)
    out = np.zeros(n, EXT_RESULT_DT)
    wfin = np.zeros(n, np.int32)
    tries = np.zeros(n, np.int32)
    cells = np.zeros(n, np.int64)
    wf = None if w_first is None else np.ascontiguousarray(w_first, dtype=np.int32)
    rc = load().ora_ext_batch_policy(_p(params), _p(policy), _p(jobs), n, _p(qseq), _p(tseq), _p(wf), _p(out),
                                     _p(wfin), _p(tries), _p(cells), threads)
    if rc:
        raise ValueError(f"oracle ext_batch_policy failed ({rc})")
    return out, wfin, tries, cells


def mate_batch(params, jobs, qseq, tseq, threads: int = 0):
    n = len(jobs)
    out = np.zeros(n, KSWR_DT)
    cells = np.zeros(n, np.int64)
    rc = load().ora_mate_batch(_p(params), _p(jobs), n, _p(qseq), _p(tseq), _p(out), _p(cells), threads)
    if rc:
        raise ValueError(f"oracle mate_batch failed ({rc})")
    return out, cells
