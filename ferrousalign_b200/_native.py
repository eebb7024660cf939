"""ctypes binding of libferrous_b200.so (the C ABI in include/ferrous_b200.h).

The library is the only compute path: if it is missing or cannot create a CUDA
context the calls raise, they never fall back to host code.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libferrous_b200.so"

FA_OK, FA_ERR_ARG, FA_ERR_CAPACITY, FA_ERR_CUDA, FA_ERR_TIMEOUT, FA_ERR_STATE = range(6)
FA_POLICY_SINGLE, FA_POLICY_BWA, FA_POLICY_LEARNED = 0, 1, 2
FA_JUDGE_CERT, FA_JUDGE_MAXOFF, FA_JUDGE_GLOBAL, FA_JUDGE_BOUND, FA_JUDGE_ONCE, FA_JUDGE_HINT = 1, 2, 4, 8, 16, 32
FA_DIR_LEFT, FA_DIR_RIGHT = 0, 1
FA_KERNEL_AUTO, FA_KERNEL_INT32, FA_KERNEL_INT16X2, FA_KERNEL_ROWS2 = 0, 1, 2, 3
KSW_XBYTE, KSW_XSTOP, KSW_XSUBO, KSW_XSTART = 0x10000, 0x20000, 0x40000, 0x80000
FA_MAX_QLEN, FA_MAX_TLEN = 4096, 65535
FA_NOALLOC_MAX_JOBS = 1 << 18
FA_PARAM_H0_ZERO = 1
FA_BAND_NPARAMS = 3201

PARAMS_DT = np.dtype([("mat", "i1", 25), ("flags", "u1"), ("_pad", "i1", 2), ("m", "<i4"), ("o_del", "<i4"),
                      ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4"), ("zdrop", "<i4"),
                      ("end_bonus", "<i4"), ("pen_clip5", "<i4"), ("pen_clip3", "<i4")])
JOB_DT = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"),
                   ("h0", "<i4"), ("w", "<i4"), ("dir", "<i4"), ("_pad", "<i4")])
EXT_RESULT_DT = np.dtype([("score", "<i4"), ("qle", "<i4"), ("tle", "<i4"), ("gtle", "<i4"),
                          ("gscore", "<i4"), ("max_off", "<i4")])
POLICY_DT = np.dtype([("mode", "<i4"), ("max_tries", "<i4"), ("judge", "<i4"), ("w_min", "<i4")])
STATS_DT = np.dtype([("cells", "<u8"), ("cells_executed", "<u8"), ("jobs", "<u4"), ("retries", "<u4"),
                     ("misses", "<u4"), ("kernel_launches", "<u4"), ("kernel_ms", "<f4"),
                     ("total_ms", "<f4")])
MATE_PARAMS_DT = np.dtype([("mat", "i1", 25), ("flags", "u1"), ("_pad", "i1", 2), ("m", "<i4"), ("o_del", "<i4"),
                           ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4")])
MATE_JOB_DT = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"),
                        ("xtra", "<u4"), ("_pad", "<i4")])
KSWR_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4"), ("score2", "<i4"),
                    ("te2", "<i4"), ("tb", "<i4"), ("qb", "<i4")])
REGION_OPTS_DT = np.dtype([("a", "<i4"), ("pen_clip5", "<i4"), ("pen_clip3", "<i4"), ("w", "<i4")])
SEED_EXT_DT = np.dtype([("ref_pos", "<u8"), ("query_pos", "<i4"), ("len", "<i4"), ("left_job", "<i4"),
                        ("right_job", "<i4")])
REGION_DT = np.dtype([("rb", "<u8"), ("re", "<u8"), ("qb", "<i4"), ("qe", "<i4"), ("score", "<i4"),
                      ("truesc", "<i4"), ("seedcov", "<i4"), ("seedlen0", "<i4"), ("w", "<i4"), ("seed", "<i4")])
COLLECT_OPTS_DT = np.dtype([("a", "<i4"), ("o_del", "<i4"), ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4"),
                            ("w", "<i4")])
CHAIN_DT = np.dtype([("read", "<u4"), ("seed_first", "<u4"), ("n_seeds", "<u4"), ("kept", "<i4")])
SEED_DT = np.dtype([("ref_pos", "<u8"), ("query_pos", "<i4"), ("len", "<i4")])
COLLECT_COUNTS_DT = np.dtype([("n_left", "<u4"), ("n_right", "<u4"), ("n_seed_ext", "<u4"), ("_pad", "<u4"),
                              ("qbuf_len", "<u8"), ("tbuf_len", "<u8")])
CIGAR_JOB_DT = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"), ("w", "<i4"),
                         ("h0", "<i4")])
CIGAR_RESULT_DT = np.dtype([("score", "<i4"), ("qle", "<i4"), ("tle", "<i4"), ("gtle", "<i4"), ("gscore", "<i4"),
                            ("max_off", "<i4"), ("n_cigar", "<i4"), ("n_ref", "<i4"), ("n_query", "<i4"),
                            ("cells", "<i4")])
INSERT_BOUNDS_DT = np.dtype([("low", "<i4"), ("high", "<i4"), ("failed", "<i4"), ("_pad", "<i4")])
INSERT_STATS_DT = np.dtype([("avg", "<f8"), ("std", "<f8"), ("low", "<i4"), ("high", "<i4"), ("failed", "<i4"),
                            ("_pad", "<i4")])
RESCUE_ALN_DT = np.dtype([("pos", "<i8"), ("ref_id", "<i4"), ("is_rev", "<i4"), ("ref_len", "<i4"), ("score", "<i4")])
RESCUE_CAND_DT = np.dtype([("read", "<u4"), ("aln_first", "<u4"), ("aln_count", "<u4"), ("primary", "<u4"),
                           ("anchor", RESCUE_ALN_DT)])
RESCUE_OPTS_DT = np.dtype([("pen_unpaired", "<i4"), ("max_matesw", "<i4"), ("min_seed_len", "<i4"),
                           ("match_score", "<i4")])
RESCUE_JOB_INFO_DT = np.dtype([("cand", "<u4"), ("orientation", "<i4"), ("is_rev", "<i4"), ("rid", "<i4"),
                               ("adj_rb", "<i8"), ("adj_re", "<i8")])

NRUN_DT = np.dtype([("pos", "<u8"), ("len", "<u8")])
PACKED_SEQ_DT = np.dtype([("bases", "<u8"), ("n_bases", "<u8"), ("n_runs", "<u8"), ("n_nruns", "<u8")])

assert NRUN_DT.itemsize == 16 and PACKED_SEQ_DT.itemsize == 32
assert PARAMS_DT.itemsize == 64 and JOB_DT.itemsize == 40 and EXT_RESULT_DT.itemsize == 24
assert STATS_DT.itemsize == 40 and MATE_PARAMS_DT.itemsize == 48 and MATE_JOB_DT.itemsize == 32
assert KSWR_DT.itemsize == 28
assert REGION_OPTS_DT.itemsize == 16 and SEED_EXT_DT.itemsize == 24 and REGION_DT.itemsize == 48
assert COLLECT_OPTS_DT.itemsize == 24 and CHAIN_DT.itemsize == 16 and SEED_DT.itemsize == 16
assert COLLECT_COUNTS_DT.itemsize == 32
assert CIGAR_JOB_DT.itemsize == 32 and CIGAR_RESULT_DT.itemsize == 40
assert INSERT_BOUNDS_DT.itemsize == 16 and RESCUE_ALN_DT.itemsize == 24 and RESCUE_CAND_DT.itemsize == 40
assert RESCUE_OPTS_DT.itemsize == 16 and RESCUE_JOB_INFO_DT.itemsize == 32
assert INSERT_STATS_DT.itemsize == 32

# Every symbol the header declares, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "fa_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "fa_ctx_destroy": (None, [_P]),
    "fa_last_error": (C.c_char_p, []),
    "fa_version": (C.c_char_p, []),
    "fa_mate_xtra": (C.c_uint32, [C.c_int32, C.c_int32, C.c_int32]),
    "fa_device_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fa_probe_int_peak": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "fa_ext_batch": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P]),
    "fa_ext_batch_policy": (C.c_int, [_P, _P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64,
                                      _P, _P, _P, _P]),
    "fa_ext_batch_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, _P, _P, _P]),
    "fa_ext_batch_packed": (C.c_int, [_P, _P, _P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P]),
    "fa_ext_batch_packed_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, _P, _P, _P]),
    "fa_ctx_sync": (C.c_int, [_P]),
    "fa_ctx_set_timing": (C.c_int, [_P, C.c_int]),
    "fa_ctx_set_kernel": (C.c_int, [_P, C.c_int]),
    "fa_ctx_set_graph": (C.c_int, [_P, C.c_int]),
    "fa_ctx_set_slices": (C.c_int, [_P, C.c_int, C.c_int]),
    "fa_ctx_set_reference": (C.c_int, [_P, _P, C.c_uint64]),
    "fa_ctx_set_threads": (C.c_int, [_P, C.c_int]),
    "fa_ctx_kernel_choice": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, _P, _P, _P,
                                       C.POINTER(C.c_int)]),
    "fa_ctx_last_timing": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "fa_ext_batch_device_noalloc": (C.c_int, [_P, _P, C.c_uint32, _P, _P, _P, _P]),
    "fa_mate_sw_batch_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, _P, _P]),
    "fa_ctx_last_cells": (C.c_int, [_P, C.POINTER(C.c_ulonglong)]),
    "fa_band_model_create": (C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
    "fa_band_model_destroy": (None, [_P]),
    "fa_band_model_get": (C.c_int, [_P, _P, _P, _P]),
    "fa_band_model_set": (C.c_int, [_P, _P, _P, _P]),
    "fa_band_model_save": (C.c_int, [_P, C.c_char_p]),
    "fa_band_model_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "fa_band_model_fit_norm": (C.c_int, [_P, _P, C.c_uint32]),
    "fa_band_features": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P]),
    "fa_band_predict": (C.c_int, [_P, _P, _P, _P, C.c_uint32, C.c_float, C.c_int, _P, _P]),
    "fa_band_grad": (C.c_int, [_P, _P, _P, _P, C.c_uint32, C.c_float, _P, _P]),
    "fa_band_train": (C.c_int, [_P, _P, _P, _P, C.c_uint32, C.c_int, C.c_uint32, C.c_float, C.c_float, C.c_uint64, _P]),
    "fa_ext_batch_learned": (C.c_int, [_P, _P, _P, _P, C.c_float, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64,
                                       _P, _P, _P, _P, _P]),
    "fa_ext_batch_learned_packed": (C.c_int, [_P, _P, _P, _P, C.c_float, _P, C.c_uint32, _P, _P, _P, _P, _P, _P,
                                              _P]),
    "fa_mate_sw_batch": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P]),
    "fa_mate_sw_batch_packed": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, _P, _P]),
    "fa_pair_batch": (C.c_int, [_P, _P, _P, _P, C.c_float, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P,
                                _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P, _P]),
    "fa_collect_ext_jobs": (C.c_int, [_P, _P, _P, C.c_uint64, _P, _P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32,
                                      _P, _P, _P, _P, C.c_uint64, _P, _P, _P, _P]),
    "fa_collect_ext_jobs_packed": (C.c_int, [_P, _P, _P, C.c_uint64, _P, _P, C.c_uint32, _P, C.c_uint32, _P,
                                             C.c_uint32, _P, _P, _P, _P, C.c_uint64, _P, C.c_uint64, _P,
                                             C.c_uint64, _P, _P, _P, _P, _P]),
    "fa_cigar_batch": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P, _P, _P]),
    "fa_cigar_batch_packed": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64, _P, _P, C.c_uint64,
                                        _P, _P, _P]),
    "fa_collect_mate_jobs": (C.c_int, [_P, _P, _P, _P, C.c_uint64, _P, _P, C.c_uint32, _P, _P, C.c_uint32, _P,
                                       C.c_uint32, _P, C.c_uint32, _P, _P, _P, C.c_uint64, _P, C.c_uint64, _P]),
    "fa_insert_size_stats": (C.c_int, [_P, C.c_uint64, _P, C.c_uint32, _P]),
    "fa_merge_regions": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32,
                                   _P]),
    "fa_merge_regions_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, C.c_uint32, _P,
                                          C.c_uint32, _P, _P]),
}


class NativeError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def load(path: Path | None = None) -> C.CDLL:
    """Loads the shared library (raising if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            p = Path(path) if path else LIB_PATH
            if not p.exists():
                raise RuntimeError(f"{p} is missing: run ferrousalign_b200.build.build_all() first")
            lib = C.CDLL(str(p))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def check(rc: int) -> None:
    if rc != FA_OK:
        msg = load().fa_last_error()
        raise NativeError(rc, msg.decode() if msg else "")


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return a.ctypes.data


class Context:
    """One CUDA context handle of the library (one per host thread)."""

    def __init__(self, device: int = 0):
        lib = load()
        h = C.c_void_p()
        check(lib.fa_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise RuntimeError("context closed")
        return self._h

    def set_kernel(self, kernel: int) -> None:
        check(load().fa_ctx_set_kernel(self.handle, kernel))

    def set_threads(self, threads_per_block: int) -> None:
        check(load().fa_ctx_set_threads(self.handle, threads_per_block))

    def kernel_choice(self) -> dict:
        """Kernel and threads per block of the last call, and the last autotuning table."""
        k, t, nc = C.c_int(), C.c_int(), C.c_int()
        ck = (C.c_int * 8)()
        ct = (C.c_int * 8)()
        cm = (C.c_float * 8)()
        check(load().fa_ctx_kernel_choice(self.handle, C.byref(k), C.byref(t), 8, ck, ct, cm, C.byref(nc)))
        names = {FA_KERNEL_INT32: "int32", FA_KERNEL_INT16X2: "int16x2", FA_KERNEL_ROWS2: "rows2"}
        # the tiling each kernel kind stands for: jobs per thread and target rows per step
        shape = {FA_KERNEL_INT32: (1, 1), FA_KERNEL_INT16X2: (2, 1), FA_KERNEL_ROWS2: (1, 2)}

        def entry(kind: int, tpb: int) -> dict:
            jobs, rows = shape.get(kind, (1, 1))
            return {"kernel": names.get(kind, str(kind)), "threads_per_block": tpb, "jobs_per_thread": jobs,
                    "rows_per_thread": rows, "jobs_per_warp": 32 * jobs}
        out = entry(k.value, t.value)
        out["candidates"] = [dict(entry(ck[i], ct[i]), sample_ms=float(cm[i])) for i in range(min(nc.value, 8))]
        return out

    def set_slices(self, single_band: int = 0, policy_rounds: int = 0) -> None:
        """Upload slices of large host batches (2..8; 1 uploads the whole batch before one run
        of the kernels; 0 keeps the current value, -1 restores the defaults: 8 for byte codes,
        3 for the rounds of a packed batch, 6 for a packed single-band batch)."""
        check(load().fa_ctx_set_slices(self.handle, single_band, policy_rounds))

    def set_reference(self, pac, l_pac: int = 0) -> None:
        """Keep the 2-bit packed reference (`pac`, l_pac bases) on the device: collection calls
        given pac=None then read it instead of uploading it again.  None drops it."""
        if pac is None:
            check(load().fa_ctx_set_reference(self.handle, None, 0))
            return
        pac = np.ascontiguousarray(pac, np.uint8)
        check(load().fa_ctx_set_reference(self.handle, pac.ctypes.data, int(l_pac)))

    def set_graph(self, enable: bool) -> None:
        """Run policy / learned batches as one recorded CUDA graph per batch shape."""
        check(load().fa_ctx_set_graph(self.handle, int(enable)))

    def close(self) -> None:
        if self._h is not None:
            load().fa_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: dict[int, Context] = {}
_tls = threading.local()


def default_context(device: int = 0) -> Context:
    """A lazily created context per (thread, device)."""
    d = getattr(_tls, "ctx", None)
    if d is None:
        d = _tls.ctx = {}
    if device not in d:
        d[device] = Context(device)
    return d[device]
