"""Build recipe for the CPU oracle (test checker and timed CPU baseline only).

Produces oracle/libksw_oracle.so from oracle/ksw_oracle.c and oracle/libsimd_baseline.so
(the reference's SIMD CPU path restated, timed as the CPU baseline) from
oracle/simd_baseline.cpp.  The reference itself is
Rust and cannot be compiled in this image (no cargo/rustc, no vendored crates), so
there is no oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "ksw_oracle.c"
LIB = HERE / "libksw_oracle.so"
DEPS = [SRC, HERE / "ksw_oracle.h", HERE.parent / "include" / "ferrous_b200.h"]

# x86-64-v3 (AVX2) runs on every current B200 host CPU; -ffp-contract=off keeps the
# band-clamp arithmetic in separately rounded double operations.
CFLAGS = ["-O3", "-std=c11", "-fPIC", "-shared", "-pthread", "-ffp-contract=off"]


SIMD_SRC = HERE / "simd_baseline.cpp"
SIMD_LIB = HERE / "libsimd_baseline.so"


def build_simd(force: bool = False, verbose: bool = False) -> Path:
    """The reference's SIMD CPU path restated (simd_baseline.cpp), compiled once for AVX2
    (no AVX-512 instructions allowed) and once for AVX-512BW, linked into one library; the
    caller picks the width at run time (simd_baseline.py checks the CPU)."""
    deps = [SIMD_SRC, HERE.parent / "include" / "ferrous_b200.h"]
    if not force and SIMD_LIB.exists() and all(d.stat().st_mtime <= SIMD_LIB.stat().st_mtime for d in deps):
        return SIMD_LIB
    if os.uname().machine != "x86_64":
        raise RuntimeError("the SIMD baseline restates x86 AVX2 / AVX-512BW kernels")
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        objs = []
        for isa, flags in ((1, ["-mavx2", "-mno-avx512f"]), (2, ["-mavx2", "-mavx512f", "-mavx512bw"])):
            obj = str(Path(td) / f"simd{isa}.o")
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", f"-DFA_ISA={isa}", *flags, "-c", str(SIMD_SRC), "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            objs.append(obj)
        tmp = SIMD_LIB.with_suffix(".so.tmp")
        subprocess.run(["g++", "-shared", "-pthread", "-o", str(tmp), *objs], check=True)
        os.replace(tmp, SIMD_LIB)
    return SIMD_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    if os.uname().machine == "x86_64":
        build_simd(force, verbose)
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in DEPS):
        return LIB
    arch = ["-march=x86-64-v3"] if os.uname().machine == "x86_64" else []
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", *CFLAGS, *arch, "-o", str(tmp), str(SRC), "-lm"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
