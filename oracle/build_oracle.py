"""Build recipe for the CPU oracle (test checker and timed CPU baseline only).

Produces oracle/libksw_oracle.so from oracle/ksw_oracle.c.  The reference itself is
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


def build(force: bool = False, verbose: bool = False) -> Path:
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
