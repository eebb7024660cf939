"""Builds the in-tree shared libraries of the package.

libferrous_b200.so  -- the CUDA kernels and the C ABI (include/ferrous_b200.h), sm_100a only
libfa_synth.so      -- seeded synthetic workload generators (host code)

Both land next to this file so they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libferrous_b200.so"
SYNTH = PKG / "libfa_synth.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-Xptxas", "-O3",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    cu = sorted(CSRC.glob("*.cu"))
    deps = cu + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "ferrous_b200.h"]
    if force or _stale(LIB, deps):
        objdir = PKG / "_build"
        objdir.mkdir(exist_ok=True)
        objs = [str(objdir / (src.stem + ".o")) for src in cu]
        # one nvcc per translation unit, run side by side
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=min(len(cu), os.cpu_count() or 1)) as ex:
            for f in [ex.submit(_run, [_nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", o], verbose)
                      for src, o in zip(cu, objs)]:
                f.result()
        tmp = LIB.with_suffix(".so.tmp")
        _run([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp), *objs,
              "-lcudart"], verbose)
        os.replace(tmp, LIB)
    return LIB


def build_synth(force: bool = False, verbose: bool = False) -> Path:
    src = CSRC / "synth.c"
    deps = [src, CSRC / "fa_synth.h", ROOT / "include" / "ferrous_b200.h"]
    if force or _stale(SYNTH, deps):
        tmp = SYNTH.with_suffix(".so.tmp")
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-pthread", "-o", str(tmp), str(src), "-lm"],
             verbose)
        os.replace(tmp, SYNTH)
    return SYNTH


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_synth(force, verbose)
    build_library(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
