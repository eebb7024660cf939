"""Builds tests/kernel_host/libpair_host.so: the extension kernels' thread bodies
compiled for the host (nvcc, no GPU needed)."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "pair_host.cu"
LIB = HERE / "libpair_host.so"
DEPS = [SRC, HERE.parent.parent / "ferrousalign_b200" / "csrc" / "extend_pair_kernel.cu",
        HERE.parent.parent / "ferrousalign_b200" / "csrc" / "fa_kernels.h",
        HERE.parent.parent / "ferrousalign_b200" / "csrc" / "fa_device.cuh"]


def build() -> Path:
    if LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in DEPS):
        return LIB
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp), str(SRC)], check=True)
    tmp.replace(LIB)
    return LIB
