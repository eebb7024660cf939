"""Builds the test harnesses that compile extension kernels' thread bodies for the host
(nvcc, no GPU needed): libpair_host.so (two jobs per thread), librows2_host.so (two
target rows per thread), liborder_host.so (the job-ordering bin mapping) and
libpacked_host.so (the packed-sequence reader)."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent.parent / "ferrousalign_b200" / "csrc"
COMMON = [CSRC / "fa_kernels.h", CSRC / "fa_device.cuh", CSRC / "fa_packed.cuh"]
HARNESSES = {
    "pair": (HERE / "pair_host.cu", [CSRC / "extend_pair_kernel.cu"]),
    "rows2": (HERE / "rows2_host.cu",
              [CSRC / "extend_kernel.cu", CSRC / "extend_pair_kernel.cu", CSRC / "extend_rows2_kernel.cu"]),
    "order": (HERE / "order_host.cu", [CSRC / "order_kernel.cu"]),
    "packed": (HERE / "packed_host.cu", []),
}


def build(name: str = "pair") -> Path:
    src, deps = HARNESSES[name]
    lib = HERE / f"lib{name}_host.so"
    if lib.exists() and all(d.stat().st_mtime <= lib.stat().st_mtime for d in [src, *deps, *COMMON]):
        return lib
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    tmp = lib.with_suffix(".so.tmp")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp), str(src)], check=True)
    tmp.replace(lib)
    return lib
