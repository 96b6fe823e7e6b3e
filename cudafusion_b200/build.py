"""Builds the sm_100a C-ABI library in place: cudafusion_b200/libcfb200.so.

    python -m cudafusion_b200.build
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcfb200.so")
SOURCES = ["cf_api.cu", "cf_kernels.cu", "cf_assemble.cu", "cf_pcg_grid.cu", "cf_pcg_cluster.cu", "cf_pcg_stream.cu",
           "cf_mpnn.cu", "cf_noalloc.cu", "cf_corr.cu",
           "cf_raster.cu", "cf_linesearch.cu", "cf_tsdf.cu"]
HEADERS = ["cf_device.cuh", "cf_internal.h", os.path.join("..", "..", "include", "cudafusion_b200.h")]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden",
    "-shared",
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
