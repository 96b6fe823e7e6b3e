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
           "cf_raster.cu", "cf_linesearch.cu", "cf_tsdf.cu", "cf_voxelknn.cu"]
HEADERS = ["cf_device.cuh", "cf_internal.h", os.path.join("..", "..", "include", "cudafusion_b200.h")]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden",
]
OBJ_DIR = os.path.join(HERE, "_build")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(CSRC, h) for h in HEADERS]


def _stale():
    return _newer(LIB, [os.path.join(CSRC, f) for f in SOURCES] + _headers())


def build(force=False, verbose=False, extra_flags=(), lib_path=LIB, obj_dir=OBJ_DIR):
    """Compiles each source to an object (in parallel, only the stale ones)
    and links the shared library."""
    from concurrent.futures import ThreadPoolExecutor

    if not force and lib_path == LIB and not extra_flags and not _stale():
        return lib_path
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(obj_dir, exist_ok=True)
    jobs = []
    for f in SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(obj_dir, f[:-3] + ".o")
        if force or extra_flags or _newer(obj, [src] + _headers()):
            jobs.append([nvcc] + NVCC_FLAGS + list(extra_flags) + ["-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    objs = [os.path.join(obj_dir, f[:-3] + ".o") for f in SOURCES]
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", lib_path] + objs
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    return lib_path


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
