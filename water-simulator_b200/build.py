"""Build libswe_b200.so (sm_100a, FP64) in-tree with nvcc.

The library is compiled with -fmad=false: no multiply-add is contracted, so
the device arithmetic rounds operation by operation like the reference's
JavaScript engine (the parity build of the step).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libswe_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("swe_api.cu", "swe_batch.cu", "swe_adjoint.cu",
                                                    "swe_noalloc.cu", "swe_gridlands.cu", "swe_render.cu")]
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
    os.path.join(HERE, "..", "include", "swe_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-fmad=false", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build_library(force=False, verbose=False, extra=()):
    """Compile the C-ABI library; returns its path."""
    if not force and up_to_date():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-o", LIB] + SOURCES
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=HERE)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
