"""Build the library (sm_100a, FP64) in-tree with nvcc, in two arithmetic
modes from the same sources:

  libswe_b200.so      -fmad=false: no multiply-add is contracted, so the
                      device arithmetic rounds operation by operation like
                      the reference's JavaScript engine -- the comparison
                      build, bit-identical to the oracle; the default.
  libswe_b200_fma.so  -fmad=true: the compiler fuses multiply-adds (one
                      rounding instead of two); results agree with the
                      comparison build to round-off (held to 1e-12 per field
                      per step by the tests).  Chosen with SWE_B200_ARITH=fma.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANTS = {"exact": ("libswe_b200.so", "-fmad=false"), "fma": ("libswe_b200_fma.so", "-fmad=true")}
LIB = os.path.join(HERE, VARIANTS["exact"][0])
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("swe_api.cu", "swe_batch.cu", "swe_adjoint.cu",
                                                    "swe_noalloc.cu", "swe_gridlands.cu", "swe_render.cu")]
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
    os.path.join(HERE, "..", "include", "swe_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def lib_path(variant="exact"):
    return os.path.join(HERE, VARIANTS[variant][0])


def up_to_date(path):
    if not os.path.exists(path):
        return False
    t = os.path.getmtime(path)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build_library(force=False, verbose=False, extra=(), variant="exact"):
    """Compile one arithmetic mode of the C-ABI library; returns its path."""
    path = lib_path(variant)
    if not force and up_to_date(path):
        return path
    cmd = [nvcc()] + NVCC_FLAGS + [VARIANTS[variant][1]] + list(extra) + ["-o", path] + SOURCES
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=HERE)
    return path


def build_all(force=False, verbose=False):
    return [build_library(force, verbose, variant=v) for v in VARIANTS]


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv, verbose=True))
