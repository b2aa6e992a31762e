"""Build the oracle (test infrastructure): oracle/liboracle_swe.so.

g++ -O2 -ffp-contract=off, no fast-math, OpenMP for the multi-threaded CPU
baseline.  The output is git-ignored and travels with the tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_swe.so")
SRC = os.path.join(HERE, "swe_oracle.cpp")
HDR = os.path.join(HERE, "swe_oracle.h")

FLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-std=c++17",
         "-fPIC", "-shared"]


def build_oracle(force=False, verbose=False):
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC), os.path.getmtime(HDR))):
        return LIB
    cmd = ["g++"] + FLAGS + ["-o", LIB, SRC]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=HERE)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv, verbose=True))
