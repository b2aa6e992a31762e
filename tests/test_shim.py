"""The Node drop-in's host side (water-simulator_b200/node/swe_shim.h, the
class the N-API addon wraps) driven through the reference suites' call
sequences by tests/shim_sequence.cpp, next to the oracle.

The addon's N-API glue itself needs node_api.h, which is absent here; the
shim underneath it is plain C++ over the C ABI and is compiled here (CPU)
and run on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "tests", "_build")


def build_sequence():
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "shim_sequence")
    lib_dir = os.path.join(ROOT, "water-simulator_b200")
    orc_dir = os.path.join(ROOT, "oracle")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wno-unused-function", os.path.join(ROOT, "tests", "shim_sequence.cpp"),
           "-I" + os.path.join(ROOT, "include"), "-L" + lib_dir, "-lswe_b200", "-L" + orc_dir, "-loracle_swe",
           "-Wl,-rpath," + lib_dir, "-Wl,-rpath," + orc_dir, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_shim_and_sequence_compile_and_link():
    for lib in (os.path.join(ROOT, "water-simulator_b200", "libswe_b200.so"),
                os.path.join(ROOT, "oracle", "liboracle_swe.so")):
        if not os.path.exists(lib):
            pytest.skip(f"{lib} is not built")
    assert os.path.exists(build_sequence())


@pytest.mark.gpu
def test_shim_call_sequences_on_the_gpu():
    exe = build_sequence()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout
