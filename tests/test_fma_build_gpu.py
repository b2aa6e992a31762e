"""The FMA build (compiled with -fmad=true, SWE_B200_ARITH=fma) held to the
specification's tolerance against the oracle: 1e-12 relative per field per
step, and the lake at rest within 4 ulp of eta.  The exact build
(-fmad=false, the default) is the comparison build, bit-identical to the
oracle; every other GPU test checks it.  The FMA build runs in a child
process (tests/fma_check.py), since a process loads one build."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_fma_build_within_tolerance():
    lib = os.path.join(os.path.dirname(HERE), "water-simulator_b200", "libswe_b200_fma.so")
    assert os.path.exists(lib), "libswe_b200_fma.so is not built (water-simulator_b200/build.py)"
    env = dict(os.environ, SWE_B200_ARITH="fma")
    r = subprocess.run([sys.executable, os.path.join(HERE, "fma_check.py")], env=env, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    print(res)
    assert res["library"] == "libswe_b200_fma.so"
    for case in ("dam_break_256", "beach_512x256", "sphere_land_tide"):
        assert res[case] <= 1e-12, (case, res[case])
    for name, v in res["lake_at_rest"].items():
        assert v["eta_ulp"] <= 4, (name, v)
        assert v["max_speed"] < 1e-12, (name, v)
