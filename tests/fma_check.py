"""The FMA build (libswe_b200_fma.so) against the oracle, run in a process
of its own with SWE_B200_ARITH=fma (a process loads one build).  Prints one
JSON object; tests/test_fma_build_gpu.py asserts on it.

Per field per step, relative to the field's max-norm: before every compared
step the oracle gets the GPU's state, both take the same step.  Cases: the
256 x 256 dam break with Manning friction, a flooding beach over dry land,
a sphere with land, Coriolis and a device tide; and the lake at rest on the
four beds of tools/verify.mjs:124-136 (400 steps; |eta - 2| in ulp).
"""
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import __graft_entry__  # noqa: E402

swe = __graft_entry__.load_package()        # registers the package scenarios imports from

from oracle_sim import OracleSim  # noqa: E402
import scenarios as S  # noqa: E402
THREADS = os.cpu_count() or 1


def rel_err(a, b):
    scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / max(scale, 1e-300)


def stepwise(gpu, ref, steps):
    worst = 0.0
    for _ in range(steps):
        for n in ("h", "hu", "hv"):
            ref._arr(n)[:] = np.asarray(gpu.field(n)).reshape(-1)
        ref.t = gpu.t
        dt = ref.maxDt()
        gpu.step(dt)
        ref.step(dt)
        for n in ("h", "hu", "hv"):
            worst = max(worst, rel_err(gpu.field(n), ref.field(n)))
    return worst


def main():
    from water_simulator_b200 import workloads
    out = {"library": os.path.basename(swe.LIB_PATH)}
    b, eta = workloads.bump_dam_break(256, 256, 5.0)
    kw = dict(nx=256, ny=256, dx=5.0, bed=b, eta0=eta, manning=0.025)
    out["dam_break_256"] = stepwise(swe.ShallowWater(**kw), OracleSim(threads=THREADS, **kw), 60)
    bb, hh = workloads.beach_dam_break(512, 256, 8.0)
    kw = dict(nx=512, ny=256, dx=8.0, bed=bb, eta0=bb + hh, manning=0.03)
    gpu, ref = swe.ShallowWater(**kw), OracleSim(threads=THREADS, **kw)
    gpu.boundaries = {"west": swe.flather(lambda t: 0.0, lambda t: 0.0)}
    ref.set_boundaries(west=("flather", lambda t: 0.0, lambda t: 0.0))
    out["beach_512x256"] = stepwise(gpu, ref, 40)
    c = workloads.globe_tide(nx=180, ny=90, lat0=-80.0, lat1=80.0, modes=12)
    sph = {"R": 6371e3, "lat0": -80.0, "lat1": 80.0, "omega": 7.2921e-5}
    kw = dict(nx=180, ny=90, bed=c["b"], eta0=c["eta0"], sphere=sph)
    gpu, ref = swe.ShallowWater(**kw), OracleSim(threads=THREADS, **kw)
    tide = swe.Tide({"M2": [1.0, 0.0]}, periods_hours={"M2": 12.42})
    gpu.boundaries = {"south": swe.flather(tide.signal()), "north": swe.flather(tide.signal())}
    tr = tide.terms
    row = ("tide", tide.msl, [k["amp"] for k in tr], [k["omega"] for k in tr], [k["phase"] for k in tr], 0.0)
    ref.set_boundaries(west="periodic", east="periodic", south=row, north=row)
    out["sphere_land_tide"] = stepwise(gpu, ref, 30)
    ulp = 4.440892098500626e-16
    lake = {}
    for name in S.LAKE_BEDS:
        sim = S.lake(swe.ShallowWater, name)
        sim.boundaries = {"west": swe.reflect, "east": swe.reflect, "south": swe.periodic, "north": swe.periodic}
        for _ in range(400):
            sim.step()
        lake[name] = {"eta_ulp": sim.maxSurfaceDeviation(2.0) / ulp, "max_speed": sim.maxSpeed()}
        sim.close()
    out["lake_at_rest"] = lake
    print(json.dumps(out))


if __name__ == "__main__":
    main()
