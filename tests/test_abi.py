"""The C ABI library: it loads, exports what include/swe_b200.h declares, its
host-side metric set-up equals the oracle's, and the Python mirror's host
logic (argument checks, reference errors) -- all without a GPU."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from oracle_sim import OracleSim

HEADER = os.path.join(ROOT, "include", "swe_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(swe_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(swe):
    lib = swe.load_library()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    from water_simulator_b200 import _lib
    assert set(names) == set(_lib.SIGNATURES), "ctypes table and header disagree"


def test_options_defaults(swe):
    from water_simulator_b200 import _lib
    o = _lib.SweOptions()
    assert swe.load_library().swe_options_init(ctypes.byref(o)) == 0
    assert (o.manning, o.min_depth, o.cfl, o.coriolis, o.order, o.limiter) == (0.025, 1e-3, 0.45, 0, 2, 0)
    assert (o.R, o.lat0, o.lat1, o.omega) == (6371e3, -90, 90, 0)


@pytest.mark.parametrize("cfg", [
    dict(nx=90, ny=60, sphere={"R": 6371000.0, "lat0": -60, "lat1": 60, "omega": 7.292115e-5}),
    dict(nx=180, ny=90, sphere={"R": 6371000.0, "lat0": -90, "lat1": 90}),
    dict(nx=36, ny=12, sphere={"R": 1000.0, "lat0": 10, "lat1": 70, "omega": 1e-4}),
    dict(nx=20, ny=7, dx=3.0, dy=5.0, coriolis=1e-4),
])
def test_metric_setup_matches_oracle(swe, cfg):
    """cartesianGeometry / sphericalGeometry (src/geometry.mjs) bit for bit."""
    if "sphere" in cfg:
        sp = cfg["sphere"]
        g = swe.sphericalGeometry(nx=cfg["nx"], ny=cfg["ny"], R=sp["R"], lat0=sp["lat0"], lat1=sp["lat1"],
                                  omega=sp.get("omega", 0))
        ref = OracleSim(nx=cfg["nx"], ny=cfg["ny"], bed=-1.0, sphere=sp)
    else:
        g = swe.cartesianGeometry(nx=cfg["nx"], ny=cfg["ny"], dx=cfg["dx"], dy=cfg["dy"],
                                  coriolis=cfg["coriolis"])
        ref = OracleSim(nx=cfg["nx"], ny=cfg["ny"], dx=cfg["dx"], dy=cfg["dy"], coriolis=cfg["coriolis"])
    for row in ["dxRow", "dyRowN", "dyRowS", "dyCFL", "area", "lx", "lyN", "lyS", "bedPhi", "phiC",
                "tanPhi", "fRow", "geoCoef"]:
        assert np.array_equal(getattr(g, row), getattr(ref.geom, row)), row
    assert g.totalArea == ref.geom.totalArea


def test_pole_face_is_exactly_closed(swe):
    """tools/verify-sphere.mjs: lyS === 0 at the south pole, lyN === 0 at the north."""
    g = swe.sphericalGeometry(nx=90, ny=45)
    assert g.lyS[2] == 0.0 and g.lyN[g.H - 3] == 0.0


def test_reference_errors(swe):
    with pytest.raises(ValueError, match="lat1"):
        swe.sphericalGeometry(nx=10, ny=5, lat0=10, lat1=5)
    with pytest.raises(ValueError, match=r"\[-90, 90\]"):
        swe.sphericalGeometry(nx=10, ny=5, lat0=-95, lat1=5)
    with pytest.raises(ValueError, match="even"):
        swe.sphericalGeometry(nx=11, ny=5)
    with pytest.raises(ValueError, match="unknown limiter"):
        swe.ShallowWater(nx=4, ny=4, dx=1, bed=lambda x, y: 0, limiter="superbee")


def test_interior_area_identity(swe):
    g = swe.sphericalGeometry(nx=180, ny=90, R=6371000.0)
    s = swe.interiorArea(g)
    assert abs(s - 4 * math.pi * 6371000.0 ** 2) / s < 1e-13


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU failure path")
def test_no_device_fails_loudly(swe):
    """No CPU fallback: without a CUDA device the constructor raises."""
    with pytest.raises(swe.SweError, match="no CUDA device"):
        swe.ShallowWater(nx=8, ny=8, dx=1, bed=lambda x, y: 0, eta0=1)


def test_row_access_refuses_bad_arguments_without_a_device(swe):
    """swe_get_rows / swe_set_rows (the row slabs' halo exchange) check
    their arguments before any device call."""
    lib = swe.load_library()
    from water_simulator_b200 import _lib
    buf = np.zeros(16)
    ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.swe_get_rows(None, _lib.FIELD["h"], 0, 1, ptr) == _lib.SWE_EINVAL
    assert lib.swe_set_rows(None, _lib.FIELD["h"], 0, 1, ptr) == _lib.SWE_EINVAL
    assert b"null" in lib.swe_last_error()
