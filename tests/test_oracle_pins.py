"""The oracle against the reference's own recorded numbers (CPU only).

Before the oracle judges the GPU it is pinned here to what the reference
recorded about itself: tools/sphere-baseline.json (area identity, resting
ocean, Merian periods), the README's lake-at-rest table and the positivity
factor printed by tools/verify-physics.mjs.  The tolerances are the
reference's own (tools/verify-sphere.mjs:1133-1146): areas at 1e-15,
round-off residuals within a factor of 4, dry-cell counts exact, Merian
errors within 0.005 percentage points.  Bed functions that use exp/sin/cos
differ from V8's in the last bit, so noise-level numbers are compared in
band; the sharp-step lake, which has no transcendental in x, is compared to
the printed digits.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle_sim import OracleSim, oracle_hllc
import scenarios as S

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
BASE = PINS["sphere_baseline"]


def test_constants_match_reference_baseline():
    c = BASE["constants"]
    assert c["G_REF"] == S.G_REF and c["R_REF"] == S.R_REF and c["OMEGA_REF"] == S.OMEGA_REF


def test_positivity_theta_one_wet_cell():
    """tools/verify-physics.mjs:552-582: the solver returns 0.66666666666666674."""
    nx, dx, h0, MULT, ic = 9, 2, 0.5, 5, 4
    sim = OracleSim(nx=nx, ny=1, dx=dx, bed=lambda x, y: 0, eta0=0, manning=0)
    kc = sim.idx(ic, 0)
    sim.h[kc] = h0
    dt = MULT * sim.maxDt()
    sim.applyBC()
    sim.residual(dt)
    assert sim.theta[kc] == float(PINS["positivity_theta_one_wet_cell"])
    end = lambda i: sim.h[sim.idx(i, 0)] + dt * sim.rh[sim.idx(i, 0)]
    assert end(ic) == 0.0
    assert end(ic - 1) + end(ic + 1) == h0
    untouched = sum(1 for i in range(nx) if i != ic and sim.theta[sim.idx(i, 0)] == 1)
    assert untouched == nx - 1


@pytest.mark.parametrize("name", list(S.LAKE_BEDS))
def test_lake_at_rest_readme_table(name):
    """README.md:50-56: four beds, 200x4, 400 self-timed steps."""
    want = PINS["lake_at_rest_200x4_400steps"][name]
    sim = S.lake(OracleSim, name)
    sim.set_boundaries(west="reflect", east="reflect", south="periodic", north="periodic")
    v0 = sim.volume()
    for _ in range(400):
        sim.step()
    dev, spd = sim.maxSurfaceDeviation(2.0), sim.maxSpeed()
    assert dev <= 4 * 4.440892098500626e-16          # <= 4 ulp of eta = 2
    assert abs(sim.volume() - v0) / v0 < 1e-13
    if name == "sharp step":
        assert dev == 0.0 and f"{spd:.4e}" == f"{want['max_speed']:.4e}"
    else:
        assert spd < 1e-12 and 0.25 <= spd / want["max_speed"] <= 4
    if name in ("smooth bump", "random rough"):
        assert f"{dev:.4e}" == f"{want['max_eta_dev']:.4e}"


def test_closed_basin_mass():
    """tools/verify.mjs:150-176 (README: 8.3047e-15 relative over 600 steps)."""
    sim = OracleSim(nx=120, ny=80, dx=4, bed=lambda x, y: -8 + 3 * math.sin(x * 0.02) * math.cos(y * 0.03),
                    eta0=lambda x, y: 1.5 if x < 240 else 0.0, manning=0.02)
    v0 = sim.volume()
    for _ in range(600):
        sim.step()
    drift = abs(sim.volume() - v0) / v0
    assert drift < 1e-12
    assert drift < 10 * PINS["closed_basin_mass_drift_600_steps"]
    assert sim.finite()


@pytest.mark.parametrize("row", BASE["areaIdentity"], ids=lambda r: f"{r['deg']}deg_{r['lat0']}_{r['lat1']}")
def test_area_identity_baseline(row):
    """tools/verify-sphere.mjs:1181-1185: interiorArea at 1e-15, residual at round-off."""
    deg = row["deg"]
    sim = OracleSim(nx=round(360 / deg), ny=round((row["lat1"] - row["lat0"]) / deg), bed=lambda a, b: -1,
                    eta0=0, sphere={"R": S.R_REF, "lat0": row["lat0"], "lat1": row["lat1"]})
    area = sim.geom.area
    s = 0.0
    for j in range(2, sim.H - 2):
        s += area[j] * sim.nx
    assert abs(s - row["area"]) <= 1e-15 * abs(row["area"])
    p0, p1 = row["lat0"] * math.pi / 180, row["lat1"] * math.pi / 180
    exact = 2 * math.pi * S.R_REF * S.R_REF * (math.sin(p1) - math.sin(p0))
    assert abs((s - exact) / exact) < 1e-13


@pytest.mark.parametrize("row", BASE["restingOcean"],
                         ids=lambda r: f"{r['case']}_{r['deg']}deg_o{r['order']}_{r['lat0']}")
def test_resting_ocean_baseline(row):
    """tools/verify-sphere.mjs:479-500 and :1161-1172."""
    sim = S.sphere(OracleSim, S.SPHERE_BEDS[row["case"]], row["deg"], order=row["order"],
                   lat0=row["lat0"], lat1=row["lat1"])
    dry = S.dry_cells(sim)
    dt = sim.maxDt()
    for _ in range(row["steps"]):
        sim.step(dt)
    sp, et = sim.maxSpeed(), sim.maxSurfaceDeviation(0)
    assert dry == row["dry"]
    for got, want in ((sp, row["maxSpeed"]), (et, row["maxEta"])):
        if got == 0 or want == 0:
            assert got == want
        else:
            assert 0.25 <= got / want <= 4


MERIAN_FAST = [r for r in BASE["merian"] if r["deg"] in (6, 4)]


@pytest.mark.parametrize("row", MERIAN_FAST, ids=lambda r: f"n{r['n']}_{r['deg']}deg")
def test_merian_baseline(row):
    """tools/verify-sphere.mjs:673-720 and :1186-1189 (0.005 pp)."""
    r = S.merian(OracleSim, row["n"], row["deg"])
    assert abs(r["errPct"] - row["errPct"]) <= 0.005


def test_threaded_oracle_is_bit_identical():
    """The OpenMP variant (gathered accumulation) equals the reference loops."""
    kw = dict(nx=70, ny=45, dx=5, bed=lambda x, y: 0.3 * math.sin(x / 40) * math.cos(y / 30),
              eta0=lambda x, y: 1.0 if x < 150 else 0.2, manning=0.03, coriolis=1e-4)
    a, b = OracleSim(**kw), OracleSim(threads=8, **kw)
    for _ in range(25):
        dt = a.maxDt()
        assert dt == b.maxDt()
        a.step(dt)
        b.step(dt)
    for f in ("h", "hu", "hv", "rh", "rhu", "rhv", "theta"):
        assert np.array_equal(a.field(f), b.field(f)), f


def test_hllc_branches():
    """Both dry, dry-left/right speeds (Toro) and the wet contact branch."""
    assert list(oracle_hllc(0, 0, 0, 0, 0, 0, 1e-3)) == [0, 0, 0]
    h0 = 0.5
    c = math.sqrt(S.G_REF * h0)
    f = oracle_hllc(h0, 0, 0, 0, 0, 0, 1e-3)        # wet left, dry right: F = 2 c h0 / 3
    assert abs(f[0] - 2 * c * h0 / 3) < 1e-15
    g = oracle_hllc(0, 0, 0, h0, 0, 0, 1e-3)
    assert abs(g[0] + 2 * c * h0 / 3) < 1e-15
