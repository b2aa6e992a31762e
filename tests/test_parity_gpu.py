"""GPU parity: libswe_b200.so (through the Python mirror of the C ABI) against
the CPU oracle on identical inputs.

The library is built with -fmad=false, so every + - * / sqrt is the same IEEE
operation in the same order as the oracle: fields are compared BIT FOR BIT
(all N cells, ghosts included).  The exceptions are the two library
functions whose last bit differs between CUDA and glibc -- pow(h, 4/3) and
hypot in the Manning friction and in maxSpeed, and cos in a device-evaluated
tide -- where the comparison is per field, per step, relative to the field's
max-norm, at the tolerance the spec states: 1e-12.
"""
import math

import numpy as np
import pytest

from oracle_sim import OracleSim, oracle_hllc
import scenarios as S

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12          # per field per step, relative to the field's max-norm


@pytest.fixture(autouse=True)
def _stage_kernels(monkeypatch):
    """These cases run on the fused stage kernel; test_parity_split_gpu.py
    runs every one of them again on the tiled pair."""
    monkeypatch.setenv("SWE_B200_STAGE", "fused")


def pair(swe, **kw):
    return swe.ShallowWater(**kw), OracleSim(**kw)


def set_bc(swe, gpu, ref, **kinds):
    d = {}
    for side, k in kinds.items():
        if isinstance(k, tuple):
            d[side] = swe.flather(k[1], k[2])
        else:
            d[side] = getattr(swe, k)
    gpu.boundaries = d
    ref.set_boundaries(**kinds)


def assert_fields_equal(gpu, ref, names=("h", "hu", "hv"), what=""):
    for n in names:
        a, b = gpu.field(n), ref.field(n)
        if not np.array_equal(a, b, equal_nan=True):
            bad = np.flatnonzero(~((a == b) | (np.isnan(a) & np.isnan(b))))
            k = bad[0]
            raise AssertionError(f"{what} field {n}: {bad.size} cells differ; first k={k} "
                                 f"(i={k % gpu.W}, j={k // gpu.W}) gpu={a[k]!r} oracle={b[k]!r}")


def assert_fields_close(gpu, ref, names=("h", "hu", "hv"), tol=REL_TOL, what=""):
    for n in names:
        a, b = gpu.field(n), ref.field(n)
        scale = np.max(np.abs(b))
        err = np.max(np.abs(a - b))
        assert err <= tol * max(scale, 1e-300), f"{what} field {n}: max|d| {err:.3e} vs scale {scale:.3e}"


def dam_break(nx, ny, dx=5.0, seed=1, **kw):
    b = S.bump_bed(nx, ny, dx, seed=seed)
    W = nx + 4
    x = (np.arange(W) - 2 + 0.5) * dx
    eta = np.where(x < nx * dx / 2, 2.0, 0.5)[None, :].repeat(ny + 4, axis=0)
    return dict(nx=nx, ny=ny, dx=dx, bed=b, eta0=eta, **kw)


CASES = {
    "dam_break_64x48": (dam_break(64, 48, manning=0), dict(west="reflect", east="reflect", south="reflect", north="reflect")),
    "multi_strip_250x37": (dam_break(250, 37, manning=0), dict(west="reflect", east="outflow", south="periodic", north="periodic")),
    "periodic_coriolis": (dam_break(70, 66, manning=0, coriolis=1.2e-4), dict(west="periodic", east="periodic", south="periodic", north="periodic")),
    "minmod_order2": (dam_break(40, 33, manning=0, limiter="minmod"), dict(west="outflow", east="reflect", south="reflect", north="outflow")),
    "central": (dam_break(31, 29, manning=0, limiter="central"), dict(west="reflect", east="reflect", south="reflect", north="reflect")),
    "order1": (dam_break(45, 21, manning=0, order=1), dict(west="reflect", east="reflect", south="periodic", north="periodic")),
    "ritter_ny1": (dict(nx=160, ny=1, dx=2.5, bed=lambda x, y: 0, eta0=lambda x, y: 4.0 if x < 200 else 0.0, manning=0),
                   dict(west="reflect", east="outflow", south="periodic", north="periodic")),
    "column_nx1": (dict(nx=1, ny=50, dx=3.0, bed=lambda x, y: 0, eta0=lambda x, y: 2.0 if y < 60 else 1.0, manning=0),
                   dict(west="periodic", east="periodic", south="reflect", north="reflect")),
    "dry_beach": (dict(nx=96, ny=40, dx=4.0, bed=lambda x, y: -2 + x / 50 + 0.2 * math.sin(y / 13),
                       eta0=lambda x, y: 1.0 if x < 60 else 0.0, manning=0),
                  dict(west="reflect", east="reflect", south="reflect", north="reflect")),
}


@pytest.mark.parametrize("name", list(CASES))
def test_step_bit_identical(swe, name):
    kw, bcs = CASES[name]
    gpu, ref = pair(swe, **kw)
    set_bc(swe, gpu, ref, **bcs)
    for step in range(12):
        dt = ref.maxDt()
        assert gpu.maxDt() == dt, f"maxDt at step {step}"
        assert gpu.step(dt) == ref.step(dt)
        assert_fields_equal(gpu, ref, what=f"{name} step {step}")
    assert gpu.t == ref.t and gpu.steps == ref.steps
    assert gpu.massFloored == ref.massFloored
    gpu.close()


def test_self_timed_step_and_refusal(swe):
    kw, bcs = CASES["dam_break_64x48"]
    gpu, ref = pair(swe, **kw)
    for _ in range(5):
        assert gpu.step() == ref.step()
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        assert gpu.step(bad) == 0 and ref.step(bad) == 0
    assert_fields_equal(gpu, ref, names=("b", "h", "hu", "hv"))
    assert gpu.steps == 5


@pytest.mark.parametrize("case", ["flat", "uneven", "piercing"])
def test_sphere_step_bit_identical(swe, case):
    bed = S.SPHERE_BEDS[case]
    eta0 = lambda lon, lat: 2.0 * math.exp(-((lon - 20) ** 2 + (lat - 30) ** 2) / 300)
    gpu = S.sphere(swe.ShallowWater, bed, 6, eta0=eta0, omega=S.OMEGA_REF)
    ref = S.sphere(OracleSim, bed, 6, eta0=eta0, omega=S.OMEGA_REF)
    assert_fields_equal(gpu, ref, names=("b", "h"), what="initial")
    dt = ref.maxDt()
    assert gpu.maxDt() == dt
    for step in range(15):
        gpu.step(dt)
        ref.step(dt)
    assert_fields_equal(gpu, ref, what=f"sphere {case}")
    assert gpu.volume() == ref.volume()
    assert gpu.energy() == ref.energy()


def test_sphere_capped_order1(swe):
    eta0 = lambda lon, lat: math.exp(-((lon + 40) ** 2 + lat ** 2) / 200)
    kw = dict(nx=72, ny=30, bed=S.bed_uneven, eta0=eta0, manning=0, order=1,
              sphere={"R": S.R_REF, "lat0": -60, "lat1": 60, "omega": S.OMEGA_REF})
    gpu, ref = pair(swe, **kw)
    for _ in range(10):
        dt = ref.maxDt()
        assert gpu.maxDt() == dt
        gpu.step(dt)
        ref.step(dt)
    assert_fields_equal(gpu, ref)


def test_residual_and_theta(swe):
    """applyBC + residual(dt): rh, rhu, rhv, theta bit for bit, at a dt 5x
    the CFL step so the positivity limiter fires."""
    kw, bcs = CASES["dry_beach"]
    gpu, ref = pair(swe, **kw)
    set_bc(swe, gpu, ref, **bcs)
    for _ in range(3):
        dt = ref.maxDt()
        gpu.step(dt)
        ref.step(dt)
    for mult in (1.0, 5.0, 0.0, -1.0):
        dt = mult * ref.maxDt()
        gpu.applyBC()
        ref.applyBC()
        gpu.residual(dt)
        ref.residual(dt)
        assert_fields_equal(gpu, ref, names=("b", "h", "hu", "hv", "rh", "rhu", "rhv", "theta"),
                            what=f"residual x{mult}")



def test_residual_limiter_fires_bit_identical(swe):
    """tools/verify-physics.mjs:470-498: a 40-cell row split into opposing
    9 m/s jets, residual at 5x the CFL step, where the limiter clips."""
    nx, dx, h0, USPLIT = 40, 2, 0.5, 9
    gpu, ref = pair(swe, nx=nx, ny=1, dx=dx, bed=lambda x, y: 0, eta0=h0, manning=0)
    for sim in (gpu, ref):
        h, hu = sim.h, sim.hu
        for i in range(nx):
            k = sim.idx(i, 0)
            h[k] = h0
            hu[k] = h0 * (-USPLIT if i < nx / 2 else USPLIT)
    dt = 5 * ref.maxDt()
    assert gpu.maxDt() * 5 == dt
    gpu.applyBC()
    ref.applyBC()
    gpu.residual(dt)
    ref.residual(dt)
    assert_fields_equal(gpu, ref, names=("h", "hu", "hv", "rh", "rhu", "rhv", "theta"))
    th = ref.field("theta")
    assert np.any(th < 1)
    end = [gpu.h[gpu.idx(i, 0)] + dt * gpu.rh[gpu.idx(i, 0)] for i in range(nx)]
    assert min(end) >= -1e-15


def test_theta_one_wet_cell_gpu(swe):
    """tools/verify-physics.mjs:552-582 on the GPU: theta = 0.66666666666666674."""
    nx, dx, h0, ic = 9, 2, 0.5, 4
    sim = swe.ShallowWater(nx=nx, ny=1, dx=dx, bed=lambda x, y: 0, eta0=0, manning=0)
    kc = sim.idx(ic, 0)
    h = sim.h
    h[kc] = h0
    dt = 5 * sim.maxDt()
    sim.applyBC()
    sim.residual(dt)
    assert sim.theta[kc] == 0.66666666666666674
    end = lambda i: sim.h[sim.idx(i, 0)] + dt * sim.rh[sim.idx(i, 0)]
    assert end(ic) == 0.0 and end(ic - 1) + end(ic + 1) == h0


@pytest.mark.parametrize("name", list(S.LAKE_BEDS))
def test_lake_at_rest_gpu(swe, name):
    """Lake at rest within 4 ulp of eta, and bit-identical to the oracle."""
    gpu, ref = S.lake(swe.ShallowWater, name), S.lake(OracleSim, name)
    set_bc(swe, gpu, ref, west="reflect", east="reflect", south="periodic", north="periodic")
    v0 = gpu.volume()
    assert v0 == ref.volume()
    for _ in range(400):
        gpu.step()
        ref.step()
    assert gpu.maxSurfaceDeviation(2.0) <= 4 * 4.440892098500626e-16
    assert gpu.maxSpeed() < 1e-12
    assert abs(gpu.volume() - v0) / v0 < 1e-13
    assert_fields_equal(gpu, ref)


def test_friction_scalar_and_field_within_tolerance(swe):
    kw = dam_break(80, 50, manning=0.03)
    gpu, ref = pair(swe, **kw)
    n = 0.015 + 0.025 * S.uniform_noise(7, (gpu.H, gpu.W), 0, 1).reshape(-1)
    for step in range(20):
        if step == 10:
            gpu.setManningField(n)
            ref.setManningField(n)
        dt = ref.maxDt()
        assert abs(gpu.maxDt() - dt) <= 1e-13 * dt
        gpu.step(dt)
        ref.step(dt)
        assert_fields_close(gpu, ref, what=f"friction step {step}")


def test_manning_field_rejects_bad_values(swe):
    sim = swe.ShallowWater(nx=6, ny=5, dx=1, bed=lambda x, y: 0, eta0=1)
    with pytest.raises(ValueError, match="Manning n must be finite"):
        sim.setManningField(lambda x, y: -0.1 if x > 3 else 0.02)


def test_sponge_bit_identical(swe):
    kw = dam_break(90, 20, manning=0)
    gpu, ref = pair(swe, **kw)
    gpu.forcing = swe.makeSponge(gpu, side="east", width=20, strength=0.08, etaRef=1.0)
    ref.setSponge(side="east", width=20, strength=0.08, etaRef=1.0)
    for _ in range(15):
        dt = ref.maxDt()
        assert gpu.maxDt() == dt
        gpu.step(dt)
        ref.step(dt)
    assert_fields_equal(gpu, ref)


def test_flather_host_values_bit_identical(swe):
    kw = dict(nx=120, ny=6, dx=5.0, bed=lambda x, y: -10 + x / 100, eta0=0.0, manning=0)
    gpu, ref = pair(swe, **kw)
    eta_ext = lambda t: 0.4 * math.sin(2 * math.pi * t / 60)
    u_ext = lambda t: math.sqrt(S.G_REF / 10) * eta_ext(t)
    set_bc(swe, gpu, ref, west=("flather", eta_ext, u_ext), east=("flather", lambda t: 0.0, lambda t: 0.0),
           south="periodic", north="periodic")
    for _ in range(40):
        dt = ref.maxDt()
        gpu.step(dt)
        ref.step(dt)
    assert_fields_equal(gpu, ref)


def test_flather_device_tide_within_tolerance(swe):
    """A harmonic tide evaluated on the device (CUDA cos) against the oracle's
    table (glibc cos)."""
    tide = swe.Tide({"M2": [0.5, 20], "S2": [0.2, 40]}, msl=0.1)
    sig = tide.signal()
    kw = dict(nx=100, ny=8, dx=50.0, bed=lambda x, y: -5 + x / 2000, eta0=0.0, manning=0)
    gpu, ref = pair(swe, **kw)
    gpu.boundaries = {"west": swe.flather(sig, sig.scaled(math.sqrt(S.G_REF / 5))), "east": swe.reflect,
                      "south": swe.periodic, "north": swe.periodic}
    terms = tide.terms
    ref.set_boundaries(west=("tide", tide.msl, [k["amp"] for k in terms], [k["omega"] for k in terms],
                             [k["phase"] for k in terms], math.sqrt(S.G_REF / 5)),
                       east="reflect", south="periodic", north="periodic")
    gpu.t = 3000.0
    ref.t = 3000.0
    for _ in range(30):
        dt = ref.maxDt()
        gpu.step(dt)
        ref.step(dt)
        assert_fields_close(gpu, ref)
    done = gpu.run(20, dt=dt)
    for _ in range(done):
        ref.step(dt)
    assert done == 20
    assert_fields_close(gpu, ref)


def test_run_device_loop_matches_driver_loop(swe):
    """run(n, tEnd=T) == `while (t < T) sim.step(Math.min(sim.maxDt(), T - sim.t))`."""
    kw, bcs = CASES["multi_strip_250x37"]
    gpu, ref = pair(swe, **kw)
    set_bc(swe, gpu, ref, **bcs)
    T = 2.5
    done = gpu.run(1000, tEnd=T)
    n = 0
    while ref.t < T:
        ref.step(min(ref.maxDt(), T - ref.t))
        n += 1
    assert done == n and gpu.t == ref.t
    assert_fields_equal(gpu, ref)
    # a fixed-dt run
    done = gpu.run(40, dt=0.01)
    for _ in range(40):
        ref.step(0.01)
    assert done == 40
    assert_fields_equal(gpu, ref)


def test_diagnostics(swe):
    kw = dam_break(60, 44, manning=0)
    gpu, ref = pair(swe, **kw)
    for _ in range(6):
        dt = ref.maxDt()
        gpu.step(dt)
        ref.step(dt)
    assert gpu.volume() == ref.volume()
    assert gpu.energy() == ref.energy()
    assert gpu.maxSurfaceDeviation(1.0) == ref.maxSurfaceDeviation(1.0)
    assert abs(gpu.maxSpeed() - ref.maxSpeed()) <= 1e-15 * ref.maxSpeed()
    assert gpu.finite() and ref.finite()
    assert gpu.dryClean() == ref.dryClean()
    gpu.applyFriction(0.1)
    ref.applyFriction(0.1)
    assert_fields_close(gpu, ref)


def test_nonfinite_is_reported(swe):
    kw = dam_break(30, 30, manning=0)
    sim = swe.ShallowWater(**kw)
    h = sim.h
    h[sim.idx(10, 10)] = float("nan")
    sim.step(0.05)
    assert not sim.finite()


def test_hllc_batch_bit_identical(swe):
    rng = np.random.default_rng(3)
    n = 4000
    h = rng.uniform(0, 3, (n, 2)) * (rng.uniform(0, 1, (n, 2)) > 0.2)
    u = rng.uniform(-6, 6, (n, 4))
    rows = np.column_stack([h[:, 0], h[:, 0] * u[:, 0], h[:, 0] * u[:, 1],
                            h[:, 1], h[:, 1] * u[:, 2], h[:, 1] * u[:, 3], np.full(n, 1e-3)])
    got = swe.hllc_batch(rows)
    for q in range(n):
        want = oracle_hllc(*rows[q])
        assert np.array_equal(got[q], want), (q, rows[q], got[q], want)
    out = [0, 0, 0]
    swe.hllc(out, 0.5, 0, 0, 0, 0, 0, 1e-3)
    assert out[0] == 2 * math.sqrt(S.G_REF * 0.5) * 0.5 / 3 or abs(out[0] - 2 * math.sqrt(S.G_REF * 0.5) * 0.5 / 3) < 1e-15


def _same_bits(a, b):
    """Equal as 64-bit patterns, or both NaN (NaN payloads are not compared)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))))


def test_zero_dividends_bit_identical(swe):
    """Still water: the momenta are +-0, and the divisions by h and by the
    velocity denominator take their zero-dividend form on the device.  The
    signs of the zero results, and infinite, NaN and zero depths, as the
    oracle gives them."""
    z = [0.0, -0.0]
    depths = [0.5, 2.0, 1.5e-3, 1e-300, 1e300, math.inf, math.nan, 0.0, -0.0, -1.0]
    rows = []
    for hL in depths:
        for hR in (0.5, 2.0, hL):
            for a in z:
                for b in z:
                    rows.append([hL, a, b, hR, b, a, 1e-3])
                    rows.append([hL, a * hL if math.isfinite(hL) else a, 1.0, hR, 0.25, b, 1e-3])
    rows = np.array(rows)
    got = swe.hllc_batch(rows)
    for q in range(len(rows)):
        want = oracle_hllc(*rows[q])
        assert _same_bits(got[q], want), (q, rows[q], got[q], want)
    sim = swe.ShallowWater(nx=4, ny=4, dx=1, bed=lambda x, y: -1, eta0=0)
    ref = OracleSim(nx=4, ny=4, dx=1, bed=lambda x, y: -1, eta0=0)
    hq = np.array([0.0, -0.0] * len(depths))
    hh = np.repeat(depths, 2)
    got = sim.vel(hq, hh)
    want = [ref.vel(float(a), float(b)) for a, b in zip(hq, hh)]
    assert _same_bits(got, want), (got, want)


def test_vel_exact(swe):
    sim = swe.ShallowWater(nx=4, ny=4, dx=1, bed=lambda x, y: -1, eta0=0)
    ref = OracleSim(nx=4, ny=4, dx=1, bed=lambda x, y: -1, eta0=0)
    for hh in (1.01e-3, 1e-2, 0.1, 1, 12, 1e3, 1e-4, 0.0):
        for u in (-9.3, 1e-6, 5):
            assert sim.vel(hh * u, hh) == ref.vel(hh * u, hh)


import json
import os

_BASE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))["sphere_baseline"]


@pytest.mark.parametrize("row", [r for r in _BASE["restingOcean"] if r["deg"] in (6, 4, 2)],
                         ids=lambda r: f"{r['case']}_{r['deg']}deg_o{r['order']}_{r['lat0']}")
def test_resting_ocean_baseline_gpu(swe, row):
    """tools/sphere-baseline.json rows on the GPU: dry counts exact, round-off
    residuals within the reference's factor-4 band, and the state bit-identical
    to the oracle after the run."""
    gpu = S.sphere(swe.ShallowWater, S.SPHERE_BEDS[row["case"]], row["deg"], order=row["order"],
                   lat0=row["lat0"], lat1=row["lat1"])
    ref = S.sphere(OracleSim, S.SPHERE_BEDS[row["case"]], row["deg"], order=row["order"],
                   lat0=row["lat0"], lat1=row["lat1"])
    assert S.dry_cells(gpu) == row["dry"]
    dt = gpu.maxDt()
    assert dt == ref.maxDt()
    assert gpu.run(row["steps"], dt=dt) == row["steps"]
    for _ in range(row["steps"]):
        ref.step(dt)
    sp, et = gpu.maxSpeed(), gpu.maxSurfaceDeviation(0)
    for got, want in ((sp, row["maxSpeed"]), (et, row["maxEta"])):
        if got == 0 or want == 0:
            assert got == want
        else:
            assert 0.25 <= got / want <= 4
    assert_fields_equal(gpu, ref)


@pytest.mark.parametrize("row", [r for r in _BASE["merian"] if r["deg"] in (6, 4)], ids=lambda r: f"n{r['n']}_{r['deg']}")
def test_merian_baseline_gpu(swe, row):
    r = S.merian(swe.ShallowWater, row["n"], row["deg"])
    assert abs(r["errPct"] - row["errPct"]) <= 0.005


def test_large_grid_against_threaded_oracle(swe):
    """1024 x 768 wet/dry beach (several strips and row chunks): bit-identical
    to the oracle after 4 steps, volume conserved."""
    nx, ny, dx = 1024, 768, 2.0
    b = S.beach_bed(nx, ny, dx)
    x = (np.arange(nx + 4) - 2 + 0.5) * dx
    eta = np.where(x < 500, 5.0, 0.0)[None, :].repeat(ny + 4, axis=0)
    kw = dict(nx=nx, ny=ny, dx=dx, bed=b, eta0=eta, manning=0)
    gpu = swe.ShallowWater(**kw)
    ref = OracleSim(threads=8, **kw)
    v0 = gpu.volume()
    assert v0 == ref.volume()
    for _ in range(4):
        dt = ref.maxDt()
        assert gpu.maxDt() == dt
        gpu.step(dt)
        ref.step(dt)
    assert_fields_equal(gpu, ref)
    assert abs(gpu.volume() - v0) / v0 < 1e-13


def _flooding_beach(cls, **extra):
    """A dam break running up a dry 1:50 beach: most 32 x 8 tiles start with
    h exactly 0 (the tiled kernels skip them) and flood one by one.  No
    friction, so the comparison with the oracle is bit for bit."""
    from water_simulator_b200 import workloads
    b, h = workloads.beach_dam_break(nx=256, ny=96, dx=8.0)
    return cls(nx=256, ny=96, dx=8.0, bed=b, eta0=b + h, manning=0, **extra)


def test_flooding_beach_bit_identical(swe):
    gpu, ref = _flooding_beach(swe.ShallowWater), _flooding_beach(OracleSim)
    set_bc(swe, gpu, ref, west=("flather", lambda t: 0.0, lambda t: 0.0))
    for step in range(60):
        gpu.step()
        ref.step()
        if step % 15 == 14:
            assert_fields_equal(gpu, ref, what=f"beach step {step}")
    assert gpu.t == ref.t


def test_sphere_with_land_bit_identical(swe):
    """Land at +50 m (h exactly 0) under the spherical metric and Coriolis."""
    from water_simulator_b200 import workloads
    c = workloads.globe_tide(nx=180, ny=90, lat0=-80.0, lat1=80.0, modes=12)
    eta0 = c["eta0"] + np.where(c["b"] < 0, 2.0 * np.exp(-((c["lon"] - 30) ** 2 + c["lat"] ** 2) / 200), 0.0)
    kw = dict(nx=180, ny=90, bed=c["b"], eta0=eta0, sphere={"R": 6371e3, "lat0": -80.0, "lat1": 80.0,
                                                            "omega": 7.2921e-5})
    gpu, ref = swe.ShallowWater(**kw), OracleSim(**kw)
    for step in range(30):
        gpu.step()
        ref.step()
    assert_fields_equal(gpu, ref, what="sphere with land")


@pytest.mark.parametrize("stage", ["fused", "split"])
def test_mass_floored_nonzero_within_tolerance(swe, monkeypatch, stage):
    """massFloored where it is not zero.  Negative depths planted in dry
    cells far apart (in different tiles and strips) are floored by both
    stages' dryClean; the reference sums them in one row-major pass
    (src/swe.mjs:734-745, 796-806), the device per tile and then in tile
    order, so the two sums of the same positive terms agree to round-off:
    1e-13 relative, stated here.  Every field stays bit-identical."""
    monkeypatch.setenv("SWE_B200_STAGE", stage)
    kw = dict(nx=150, ny=90, dx=4.0, bed=lambda x, y: 1.0, eta0=0.0, manning=0)
    gpu, ref = pair(swe, **kw)
    rng = np.random.default_rng(21)
    cells = [(int(i), int(j)) for i, j in zip(rng.integers(3, 147, 40), rng.integers(3, 87, 40))]
    depths = -rng.uniform(1e-4, 3e-2, len(cells))
    for sim in (gpu, ref):
        h = sim.h
        for (i, j), d in zip(cells, depths):
            h[sim.idx(i, j)] = d
    for step in range(3):
        gpu.step(0.05)
        ref.step(0.05)
        want = ref.massFloored
        if step == 0:
            assert want > 0
        assert abs(gpu.massFloored - want) <= 1e-13 * max(want, 1e-300), (step, gpu.massFloored, want)
        assert_fields_equal(gpu, ref, what=f"floored step {step}")
    gpu.close()
