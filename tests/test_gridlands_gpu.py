"""The gridlands import on the device: base64 decoding against Python's own,
the sampled bed / depth / Manning fields against a numpy restatement of
gridlandsTerrain()'s sampling (src/gridlands.mjs:262-291) bit for bit, and
the reference suite's gates on an imported world (tools/verify-gridlands.mjs):
row flip, ghost clamp, lake at rest once settled, volume, per-cell Manning."""
import base64
import math

import numpy as np
import pytest

from gridlands_doc import b64, make_doc, terrain_arrays

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


# ---- the checker: gridlandsTerrain()'s sampling, vectorised -----------------
def js_round(x):
    f = np.floor(x)
    return np.where(x - f >= 0.5, f + 1, f)


def sample_reference(bedM, surfM, nM, Wg, Hg, C, nx, ny, dx, dy, flip=True):
    """b, h (= Math.max(0, eta0 - b)) and n at every padded cell centre."""
    i = np.arange(nx + 4, dtype=np.float64) - 2
    j = np.arange(ny + 4, dtype=np.float64) - 2
    X, Y = np.meshgrid((i + 0.5) * dx, (j + 0.5) * dy)
    fc = np.minimum(Wg - 1, np.maximum(0, X / C - 0.5))
    rr = np.minimum(Hg - 1, np.maximum(0, Y / C - 0.5))
    fr = (Hg - 1) - rr if flip else rr
    c0, r0 = np.floor(fc).astype(np.int64), np.floor(fr).astype(np.int64)
    c1, r1 = np.minimum(Wg - 1, c0 + 1), np.minimum(Hg - 1, r0 + 1)
    tc, tr = fc - c0, fr - r0
    B = bedM.astype(np.float64)
    v00, v10, v01, v11 = B[r0 * Wg + c0], B[r0 * Wg + c1], B[r1 * Wg + c0], B[r1 * Wg + c1]
    b = (v00 * (1 - tc) + v10 * tc) * (1 - tr) + (v01 * (1 - tc) + v11 * tc) * tr
    kn = js_round(fr).astype(np.int64) * Wg + js_round(fc).astype(np.int64)
    e = surfM.astype(np.float64)[kn]
    d = e - b
    h = np.where(d > 0, d, 0.0)
    n = nM.astype(np.float64)[kn] if nM is not None else None
    return b.reshape(-1), h.reshape(-1), (n.reshape(-1) if n is not None else None)


# ---- decoding -----------------------------------------------------------------
def test_decode_matches_python_base64(swe):
    from water_simulator_b200 import gridlands as gl
    doc = make_doc()
    n = 64 * 48
    for name in ("bedM", "surfaceM", "manningN"):
        txt = doc["layers"][name]["data"]
        want = np.frombuffer(base64.b64decode(txt), dtype="<f4")
        got = gl.decodeF32(doc["layers"][name], n, name)
        assert got.view(np.uint32).tolist() == want.view(np.uint32).tolist(), name


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 1000])
def test_decode_lengths_padding_and_urlsafe(swe, n):
    from water_simulator_b200 import gridlands as gl
    a = np.random.default_rng(n).normal(0, 100, n).astype(np.float32)
    std = b64(a)
    for txt in (std, std.rstrip("="), base64.urlsafe_b64encode(a.astype("<f4").tobytes()).decode()):
        got = gl.decodeF32({"encoding": "b64f32le", "data": txt}, n, "bedM")
        assert np.array_equal(got.view(np.uint32), a.view(np.uint32))


def test_decode_refuses_truncated_and_foreign(swe):
    from water_simulator_b200 import gridlands as gl
    a = np.arange(100, dtype=np.float32)
    txt = b64(a)
    with pytest.raises(ValueError, match="layer bedM decoded to 300 bytes, expected 400"):
        gl.decodeF32({"encoding": "b64f32le", "data": txt[:400]}, 100, "bedM")
    with pytest.raises(ValueError, match="outside the alphabet"):
        gl.decodeF32({"encoding": "b64f32le", "data": txt[:10] + "*" + txt[11:]}, 100, "bedM")
    # a truncated layer inside a document is refused, not read as terrain
    doc = make_doc()
    doc["layers"]["bedM"]["data"] = doc["layers"]["bedM"]["data"][:1000]
    with pytest.raises(ValueError, match="decoded to"):
        gl.gridlandsTerrain(doc)


# ---- sampling -------------------------------------------------------------------
@pytest.mark.parametrize("grid", [
    dict(nx=64, ny=48, dx=50.0, dy=50.0),          # native 1:1
    dict(nx=128, ny=96, dx=25.0, dy=25.0),         # finer than the export: bilinear for real
    dict(nx=40, ny=30, dx=80.0, dy=80.0),          # coarser
    dict(nx=53, ny=61, dx=37.0, dy=41.0),          # unrelated spacing, anisotropic
])
def test_device_sampling_is_the_reference_sampling(swe, grid):
    doc = make_doc()
    t = swe.gridlandsTerrain(doc)
    sim = swe.ShallowWater(bed=t.bed, eta0=t.eta0, manning=0.03, **grid)
    b, h, _ = sample_reference(t.bedM, t.surfaceM, None, 64, 48, 50.0, grid["nx"], grid["ny"],
                               grid["dx"], grid["dy"])
    assert np.array_equal(sim.field("b"), b)
    assert np.array_equal(sim.field("h"), h)
    # and the host functions the terrain hands out give the same doubles
    W = grid["nx"] + 4
    for k in range(0, (grid["ny"] + 4) * W, 97):
        x, y = sim.cellCentre(k % W - 2, k // W - 2)
        assert t.bed(x, y) == b[k]
        assert max(0.0, t.eta0(x, y) - t.bed(x, y)) == h[k]
    sim.close()


def test_row_flip_probe_and_its_mutant(swe):
    """tools/verify-gridlands.mjs:136-168: the sim's top row is the export's row 0."""
    doc = make_doc()
    t = swe.gridlandsTerrain(doc)
    sim = swe.ShallowWater.fromGridlands(t)
    W, H = t.W, t.H
    b = sim.field("b").reshape(H + 4, W + 4)
    top = b[2 + H - 1, 2:-2]
    assert np.array_equal(top, t.bedM[:W].astype(np.float64))            # north row
    assert not np.array_equal(top, t.bedM[(H - 1) * W:].astype(np.float64))
    tf = swe.gridlandsTerrain(doc, flipRows=False)
    simf = swe.ShallowWater.fromGridlands(tf)
    topf = simf.field("b").reshape(H + 4, W + 4)[2 + H - 1, 2:-2]
    assert not np.array_equal(topf, t.bedM[:W].astype(np.float64))       # the mutant is caught
    sim.close(); simf.close()


def test_ghost_rings_are_clamped(swe):
    t = swe.gridlandsTerrain(make_doc())
    sim = swe.ShallowWater.fromGridlands(t)
    b = sim.field("b").reshape(t.H + 4, t.W + 4)
    assert np.all(np.isfinite(b))
    assert np.array_equal(b[:, 0], b[:, 2]) and np.array_equal(b[:, 1], b[:, 2])
    assert np.array_equal(b[0, :], b[2, :]) and np.array_equal(b[-1, :], b[-3, :])
    sim.close()


# ---- the imported world in the solver -------------------------------------------
def rest_run(swe, t, steps, fixed_dt=True):
    """tools/verify-gridlands.mjs:189-226 (fixed dt from the still state).  A
    world that is not at rest is stepped with dt = maxDt() instead: a spill
    speeds up past the still state's CFL limit, and a fixed dt would then be
    the test violating the Courant condition (tools/verify-gridlands.mjs:276-281)."""
    sim = swe.ShallowWater.fromGridlands(t, manning=0, cfl=0.45)
    e0 = sim.field("b") + sim.field("h")
    hmax = float(sim.field("h").reshape(t.H + 4, t.W + 4)[2:-2, 2:-2].max())
    v0, dt = sim.volume(), sim.maxDt()
    for _ in range(steps):
        sim.step(dt if fixed_dt else None)
    h = sim.field("h")
    wet = np.zeros(h.shape, bool)
    wet.reshape(t.H + 4, t.W + 4)[2:-2, 2:-2] = h.reshape(t.H + 4, t.W + 4)[2:-2, 2:-2] > sim.minDepth
    dEta = float(np.max(np.abs((sim.field("b") + h) - e0)[wet]))
    out = dict(spd=sim.maxSpeed(), dEta=dEta, drift=abs((sim.volume() - v0) / v0), dt=dt, hmax=hmax,
               finite=sim.finite())
    sim.close()
    return out


def test_lake_at_rest_once_settled_and_not_before(swe):
    doc = make_doc()
    steps = 300
    settled = rest_run(swe, swe.gridlandsTerrain(doc, settle=True), steps)
    # The perched lake spills down bare 1:2 slopes with no friction; the
    # oracle (the reference's arithmetic) stays finite past step 200 and
    # blows up at 221 on the thin film, so the spill is watched for 100.
    imported = rest_run(swe, swe.gridlandsTerrain(doc), 100, fixed_dt=False)
    uTol = 4 * EPS * 9.80665 * settled["hmax"] * settled["dt"] * steps / 50.0
    assert settled["spd"] < uTol, settled
    assert settled["dEta"] < 1e-9, settled
    assert settled["finite"] and imported["finite"]
    assert settled["drift"] < 1e-13 and imported["drift"] < 1e-13
    assert imported["spd"] > settled["spd"] * 1e3            # the perched lake spills


def test_per_cell_manning_lands_on_the_bed_cells(swe):
    doc = make_doc()
    t = swe.gridlandsTerrain(doc, settle=True)
    sim = swe.ShallowWater.fromGridlands(t, manningField=True)
    _, _, n = sample_reference(t.bedM, t.surfaceM, t.manningN, 64, 48, 50.0, 64, 48, 50.0, 50.0)
    assert np.array_equal(sim.manningField, n)
    assert np.array_equal(sim.field("manning"), n)
    nf = sim.manningField.reshape(t.H + 4, t.W + 4)
    for j in range(t.H):
        assert np.array_equal(nf[2 + j, 2:-2], t.manningN[(t.H - 1 - j) * t.W:(t.H - j) * t.W].astype(np.float64))
    # the host sampler handed out for setManningField gives the same field
    sim2 = swe.ShallowWater.fromGridlands(t)
    sim2.setManningField(t.manningAt)
    assert np.array_equal(sim2.field("manning"), n)
    sim.close(); sim2.close()


def test_per_cell_manning_changes_the_flood(swe):
    """tools/verify-gridlands.mjs:339-374: the field must give a different answer."""
    doc = make_doc()
    t = swe.gridlandsTerrain(doc, settle=True)

    def flood(field):
        s = swe.ShallowWater.fromGridlands(t, manningField=field)
        h = s.field("h").reshape(t.H + 4, t.W + 4)
        b = s.field("b").reshape(t.H + 4, t.W + 4)
        Y, X = np.meshgrid((np.arange(t.H + 4) - 1.5) * 50.0, (np.arange(t.W + 4) - 1.5) * 50.0, indexing="ij")
        bump = 3.0 * np.exp(-(((X - 1200) / 400) ** 2 + ((Y - 600) / 400) ** 2))
        h2 = np.where(h > 0, h + bump, h)
        s.h[:] = h2.reshape(-1)
        for _ in range(200):
            s.step()
        v = s.maxSpeed()
        ok = s.finite()
        s.close()
        return v, ok

    vS, okS = flood(False)
    vF, okF = flood(True)
    assert okS and okF
    assert abs(vS - vF) > 1e-9


def test_bad_manning_layer_is_refused(swe):
    doc = make_doc()
    b, s, n = terrain_arrays()
    n = n.copy()
    n[5, 7] = -1.0
    doc["layers"]["manningN"]["data"] = b64(n)
    t = swe.gridlandsTerrain(doc)
    with pytest.raises(swe.SweError, match="Manning n must be finite and >= 0"):
        swe.ShallowWater.fromGridlands(t, manningField=True)
    with pytest.raises(ValueError, match="Manning n must be finite and >= 0"):
        swe.ShallowWater.fromGridlands(t).setManningField(t.manningAt)
