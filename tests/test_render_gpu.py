"""Headless frames on the device against restatements of the reference's
drawing code: WaterView's map panel (src/render.mjs:220-247), buildGlobeLut
(src/globe.mjs:554-629) and renderGlobe (src/globe.mjs:770-812); and the
reference's own recorded end-to-end pixels (src/render.mjs:59-64)."""
import math

import numpy as np
import pytest

from test_render_tables import js_round, u8clamp

pytestmark = pytest.mark.gpu
MID = 512


def u8v(x):
    return np.array([u8clamp(v) for v in x], dtype=np.uint8)


def near_half(x, tol=1e-9):
    f = math.floor(x)
    return abs((x - f) - 0.5) < tol


def map_reference(swe, sim, msl, scale, show_bed):
    """WaterView.draw()'s map loop; returns bytes and the pre-rounding values."""
    ramp, _ = swe.colourTables()
    nx, ny, W = sim.nx, sim.ny, sim.W
    b, h = sim.field("b"), sim.field("h")
    out = np.zeros((ny, nx, 4), np.uint8)
    raw = np.zeros((ny, nx, 3))
    for j in range(ny):
        for i in range(nx):
            k = (j + 2) * W + (i + 2)
            depth = h[k]
            if depth <= sim.minDepth:
                t = max(0, min(1, b[k] / 6))
                c = [96 + 70 * t, 88 + 62 * t, 74 + 52 * t]
            else:
                v = b[k] + depth - msl
                t = max(-1, min(1, v / scale))
                q = js_round(abs(t) * MID)
                c = list(ramp[MID + q] if t >= 0 else ramp[MID - q])
                if show_bed:
                    still = max(0, msl - b[k])
                    shade = 0.55 + 0.45 * math.exp(-still / 12)
                    c = [c[0] * shade, c[1] * shade, c[2] * shade]
            out[ny - 1 - j, i, :3] = u8v(c)
            out[ny - 1 - j, i, 3] = 255
            raw[ny - 1 - j, i] = c
    return out, raw


@pytest.mark.parametrize("show_bed", [True, False])
def test_map_panel_matches_the_drawing_loop(swe, show_bed):
    from water_simulator_b200 import workloads
    b, eta = workloads.bump_dam_break(nx=48, ny=40, dx=5.0)
    b = b - 1.0                                  # some dry land above the dam break's low side
    sim = swe.ShallowWater(nx=48, ny=40, dx=5.0, bed=b, eta0=eta)
    for _ in range(20):
        sim.step()
    got = swe.renderMap(sim, msl=0.3, scale=1.5, showBed=show_bed)
    want, raw = map_reference(swe, sim, 0.3, 1.5, show_bed)
    diff = np.argwhere(got != want)
    for (y, x, c) in diff:                       # only exp() rounding at an exact half may differ
        assert c < 3 and near_half(raw[y, x, c]) and abs(int(got[y, x, c]) - int(want[y, x, c])) == 1
    assert len(diff) <= 2
    sim.close()


def test_map_recorded_crest_and_trough_pixels(swe):
    """src/render.mjs:59-64: 12 m of water at scale 1 m, a +1.00 m crest beside a
    -1.00 m trough: rgb(181,149,94) and rgb(2,34,70) against rgb(75,93,107)."""
    sim = swe.ShallowWater(nx=8, ny=4, dx=10.0, bed=-12.0, eta0=0.0)
    h = sim.h
    W = sim.W
    h[(2 + 1) * W + (2 + 3)] = 13.0
    h[(2 + 1) * W + (2 + 4)] = 11.0
    img = swe.renderMap(sim, msl=0.0, scale=1.0, showBed=True)
    row = img[4 - 1 - 1]
    assert tuple(row[3, :3]) == (181, 149, 94)
    assert tuple(row[4, :3]) == (2, 34, 70)
    assert tuple(row[0, :3]) == (75, 93, 107)
    sim.close()


def test_map_nan_paints_zero(swe):
    sim = swe.ShallowWater(nx=6, ny=5, dx=1.0, bed=-2.0, eta0=0.0)
    sim.h[(2 + 2) * sim.W + 3] = float("nan")
    img = swe.renderMap(sim)
    assert tuple(img[5 - 1 - 2, 1]) == (0, 0, 0, 255)
    sim.close()


# ---- the globe ------------------------------------------------------------------
def bake_reference(size, tilt, margin, nx, ny, lat0, lat1, sun=(-0.42, 0.48, 0.77)):
    D2R, R2D = math.pi / 180, 180 / math.pi
    r, cx, cy = 0.5 * size * margin, 0.5 * size, 0.5 * size
    sinT, cosT = math.sin(tilt * D2R), math.cos(tilt * D2R)
    m = math.sqrt(sun[0] ** 2 + sun[1] ** 2 + sun[2] ** 2)
    su = [s / m for s in sun]
    px, lon, rb, lit = [], [], [], []
    bg = np.zeros(4 * size * size, np.uint8)
    inside = capped = 0
    W = nx + 4
    for y in range(size):
        for x in range(size):
            o = 4 * (y * size + x)
            X, Y = (x + 0.5 - cx) / r, (cy - y - 0.5) / r
            s = X * X + Y * Y
            if s > 1:
                g = math.exp(-(s - 1) * 5.5)
                bg[o:o + 3] = u8v([8 + (36 - 8) * g, 11 + (58 - 11) * g, 16 + (84 - 16) * g])
                bg[o + 3] = 255
                continue
            inside += 1
            z = math.sqrt(1 - s)
            phi = math.asin(z * sinT + Y * cosT)
            lam = math.atan2(X, z * cosT - Y * sinT)
            lonD, latD = 0 + lam * R2D, phi * R2D
            if latD < lat0 or latD > lat1:
                j = -1
            else:
                j = math.floor((latD - lat0) * ny / (lat1 - lat0))
                j = ny - 1 if j >= ny else max(j, 0)
            if j < 0:
                capped += 1
                t = 1 if ((x + y) & 7) < 3 else 0
                bg[o:o + 4] = [52 + 14 * t, 56 + 14 * t, 62 + 14 * t, 255]
                continue
            px.append(o)
            lon.append(lonD)
            rb.append((j + 2) * W + 2)
            lit.append(np.float32(max(0, X * su[0] + Y * su[1] + z * su[2])))
    return {"px": np.array(px, np.int32), "lonBase": np.array(lon), "rowBase": np.array(rb, np.int32),
            "lit": np.array(lit, np.float32), "bg": bg, "inside": inside, "capped": capped}


def frame_reference(swe, sim, lut, rot, scale, msl, land_light):
    _, cb = swe.colourTables()
    cb = cb.reshape(-1)
    out = lut["bg"].copy()
    b, h = sim.field("b"), sim.field("h")
    nx = sim.nx
    wet = dry = sat = 0
    lo, hi = math.inf, -math.inf
    for p in range(len(lut["px"])):
        lonD = lut["lonBase"][p] + rot
        i = math.floor((lonD + 180) * nx / 360)
        k = int(lut["rowBase"][p]) + ((i % nx) + nx) % nx
        o = int(lut["px"][p])
        if h[k] <= sim.minDepth:
            dry += 1
            t = max(0, min(1, b[k] / 2500))
            s = 0.30 + 0.70 * float(lut["lit"][p]) if land_light else 1
            c = [92 + (188 - 92) * t, 84 + (172 - 84) * t, 70 + (144 - 70) * t]
            out[o:o + 3] = u8v([c[0] * s, c[1] * s, c[2] * s])
        else:
            wet += 1
            e = b[k] + h[k] - msl
            lo, hi = min(lo, e), max(hi, e)
            if e >= scale or e <= -scale:
                sat += 1
            t = max(-1, min(1, e / scale))
            q = js_round(abs(t) * MID)
            c = 3 * (MID + q if t >= 0 else MID - q)
            out[o:o + 3] = cb[c:c + 3]
        out[o + 3] = 255
    return out, {"wet": wet, "dry": dry, "etaMin": lo, "etaMax": hi, "sat": sat}


def globe_sim(swe, nx=72, ny=30, lat0=-60.0, lat1=60.0):
    from water_simulator_b200 import workloads
    c = workloads.globe_tide(nx=nx, ny=ny, lat0=lat0, lat1=lat1, modes=12)
    sim = swe.ShallowWater(nx=nx, ny=ny, bed=c["b"], eta0=c["eta0"],
                           sphere={"R": 6371e3, "lat0": lat0, "lat1": lat1, "omega": 7.2921e-5})
    sim.h[:] = np.where(sim.h > 0, sim.h + 0.4 * np.sin(np.arange(sim.h.size) * 0.37), sim.h)
    return sim


def test_globe_lut_is_the_reference_bake(swe):
    sim = globe_sim(swe)
    cam = swe.globeCamera(96, tiltDeg=22, margin=0.94)
    lut = swe.buildGlobeLut(cam, sim)
    got = lut.arrays()
    ref = bake_reference(96, 22, 0.94, sim.nx, sim.ny, -60.0, 60.0)
    assert (lut.count, lut.inside, lut.capped) == (len(ref["px"]), ref["inside"], ref["capped"])
    assert ref["capped"] > 0 and lut.count > 0
    assert np.array_equal(got["px"], ref["px"]) and np.array_equal(got["rowBase"], ref["rowBase"])
    assert np.max(np.abs(got["lonBase"] - ref["lonBase"])) <= 1e-12
    assert np.max(np.abs(got["lit"].astype(np.float64) - ref["lit"])) <= 1e-6
    assert np.max(np.abs(got["bg"].astype(int) - ref["bg"].astype(int))) <= 1
    lut.close(); sim.close()


@pytest.mark.parametrize("rot,land_light", [(0.0, True), (37.5, True), (-400.25, False)])
def test_globe_frame_matches_the_render_loop(swe, rot, land_light):
    sim = globe_sim(swe)
    for _ in range(5):
        sim.step()
    cam = swe.globeCamera(96, tiltDeg=30, margin=0.9)
    lut = swe.buildGlobeLut(cam, sim)
    out = np.zeros(4 * 96 * 96, np.uint8)
    stats = swe.renderGlobe(out, sim, lut, rotDeg=rot, scale=0.3, msl=0.0, landLight=land_light)
    want, ws = frame_reference(swe, sim, lut.arrays(), rot, 0.3, 0.0, land_light)
    assert np.array_equal(out, want)
    for key in ("wet", "dry", "etaMin", "etaMax", "sat"):
        assert stats[key] == ws[key], key
    assert stats["capped"] == lut.capped and stats["inside"] == lut.inside
    assert stats["satFrac"] == (ws["sat"] / ws["wet"] if ws["wet"] else 0)
    lut.close(); sim.close()


def test_resting_ocean_is_one_colour(swe):
    """A resting ocean paints every wet pixel with the mean-sea-level byte: the
    water is never lit (src/globe.mjs: the Lambert factor is refused)."""
    from water_simulator_b200 import workloads
    c = workloads.globe_tide(nx=72, ny=36, lat0=-90.0, lat1=90.0, modes=12)
    sim = swe.ShallowWater(nx=72, ny=36, bed=c["b"], eta0=0.0, sphere={"R": 6371e3})
    lut = swe.buildGlobeLut(swe.globeCamera(80), sim)
    out = np.zeros(4 * 80 * 80, np.uint8)
    st = swe.renderGlobe(out, sim, lut)
    _, cb = swe.colourTables()
    px = lut.arrays()["px"]
    cols = out.reshape(-1, 4)[px // 4][:, :3]
    wet = np.all(cols == cb[MID], axis=1)
    assert wet.sum() == st["wet"] and st["wet"] > 0 and st["capped"] == 0
    assert st["etaMin"] == 0 and st["etaMax"] == 0
    lut.close(); sim.close()


def test_globe_refusals(swe):
    flat = swe.ShallowWater(nx=8, ny=8, dx=1.0, bed=-1.0, eta0=0.0)
    with pytest.raises(swe.SweError, match="spherical fields only"):
        swe.buildGlobeLut(swe.globeCamera(32), flat)
    a = globe_sim(swe, nx=36, ny=18)
    bsim = globe_sim(swe, nx=40, ny=18)
    lut = swe.buildGlobeLut(swe.globeCamera(32), a)
    with pytest.raises(swe.SweError, match="LUT was baked for"):
        swe.renderGlobe(np.zeros(4 * 32 * 32, np.uint8), bsim, lut)
    lut.close(); a.close(); bsim.close(); flat.close()
