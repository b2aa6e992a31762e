"""Spherical scenarios that drive ShallowWater({sphere}) (src/globe.mjs of the
reference: GLOBE_BEDS, GLOBE_INITS, legendreP, dropBump, surveyBed,
polarTimestepTax, measureModePeriod).  These are callers of the step; the
step itself runs on the GPU.  The Canvas views of that file are not part of
the solver path and are not restated.
"""
import math

import numpy as np

from .swe import ShallowWater

D2R = math.pi / 180
R2D = 180 / math.pi


def wrapLon(lonDeg):
    """src/globe.mjs:470-472: longitude folded into [-180, 180)."""
    return math.fmod(math.fmod(lonDeg + 180, 360) + 360, 360) - 180


def _grid_of(sim):
    g = sim.geom
    if g is None or g.kind != "sphere":
        raise ValueError("globe scenarios take spherical simulations only: sim.geom.kind is "
                         f"{getattr(g, 'kind', None)}")
    return g


def _seamount(lon, lat):
    dl, dp = wrapLon(lon + 40), lat - 30
    return -4000 + 5200 * math.exp(-((dl * dl + dp * dp) / (2 * 14 * 14)))


def _cone(lon, lat):
    dl, dp = wrapLon(lon + 90), lat - 30
    rr = min(20, math.hypot(dl, dp))
    return -4000 + 2000 * (1 - rr / 20)


# src/globe.mjs:1048-1085
GLOBE_BEDS = {
    "flat": {"title": "aquaplanet - flat bed, uniform 4000 m", "bed": lambda lon, lat: -4000.0},
    "zonalRidge": {"title": "zonal ridge - 2500 m sill at 18 N",
                   "bed": lambda lon, lat: -4000 + 2500 * math.exp(-(((lat - 18) / 7) ** 2))},
    "seamount": {"title": "Gaussian seamount - pierces the surface", "bed": _seamount},
    "williamsonCone": {"title": "Williamson-case-5-style cone (shape unverified)", "bed": _cone},
}


def legendreP(n, x):
    """src/globe.mjs:1088-1094"""
    if n == 2:
        return 0.5 * (3 * x * x - 1)
    if n == 3:
        return 0.5 * (5 * x * x * x - 3 * x)
    if n == 4:
        return (35 * x ** 4 - 30 * x * x + 3) / 8
    raise ValueError(f"legendreP: n = {n} is not one of 2, 3, 4. n = 1 is a rigid translation of "
                     "the shell and has no restoring force, n = 0 is a change of total volume.")


def _blob(a):
    def f(lon, lat):
        dl, dp = wrapLon(lon), lat - 20
        return a * math.exp(-((dl * dl + dp * dp) / (2 * 12 * 12)))
    return f


# src/globe.mjs:1106-1119
GLOBE_INITS = {
    "still": {"mode": 0, "eta": lambda a: (lambda lon, lat: 0.0)},
    "mode2": {"mode": 2, "eta": lambda a: (lambda lon, lat: a * legendreP(2, math.sin(lat * D2R)))},
    "mode3": {"mode": 3, "eta": lambda a: (lambda lon, lat: a * legendreP(3, math.sin(lat * D2R)))},
    "mode4": {"mode": 4, "eta": lambda a: (lambda lon, lat: a * legendreP(4, math.sin(lat * D2R)))},
    "blob": {"mode": 0, "eta": _blob},
}


def dropBump(sim, lonDeg, latDeg, amp=1.0, sigmaDeg=8.0):
    """src/globe.mjs:1122-1133: add a Gaussian to every wet cell's depth."""
    _grid_of(sim)
    h = sim.h
    for j in range(sim.ny):
        for i in range(sim.nx):
            lo, la = sim.cellLonLat(i, j)
            dl, dp = wrapLon(lo - lonDeg), la - latDeg
            e = amp * math.exp(-((dl * dl + dp * dp) / (2 * sigmaDeg * sigmaDeg)))
            k = sim.idx(i, j)
            if h[k] > sim.minDepth:
                h[k] += e


def surveyBed(sim):
    """src/globe.mjs:1003-1015"""
    _grid_of(sim)
    b, h = sim.field("b"), sim.field("h")
    mn, mx, dry, crest = math.inf, -math.inf, 0, -math.inf
    for j in range(sim.ny):
        for i in range(sim.nx):
            k = sim.idx(i, j)
            bk = b[k]
            mn = min(mn, bk)
            mx = max(mx, bk)
            if h[k] <= sim.minDepth:
                dry += 1
                crest = max(crest, bk)
    return {"min": mn, "max": mx, "relief": mx - mn, "dry": dry, "crest": crest if dry else math.nan}


def polarTimestepTax(sim, H=4000.0):
    """src/globe.mjs:1022-1037: CFL step at the equator row over the worst row."""
    g = _grid_of(sim)
    ng = g.ng
    c = math.sqrt(9.80665 * H)
    dxRow, dyCFL, phiC = g._rows["dxRow"], g._rows["dyCFL"], g._rows["phiC"]
    dtOf = lambda j: sim.cfl / (c / dxRow[j] + c / dyCFL[j])
    eqJ, best = ng, math.inf
    for j in range(ng, g.H - ng):
        a = abs(phiC[j])
        if a < best:
            best, eqJ = a, j
    worstJ = ng
    for j in range(ng, g.H - ng):
        if dtOf(j) < dtOf(worstJ):
            worstJ = j
    eq, pole = dtOf(eqJ), dtOf(worstJ)
    return {"eq": eq, "pole": pole, "ratio": eq / pole, "poleLat": phiC[worstJ] * R2D,
            "eqLat": phiC[eqJ] * R2D}


def measureModePeriod(n=2, deg=6, H=4000.0, R=6371e3, gRef=None, amp=1.0, periods=2, cfl=0.45,
                      lat0=-90, lat1=90, order=2, onProgress=None):
    """src/globe.mjs:1387-1450: period of the zonal mode P_n(sin lat) from
    zero crossings of its area-weighted projection."""
    if not (gRef is not None and gRef > 0):
        raise ValueError("measureModePeriod: gRef is required. A closed form built from the "
                         "solver's own G rescales with any error in it and can never detect one.")
    nx, ny = round(360 / deg), round((lat1 - lat0) / deg)
    closed = 2 * math.pi * R / math.sqrt(gRef * H * n * (n + 1))
    sim = ShallowWater(nx=nx, ny=ny, bed=lambda lon, lat: -H, manning=0, cfl=cfl, order=order,
                       eta0=lambda lon, lat: amp * legendreP(n, math.sin(lat * D2R)),
                       sphere={"R": R, "lat0": lat0, "lat1": lat1, "omega": 0})
    g = sim.geom
    ng = g.ng
    phiC, area = g._rows["phiC"], g._rows["area"]
    wRow, pRow = np.zeros(ny), np.zeros(ny)
    norm = 0.0
    for j in range(ny):
        P = legendreP(n, math.sin(phiC[j + ng]))
        pRow[j] = P
        wRow[j] = area[j + ng] * nx
        norm += wRow[j] * P * P

    def project():
        eta = (sim.field("b") + sim.field("h")).reshape(sim.H, sim.W)[2:-2, 2:-2]
        rows = np.cumsum(eta, axis=1)[:, -1]            # left-to-right, as `row += ...`
        s = 0.0
        for j in range(ny):
            s += (wRow[j] / nx) * pRow[j] * rows[j]
        return s / norm

    tEnd = periods * closed
    cross = []
    prevT, prevC, steps = 0.0, project(), 0
    c0 = prevC
    t = 0.0
    while t < tEnd:
        dt = min(sim.maxDt(), tEnd - t)
        if not dt > 0:
            break
        sim.step(dt)
        steps += 1
        t = sim.t
        c = project()
        if (prevC < 0) != (c < 0):
            cross.append(prevT + (t - prevT) * (0 - prevC) / (c - prevC))
        prevT, prevC = t, c
        if onProgress and steps % 200 == 0:
            onProgress(t / tEnd)
    sim.close()
    if len(cross) < 2:
        return {"measured": math.nan, "closed": closed, "rel": math.nan, "steps": steps,
                "crossings": len(cross), "amp0": c0, "ampEnd": prevC,
                "note": "fewer than two zero crossings: nothing to measure"}
    measured = 2 * (cross[-1] - cross[0]) / (len(cross) - 1)
    return {"measured": measured, "closed": closed, "rel": (measured - closed) / closed, "steps": steps,
            "crossings": len(cross), "amp0": c0, "ampEnd": prevC, "nx": nx, "ny": ny, "deg": deg}
