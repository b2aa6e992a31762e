"""Spherical scenarios that drive ShallowWater({sphere}): the callers of the
step in src/globe.mjs of the reference (GLOBE_BEDS, GLOBE_INITS, legendreP,
dropBump, surveyBed, polarTimestepTax, measureModePeriod).

The step runs on the GPU; so does the one per-step reduction a scenario
needs, the area-weighted projection of eta onto a zonal mode
(swe_eta_projection), so measureModePeriod moves 8 bytes to the host per
step.  The per-cell helpers work on whole arrays at once.  The Canvas views
of src/globe.mjs are not part of the solver path.
"""
import ctypes
import math

import numpy as np

from ._lib import check, dptr
from .swe import ShallowWater

D2R = math.pi / 180
R2D = 180 / math.pi
G_LOCAL = 9.80665               # polarTimestepTax's own gravity (src/globe.mjs:1024)


def wrapLon(lonDeg):
    """Longitude folded into [-180, 180) (src/globe.mjs:470-472); scalars or arrays."""
    if np.ndim(lonDeg):
        return np.fmod(np.fmod(np.asarray(lonDeg, dtype=np.float64) + 180, 360) + 360, 360) - 180
    return math.fmod(math.fmod(lonDeg + 180, 360) + 360, 360) - 180


def _sphere_of(sim):
    g = sim.geom
    if getattr(g, "kind", None) != "sphere":
        raise ValueError(f"globe scenarios need a spherical simulation (geom.kind is {getattr(g, 'kind', None)!r})")
    return g


def _gauss_deg(dlon, dlat, sigma):
    return math.exp(-((dlon * dlon + dlat * dlat) / (2 * sigma * sigma)))


# ---------------------------------------------------------------------------
# Beds, (lonDeg, latDeg) -> bed elevation [m], positive up (src/globe.mjs:1048-1085).
def _bed_flat(lon, lat):
    return -4000.0


def _bed_ridge(lon, lat):
    return -4000 + 2500 * math.exp(-(((lat - 18) / 7) ** 2))


def _bed_seamount(lon, lat):                # 30 N 40 W, crest 1200 m above sea level
    return -4000 + 5200 * _gauss_deg(wrapLon(lon + 40), lat - 30, 14)


def _bed_cone(lon, lat):                    # radius 20 deg, 2000 m tall, 30 N 90 W
    r = min(20, math.hypot(wrapLon(lon + 90), lat - 30))
    return -4000 + 2000 * (1 - r / 20)


GLOBE_BEDS = {
    "flat": {"title": "aquaplanet - flat bed, uniform 4000 m", "bed": _bed_flat},
    "zonalRidge": {"title": "zonal ridge - 2500 m sill at 18 N", "bed": _bed_ridge},
    "seamount": {"title": "Gaussian seamount - pierces the surface", "bed": _bed_seamount},
    "williamsonCone": {"title": "Williamson-case-5-STYLE cone (UNVERIFIED shape)", "bed": _bed_cone},
}


def legendreP(n, x):
    """P_n(x) for the zonal modes n = 2, 3, 4 (src/globe.mjs:1088-1094).
    n = 0 and n = 1 are not modes (a volume change and a rigid shift)."""
    if n == 2:
        return 0.5 * (3 * x * x - 1)
    if n == 3:
        return 0.5 * (5 * x * x * x - 3 * x)
    if n == 4:
        return (35 * x ** 4 - 30 * x * x + 3) / 8
    raise ValueError(f"legendreP: n = {n} is not one of 2, 3, 4")


def _mode_eta(n):
    return lambda a: (lambda lon, lat: a * legendreP(n, math.sin(lat * D2R)))


# Initial surfaces, amp -> (lonDeg, latDeg) -> eta [m] (src/globe.mjs:1106-1119).
GLOBE_INITS = {
    "still": {"mode": 0, "eta": lambda a: (lambda lon, lat: 0.0)},
    "mode2": {"mode": 2, "eta": _mode_eta(2)},
    "mode3": {"mode": 3, "eta": _mode_eta(3)},
    "mode4": {"mode": 4, "eta": _mode_eta(4)},
    "blob": {"mode": 0, "eta": lambda a: (lambda lon, lat: a * _gauss_deg(wrapLon(lon), lat - 20, 12))},
}


# ---------------------------------------------------------------------------
def _interior_lonlat(sim):
    """Cell-centre longitude and latitude [deg] of the interior, (ny, nx),
    as cellLonLat gives them."""
    g = _sphere_of(sim)
    lon = (np.arange(sim.nx) + 0.5) * g.dlam * R2D
    lon = np.fmod(np.fmod(lon, 360) + 360, 360) - 180
    lat = np.asarray(g._rows["phiC"])[2:2 + sim.ny] * R2D
    return np.broadcast_to(lon, (sim.ny, sim.nx)), np.broadcast_to(lat[:, None], (sim.ny, sim.nx))


def _interior(a, sim):
    return np.asarray(a).reshape(sim.H, sim.W)[2:-2, 2:-2]


def dropBump(sim, lonDeg, latDeg, amp=1.0, sigmaDeg=8.0):
    """Add a Gaussian (amp, sigmaDeg of arc) to the depth of every wet cell
    (src/globe.mjs:1122-1133)."""
    lon, lat = _interior_lonlat(sim)
    dl, dp = wrapLon(lon - lonDeg), lat - latDeg
    bump = amp * np.exp(-((dl * dl + dp * dp) / (2 * sigmaDeg * sigmaDeg)))
    h = sim.h                                    # writable host copy, uploaded at the next call
    hi = _interior(h, sim)
    wet = hi > sim.minDepth
    hi[wet] += bump[wet]


def surveyBed(sim):
    """What the bed actually is, measured over the interior (src/globe.mjs:1003-1015):
    min, max, relief, the number of dry cells and the highest dry bed."""
    _sphere_of(sim)
    b, h = _interior(sim.field("b"), sim), _interior(sim.field("h"), sim)
    dry = h <= sim.minDepth
    nd = int(np.count_nonzero(dry))
    lo, hi = float(b.min()), float(b.max())
    return {"min": lo, "max": hi, "relief": hi - lo, "dry": nd,
            "crest": float(b[dry].max()) if nd else math.nan}


def polarTimestepTax(sim, H=4000.0):
    """The CFL step of a uniform-depth ocean at the row nearest the equator
    against the smallest row step, from the simulation's own metric
    (src/globe.mjs:1022-1037)."""
    g = _sphere_of(sim)
    ng = g.ng
    c = math.sqrt(G_LOCAL * H)
    dx, dy, phi = (np.asarray(g._rows[r])[ng:g.H - ng] for r in ("dxRow", "dyCFL", "phiC"))
    dt = np.array([sim.cfl / (c / a + c / b) for a, b in zip(dx, dy)])
    eq = int(np.argmin(np.abs(phi)))             # first of equal minima, as the loop's `<`
    worst = int(np.argmin(dt))
    return {"eq": float(dt[eq]), "pole": float(dt[worst]), "ratio": float(dt[eq] / dt[worst]),
            "poleLat": float(phi[worst] * R2D), "eqLat": float(phi[eq] * R2D)}


class ModeProjection:
    """The area-weighted projection of eta onto P_n(sin lat), in metres:
    sum_j (w_j / nx) P_j (sum_i eta_ij) / sum_j w_j P_j^2 with w_j = area_j nx
    (src/globe.mjs:1405-1422).  Evaluated on the device in the reference's
    order by swe_eta_projection; the weights are formed here as the
    reference forms them."""

    def __init__(self, sim, n):
        g = _sphere_of(sim)
        ng, nx = g.ng, sim.nx
        area, phi = np.asarray(g._rows["area"]), np.asarray(g._rows["phiC"])
        coef = np.empty(sim.ny)
        norm = 0.0
        for j in range(sim.ny):
            p = legendreP(n, math.sin(phi[j + ng]))
            w = area[j + ng] * nx
            norm += w * p * p
            coef[j] = (w / nx) * p
        self.sim, self.coef, self.norm = sim, coef, norm

    def __call__(self):
        sim = self.sim
        sim._push()
        v = ctypes.c_double()
        check(sim._lib.swe_eta_projection(sim._h, dptr(self.coef), ctypes.byref(v)))
        return v.value / self.norm


def measureModePeriod(n=2, deg=6, H=4000.0, R=6371e3, gRef=None, amp=1.0, periods=2, cfl=0.45,
                      lat0=-90, lat1=90, order=2, onProgress=None):
    """Period of the zonal free mode P_n(sin lat) of a uniform ocean of depth H
    on a deg-degree grid, from the interpolated zero crossings of its
    projection over `periods` closed-form periods (src/globe.mjs:1387-1450).
    gRef is the caller's gravity for the closed form 2 pi R / sqrt(g H n(n+1));
    the solver's own G would rescale with any error in it."""
    if not (gRef is not None and gRef > 0):
        raise ValueError("measureModePeriod: gRef is required")
    nx, ny = round(360 / deg), round((lat1 - lat0) / deg)
    closed = 2 * math.pi * R / math.sqrt(gRef * H * n * (n + 1))
    sim = ShallowWater(nx=nx, ny=ny, bed=lambda lon, lat: -H, manning=0, cfl=cfl, order=order,
                       eta0=lambda lon, lat: amp * legendreP(n, math.sin(lat * D2R)),
                       sphere={"R": R, "lat0": lat0, "lat1": lat1, "omega": 0})
    try:
        proj = ModeProjection(sim, n)
        t_end = periods * closed
        zeros = []
        c0 = c_prev = proj()
        t_prev, steps = 0.0, 0
        while sim.t < t_end:
            dt = min(sim.maxDt(), t_end - sim.t)
            if not dt > 0:
                break
            sim.step(dt)
            steps += 1
            t, c = sim.t, proj()
            if (c_prev < 0) != (c < 0):           # a sign change: interpolate the zero
                zeros.append(t_prev + (t - t_prev) * (0 - c_prev) / (c - c_prev))
            t_prev, c_prev = t, c
            if onProgress and steps % 200 == 0:
                onProgress(t / t_end)
    finally:
        sim.close()
    out = {"closed": closed, "steps": steps, "crossings": len(zeros), "amp0": c0, "ampEnd": c_prev}
    if len(zeros) < 2:
        out.update(measured=math.nan, rel=math.nan, note="fewer than two zero crossings: nothing to measure")
        return out
    measured = 2 * (zeros[-1] - zeros[0]) / (len(zeros) - 1)
    out.update(measured=measured, rel=(measured - closed) / closed, nx=nx, ny=ny, deg=deg,
               note=f"{len(zeros)} crossings, {steps} steps, amplitude {c0:.4f} -> {c_prev:.4f} m")
    return out
