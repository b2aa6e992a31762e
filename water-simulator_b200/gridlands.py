"""Terrain exported by gridlands (format `gridlands-terrain` v1), src/gridlands.mjs.

A document carries width x height float32 layers -- bedM, surfaceM and an
optional per-cell manningN -- little-endian and base64-encoded, row 0 north.
`gridlandsTerrain(doc)` checks the document, decodes the layers on the device
(swe_gridlands_decode) and returns the terrain: its `bed(x, y)` (bilinear,
clamped) and `eta0(x, y)` (nearest) sampling functions, the decoded arrays
and the provenance.  Handing `t.bed` and `t.eta0` to `ShallowWater` builds
the fields on the device from the layers (swe_gridlands_create) instead of
calling the functions cell by cell; the values are the same doubles.
`waterbodies`, `verifyInvariants` and `settleLakes` are the host-side checks
and the opt-in repair of src/gridlands.mjs:108-220.
"""
import ctypes
import math
import sys

import numpy as np

from . import _lib
from ._lib import check

LITTLE_ENDIAN = sys.byteorder == "little"


def _js_round(x):
    """Math.round: nearest integer, ties towards +Infinity."""
    f = math.floor(x)
    return f + 1 if x - f >= 0.5 else f


def decodeF32(layer, n, name):
    """src/gridlands.mjs:82-98: a b64f32le layer to exactly n float32 values,
    decoded on the device."""
    if not layer:
        raise ValueError(f"gridlands: layer {name} is missing")
    if layer.get("encoding") != "b64f32le":
        raise ValueError(f"gridlands: layer {name} has encoding {layer.get('encoding')}, expected b64f32le")
    if not LITTLE_ENDIAN:
        raise ValueError("gridlands: b64f32le needs a little-endian host; this one is big-endian.")
    data = layer.get("data") or ""
    raw = data.encode("ascii") if isinstance(data, str) else bytes(data)
    out = np.empty(n, dtype=np.float32)
    rc = _lib.load().swe_gridlands_decode(raw, len(raw), int(n), out.ctypes.data_as(ctypes.c_void_p))
    if rc != _lib.SWE_OK:
        msg = _lib.load().swe_last_error().decode()
        raise ValueError(msg.replace("layer data", f"layer {name}"))
    return out


def waterbodies(bedM, surfaceM, W, H):
    """src/gridlands.mjs:108-139: 4-connected wet bodies with the lowest bed on
    each one's boundary ring (its spill level)."""
    bed = np.asarray(bedM).tolist()
    srf = np.asarray(surfaceM).tolist()
    n = W * H
    seen = bytearray(n)
    out = []
    for k0 in range(n):
        if seen[k0] or not (srf[k0] - bed[k0] > 0):
            continue
        level = srf[k0]
        cells, ring, spread = [], set(), 0.0
        stack = [k0]
        seen[k0] = 1
        while stack:
            k = stack.pop()
            cells.append(k)
            if srf[k] != level:
                spread = max(spread, abs(srf[k] - level))
            c = k % W
            r = (k - c) // W
            nb = []
            if c > 0:
                nb.append(k - 1)
            if c < W - 1:
                nb.append(k + 1)
            if r > 0:
                nb.append(k - W)
            if r < H - 1:
                nb.append(k + W)
            for m in nb:
                if srf[m] - bed[m] > 0:
                    if not seen[m]:
                        seen[m] = 1
                        stack.append(m)
                else:
                    ring.add(m)
        ringMin = math.inf
        for m in ring:
            ringMin = min(ringMin, bed[m])
        out.append({"level": level, "cells": cells, "spread": spread, "ringMin": ringMin,
                    "perch": level - ringMin, "isOcean": level == 0})
    return out


def verifyInvariants(t):
    """src/gridlands.mjs:157-195: the exporter's guarantees re-derived from the
    decoded arrays, plus the one the solver needs (no lake above its spill)."""
    bedM, surfaceM, W, H = t.bedM, t.surfaceM, t.W, t.H
    d = surfaceM.astype(np.float64) - bedM.astype(np.float64)
    below = int(np.count_nonzero(d < 0))
    worstBelow = float(min(0.0, d.min())) if d.size else 0.0
    wet = int(np.count_nonzero(d > 0))
    oceanCells = int(np.count_nonzero((surfaceM == 0) & (bedM < 0)))
    bodies = waterbodies(bedM, surfaceM, W, H)
    lakes = [b for b in bodies if not b["isOcean"]]
    notFlat = [b for b in bodies if b["spread"] > 0]
    perched = sorted([b for b in lakes if b["perch"] > 1e-6], key=lambda b: -b["perch"])
    perchedVolume = 0.0
    for b in perched:
        perchedVolume += len(b["cells"]) * b["perch"]
    ocean = [b["perch"] for b in bodies if b["isOcean"]]
    return {
        "cells": W * H, "wet": wet, "oceanCells": oceanCells,
        "surfaceBelowBed": below, "worstBelowBed": worstBelow, "dryMismatch": 0,
        "bodies": len(bodies), "lakeBodies": len(lakes), "lakesNotFlat": len(notFlat),
        "worstLakeSpread": max([b["spread"] for b in notFlat], default=0),
        "largestBody": max([len(b["cells"]) for b in bodies], default=0),
        "perchedLakes": len(perched), "worstPerch": perched[0]["perch"] if perched else 0,
        "perchedCells": sum(len(b["cells"]) for b in perched),
        "perchedVolumeCells": perchedVolume,
        "worstOceanPerch": max(ocean, default=-math.inf),
    }


def settleLakes(bedM, surfaceM, W, H):
    """src/gridlands.mjs:209-219: lower every perched body to its spill level,
    in place (float32, as the reference's Float32Array), and report it."""
    bodies = waterbodies(bedM, surfaceM, W, H)
    moved = []
    for b in bodies:
        if not (b["perch"] > 1e-6):
            continue
        to = b["ringMin"]
        for k in b["cells"]:
            surfaceM[k] = max(float(bedM[k]), to)
        moved.append({"from": b["level"], "to": to, "drop": b["perch"], "cells": len(b["cells"])})
    return {"bodiesMoved": len(moved), "worstDrop": max([m["drop"] for m in moved], default=0), "moved": moved}


class GridlandsTerrain:
    """What gridlandsTerrain() returns (src/gridlands.mjs:293-309)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def __getitem__(self, k):
        return getattr(self, k)


def gridlandsTerrain(doc, flipRows=True, settle=False):
    """src/gridlands.mjs:228-305."""
    if not isinstance(doc, dict):
        raise ValueError("gridlands: not a document")
    if doc.get("format") != "gridlands-terrain" or doc.get("version") != 1:
        raise ValueError(f"gridlands: unsupported terrain {doc.get('format')} v{doc.get('version')}; "
                         "this adapter reads gridlands-terrain v1.")
    g = doc.get("grid") or {}
    W, H, C = g.get("width"), g.get("height"), g.get("cellMeters")
    if not (isinstance(W, (int, float)) and isinstance(H, (int, float)) and isinstance(C, (int, float))
            and W > 0 and H > 0 and C > 0):
        raise ValueError(f"gridlands: bad grid {g}")
    if g.get("rowOrder") and g["rowOrder"] != "north-first":
        raise ValueError(f"gridlands: rowOrder is {g['rowOrder']}; this adapter assumes north-first")
    W, H = int(W), int(H)
    n = W * H
    layers = doc.get("layers") or {}
    bedM = decodeF32(layers.get("bedM"), n, "bedM")
    surfaceM = decodeF32(layers.get("surfaceM"), n, "surfaceM")
    manningN = decodeF32(layers["manningN"], n, "manningN") if layers.get("manningN") else None
    settled = settleLakes(bedM, surfaceM, W, H) if settle else None

    if flipRows:
        def rowOf(y):
            return (H - 1) - min(H - 1, max(0, y / C - 0.5))
    else:
        def rowOf(y):
            return min(H - 1, max(0, y / C - 0.5))

    def colOf(x):
        return min(W - 1, max(0, x / C - 0.5))

    bl, sl = bedM.tolist(), surfaceM.tolist()

    def bed(x, y):
        fc, fr = colOf(x), rowOf(y)
        c0, r0 = math.floor(fc), math.floor(fr)
        c1, r1 = min(W - 1, c0 + 1), min(H - 1, r0 + 1)
        tc, tr = fc - c0, fr - r0
        v00, v10 = bl[r0 * W + c0], bl[r0 * W + c1]
        v01, v11 = bl[r1 * W + c0], bl[r1 * W + c1]
        return (v00 * (1 - tc) + v10 * tc) * (1 - tr) + (v01 * (1 - tc) + v11 * tc) * tr

    def eta0(x, y):
        return sl[int(_js_round(rowOf(y))) * W + int(_js_round(colOf(x)))]

    meta = doc.get("meta") or {}
    stats = doc.get("stats") or {}
    sug = stats.get("suggestedManningScalar")
    t = GridlandsTerrain(
        bed=bed, eta0=eta0,
        domain={"nx": W, "ny": H, "dx": C, "dy": C},
        manning=sug if sug is not None else 0.03,
        manningN=manningN, bedM=bedM, surfaceM=surfaceM, W=W, H=H, cellMeters=C,
        settled=settled, stats=stats, meta=meta, flipRows=bool(flipRows),
        label=f"gridlands {meta.get('preset')}/{meta.get('seed')} #{meta.get('mapId')}",
        provenance={"tool": meta.get("tool"), "mapId": meta.get("mapId"), "preset": meta.get("preset"),
                    "seed": meta.get("seed"), "spec": meta.get("spec"), "format": doc.get("format"),
                    "version": doc.get("version"),
                    "grid": f"{W}x{H} @ {C} m = {W * C / 1000:.1f} x {H * C / 1000:.1f} km"},
        shortestHonestWavelength=40 * C,
        _layers=layers, _settled=bool(settle))

    def manningAt(x, y):
        """The per-cell Manning sampler of tools/verify-gridlands.mjs:330-331."""
        return float(manningN[int(_js_round(rowOf(y))) * W + int(_js_round(colOf(x)))])

    bed._gridlands = t
    eta0._gridlands = t
    manningAt._gridlands = t
    t.manningAt = manningAt if manningN is not None else None
    return t


def loadGridlandsTerrain(text, **opts):
    """Parse + adapt in one call (src/gridlands.mjs:308-310)."""
    import json
    return gridlandsTerrain(json.loads(text) if isinstance(text, (str, bytes)) else text, **opts)


def _create_args(t, manning_field):
    """The swe_gridlands struct for a terrain: the layers as base64 text (decoded
    on the device), except a surface settled on the host, which goes as floats."""
    g = _lib.SweGridlands()
    g.width, g.height, g.cell_m, g.flip_rows = t.W, t.H, float(t.cellMeters), 1 if t.flipRows else 0
    keep = []

    def text(name):
        d = t._layers[name]["data"]
        raw = d.encode("ascii") if isinstance(d, str) else bytes(d)
        keep.append(raw)
        return raw, len(raw)

    g.bed_b64, g.bed_len = text("bedM")
    if t._settled:
        s = np.ascontiguousarray(t.surfaceM, dtype=np.float32)
        keep.append(s)
        g.surface_f32 = s.ctypes.data
    else:
        g.surface_b64, g.surface_len = text("surfaceM")
    if manning_field:
        g.manning_b64, g.manning_len = text("manningN")
        g.manning_field = 1
    return g, keep


def create_sim_handle(opts, t, manning_field=False):
    """swe_gridlands_create for a terrain; returns the handle."""
    g, keep = _create_args(t, manning_field)
    h = ctypes.c_void_p()
    check(_lib.load().swe_gridlands_create(ctypes.byref(opts), ctypes.byref(g), ctypes.byref(h)))
    del keep
    return h
