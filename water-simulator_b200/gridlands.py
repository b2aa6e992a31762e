"""Terrain exported by gridlands (format `gridlands-terrain` v1), src/gridlands.mjs.

A document carries width x height float32 layers -- bedM, surfaceM and an
optional per-cell manningN -- little-endian and base64-encoded, row 0 north.
`gridlandsTerrain(doc)` checks the document, decodes the layers on the device
(swe_gridlands_decode) and returns the terrain: its `bed(x, y)` (bilinear,
clamped) and `eta0(x, y)` (nearest) sampling functions, the decoded arrays
and the provenance.  Handing `t.bed` and `t.eta0` to `ShallowWater` builds
the fields on the device from the layers (swe_gridlands_create) instead of
calling the functions cell by cell; the values are the same doubles.
`waterbodies` labels the wet bodies with a connected-components pass on the
device (swe_gridlands_bodies); `verifyInvariants` and the opt-in
`settleLakes` repair build on it (src/gridlands.mjs:107-220).
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


def body_labels(bedM, surfaceM, W, H):
    """Each cell's waterbody, from the device's connected-components pass
    (swe_gridlands_bodies): the lowest cell index of the cell's 4-connected
    wet body (surface - bed > 0), -1 for a dry cell."""
    bed = np.ascontiguousarray(bedM, dtype=np.float32).reshape(-1)
    srf = np.ascontiguousarray(surfaceM, dtype=np.float32).reshape(-1)
    n = int(W) * int(H)
    if bed.size != n or srf.size != n:
        raise ValueError(f"gridlands: layers of {bed.size} and {srf.size} cells for a {W}x{H} grid")
    label = np.empty(n, dtype=np.int32)
    check(_lib.load().swe_gridlands_bodies(int(W), int(H), bed.ctypes.data, srf.ctypes.data, label.ctypes.data))
    return label


def waterbodies(bedM, surfaceM, W, H):
    """The connected wet bodies with the lowest bed on each one's boundary
    ring, its spill level (src/gridlands.mjs:107-139).

    The bodies come from the device pass and are listed by their lowest cell
    (the reference's scan order), each with its surface level at that cell,
    its cells (ascending), the largest departure of its surface from that
    level (spread), the lowest bed among the dry cells that touch it
    (ringMin, Infinity if none), perch = level - ringMin and isOcean
    (level 0).  The per-body reductions run over whole arrays at once."""
    bed = np.asarray(bedM, dtype=np.float32).reshape(-1).astype(np.float64)
    srf = np.asarray(surfaceM, dtype=np.float32).reshape(-1).astype(np.float64)
    W, H = int(W), int(H)
    label = body_labels(bedM, surfaceM, W, H)
    wet = label >= 0
    roots = np.flatnonzero(wet & (label == np.arange(label.size)))      # ascending = scan order
    if roots.size == 0:
        return []
    body = np.full(label.size, -1, dtype=np.int64)                     # cell -> body number
    index = np.full(label.size, -1, dtype=np.int64)
    index[roots] = np.arange(roots.size)
    body[wet] = index[label[wet]]
    level = srf[roots]
    spread = np.zeros(roots.size)
    np.maximum.at(spread, body[wet], np.abs(srf[wet] - level[body[wet]]))
    # the ring: dry 4-neighbours of a body's cells, each pair seen from the wet side
    ring = np.full(roots.size, np.inf)
    grid = np.arange(label.size).reshape(H, W)
    for a, b in ((grid[:, :-1], grid[:, 1:]), (grid[:-1, :], grid[1:, :])):
        a, b = a.reshape(-1), b.reshape(-1)
        for inner, outer in ((a, b), (b, a)):
            edge = wet[inner] & ~wet[outer]
            np.minimum.at(ring, body[inner[edge]], bed[outer[edge]])
    order = np.argsort(body[wet], kind="stable")
    cells = np.split(np.flatnonzero(wet)[order], np.cumsum(np.bincount(body[wet], minlength=roots.size))[:-1])
    return [{"level": float(level[q]), "cells": cells[q], "spread": float(spread[q]), "ringMin": float(ring[q]),
             "perch": float(level[q] - ring[q]), "isOcean": bool(level[q] == 0)} for q in range(roots.size)]


def verifyInvariants(t):
    """The exporter's guarantees re-derived from the decoded arrays, and the
    one the solver needs besides: no lake above its spill level
    (src/gridlands.mjs:141-195).  A report; nothing is raised."""
    bedM, surfaceM, W, H = t.bedM, t.surfaceM, t.W, t.H
    b = np.asarray(bedM, dtype=np.float64).reshape(-1)
    s = np.asarray(surfaceM, dtype=np.float64).reshape(-1)
    d = s - b
    bodies = waterbodies(bedM, surfaceM, W, H)
    lakes = [x for x in bodies if not x["isOcean"]]
    uneven = [x["spread"] for x in bodies if x["spread"] > 0]
    perched = sorted((x for x in lakes if x["perch"] > 1e-6), key=lambda x: -x["perch"])
    volume = 0.0
    for x in perched:                            # summed in the report's order
        volume += len(x["cells"]) * x["perch"]
    sizes = [len(x["cells"]) for x in bodies]
    ocean = [x["perch"] for x in bodies if x["isOcean"]]
    return {
        "cells": int(W) * int(H), "wet": int(np.count_nonzero(d > 0)),
        "oceanCells": int(np.count_nonzero((s == 0) & (b < 0))),
        "surfaceBelowBed": int(np.count_nonzero(d < 0)), "worstBelowBed": float(min(0.0, d.min(initial=0.0))),
        "dryMismatch": 0,
        "bodies": len(bodies), "lakeBodies": len(lakes), "lakesNotFlat": len(uneven),
        "worstLakeSpread": max(uneven, default=0), "largestBody": max(sizes, default=0),
        "perchedLakes": len(perched), "worstPerch": perched[0]["perch"] if perched else 0,
        "perchedCells": sum(len(x["cells"]) for x in perched), "perchedVolumeCells": volume,
        "worstOceanPerch": max(ocean, default=-math.inf),
    }


def settleLakes(bedM, surfaceM, W, H):
    """Lower every perched body to its spill level in place (cells left above
    it become dry) and report what moved (src/gridlands.mjs:197-220).  Opt-in:
    a repair on this side, never applied unasked."""
    moved = []
    flat = surfaceM.reshape(-1)
    bed = np.asarray(bedM).reshape(-1)
    for x in waterbodies(bedM, surfaceM, W, H):
        if not (x["perch"] > 1e-6):
            continue
        k = x["cells"]
        flat[k] = np.maximum(bed[k].astype(np.float64), x["ringMin"])
        moved.append({"from": x["level"], "to": x["ringMin"], "drop": x["perch"], "cells": len(k)})
    return {"bodiesMoved": len(moved), "worstDrop": max((m["drop"] for m in moved), default=0), "moved": moved}


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
