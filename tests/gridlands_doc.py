"""A seeded synthetic `gridlands-terrain` v1 document for the import tests.

The real export the reference's suite reads (a 200 x 150 map at 50 m) is not
available, so this builds a document of the same format: float32 layers,
little-endian, base64, row 0 north.  The map has a sea in the south (bed
below 0, surface exactly 0), dry land whose surface equals its bed, one lake
seated below its rim and one perched 2 m above its spill level (the defect
the reference's gate reports), and a Manning layer of three ground classes.
North and south rows differ, so a dropped row flip is detectable.
"""
import base64
import math

import numpy as np


def b64(a):
    return base64.b64encode(np.ascontiguousarray(a, dtype="<f4").tobytes()).decode("ascii")


def terrain_arrays(W=64, H=48, C=50.0, seed=7):
    rng = np.random.default_rng(seed)
    r = np.arange(H)[:, None].astype(np.float64)        # row 0 = north
    c = np.arange(W)[None, :].astype(np.float64)
    bed = 60.0 - 110.0 * (r / (H - 1)) ** 1.5 + 6.0 * np.sin(2 * math.pi * c / 23.0 + 0.7) \
        + 4.0 * np.cos(2 * math.pi * r / 17.0) + rng.uniform(-0.5, 0.5, (H, W))
    # seated lake: a bowl with its rim at 40 m, water at 38.5 m
    d2 = (r - 10) ** 2 + (c - 16) ** 2
    bowl = d2 <= 36
    bed = np.where(bowl, 40.0 - 12.0 * (1 - d2 / 36.0), bed)
    bed = np.where((d2 > 36) & (d2 <= 64), np.maximum(bed, 40.0), bed)
    # perched lake: a bowl whose rim ring sits at 30 m, water at 32 m
    d2b = (r - 14) ** 2 + (c - 46) ** 2
    bowl2 = d2b <= 25
    bed = np.where(bowl2, 30.0 - 8.0 * (1 - d2b / 25.0), bed)
    bed = np.where((d2b > 25) & (d2b <= 49), 30.0, bed)
    surface = bed.copy()                                # dry land: surface == bed
    surface = np.where(bowl & (bed < 38.5), 38.5, surface)
    surface = np.where(bowl2, 32.0, surface)
    # sea: every cell below 0 is sea at level 0
    sea = bed < 0
    surface = np.where(sea, 0.0, surface)
    bed32, surf32 = bed.astype(np.float32), surface.astype(np.float32)
    surf32 = np.where(surf32 < bed32, bed32, surf32)
    wet = surf32 > bed32
    n = np.where(wet, 0.02, np.where(bed32 < 20, 0.035, 0.1)).astype(np.float32)
    return bed32, surf32, n


def make_doc(W=64, H=48, C=50.0, seed=7, with_manning=True):
    bed, surf, n = terrain_arrays(W, H, C, seed)
    layers = {"bedM": {"encoding": "b64f32le", "data": b64(bed)},
              "surfaceM": {"encoding": "b64f32le", "data": b64(surf)}}
    if with_manning:
        layers["manningN"] = {"encoding": "b64f32le", "data": b64(n)}
    return {
        "format": "gridlands-terrain", "version": 1,
        "grid": {"width": W, "height": H, "cellMeters": C, "rowOrder": "north-first"},
        "layers": layers,
        "stats": {"suggestedManningScalar": 0.035},
        "meta": {"tool": "gridlands", "mapId": f"synthetic-{seed}", "preset": "continent", "seed": seed,
                 "spec": "gridlands docs/TERRAIN-FORMAT.md"},
    }
