"""Oracle for the waterbodies of src/gridlands.mjs:107-139 (test
infrastructure only; the product labels bodies on the device).

A breadth-first flood fill from each unvisited wet cell in row-major order:
the body's level is the surface at that first cell, its spread the largest
|surface - level| over its cells, its ring the dry 4-neighbours it touches,
ringMin the lowest bed on that ring.  Arithmetic in double on the float32
layers, as the reference's Float32Array reads are."""
from collections import deque
import math

import numpy as np


def flood_bodies(bed, srf, W, H):
    bed = np.asarray(bed, dtype=np.float32).reshape(-1).astype(np.float64).tolist()
    srf = np.asarray(srf, dtype=np.float32).reshape(-1).astype(np.float64).tolist()
    n = W * H
    wet = [srf[k] - bed[k] > 0 for k in range(n)]
    done = [False] * n
    bodies = []
    for start in range(n):
        if done[start] or not wet[start]:
            continue
        level = srf[start]
        members, ring = [], set()
        spread = 0.0
        todo = deque([start])
        done[start] = True
        while todo:
            k = todo.popleft()
            members.append(k)
            spread = max(spread, abs(srf[k] - level))
            r, c = divmod(k, W)
            for ok, m in ((c > 0, k - 1), (c < W - 1, k + 1), (r > 0, k - W), (r < H - 1, k + W)):
                if not ok:
                    continue
                if wet[m]:
                    if not done[m]:
                        done[m] = True
                        todo.append(m)
                else:
                    ring.add(m)
        ring_min = min((bed[m] for m in ring), default=math.inf)
        bodies.append({"level": level, "cells": sorted(members), "spread": spread, "ringMin": ring_min,
                       "perch": level - ring_min, "isOcean": level == 0})
    return bodies
