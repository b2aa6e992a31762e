"""Ensemble: many independent basins advanced together on the GPU.

Each basin is a full ShallowWater (src/swe.mjs:145 of the reference) with its
own grid, bed, Manning n, boundaries and Flather tide, stepping with its own
dt = maxDt().  One ensemble step is a handful of kernel launches over a tile
list of all basins (swe_batch_* in include/swe_b200.h), captured as CUDA
graphs; the stage kernels and the tile schedule are chosen by `autotune`,
which times candidates on the ensemble itself and keeps the state unchanged.
"""
import ctypes
import json
import os

import numpy as np

from . import _lib
from ._lib import FIELD, SIDES, BC_KIND, LIMITERS, check, dptr
from .swe import _jmax0


class Ensemble:
    def __init__(self, basins, minDepth=1e-3, cfl=0.45, order=2, limiter="mc"):
        """basins: dicts with nx, ny, dx[, dy], b (padded array), eta0 (number
        or padded array), manning[, coriolis]."""
        lib = _lib.load()
        self._lib = lib
        n = len(basins)
        opts = (_lib.SweOptions * n)()
        self._keep = []
        bptr = (_lib._DP * n)()
        hptr = (_lib._DP * n)()
        self.dims = []
        for q, bs in enumerate(basins):
            o = opts[q]
            lib.swe_options_init(ctypes.byref(o))
            o.nx, o.ny = int(bs["nx"]), int(bs["ny"])
            o.dx = float(bs["dx"])
            o.dy = float(bs.get("dy", bs["dx"]))
            o.manning = float(bs.get("manning", 0.025))
            o.min_depth, o.cfl, o.order = minDepth, cfl, order
            o.coriolis = float(bs.get("coriolis", 0.0))
            o.limiter = LIMITERS[limiter]
            W, H = o.nx + 4, o.ny + 4
            b = np.ascontiguousarray(bs["b"], dtype=np.float64).reshape(-1)
            e = bs["eta0"]
            e = np.full(W * H, float(e)) if np.isscalar(e) else np.ascontiguousarray(e, dtype=np.float64).reshape(-1)
            h = _jmax0(e - b)
            self._keep += [b, h]
            bptr[q] = dptr(b)
            hptr[q] = dptr(h)
            self.dims.append((W, H))
        handle = ctypes.c_void_p()
        check(lib.swe_batch_create(n, opts, bptr, hptr, ctypes.byref(handle)))
        self._h = handle
        self.n = n
        self._keep = []
        for q, bs in enumerate(basins):
            if "tide" in bs:
                t = bs["tide"]
                self.set_tide(q, "west", t["msl"], t["amp"], t["omega"], t.get("phase_deg", [0] * len(t["amp"])),
                              t.get("u_coef", 0.0))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.swe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_boundary(self, basin, side, kind):
        check(self._lib.swe_batch_set_boundary(self._h, basin, SIDES[side], BC_KIND[kind]))

    def set_tide(self, basin, side, msl, amp, omega, phase_deg, u_coef=0.0):
        a, w, p = (np.ascontiguousarray(x, dtype=np.float64) for x in (amp, omega, phase_deg))
        check(self._lib.swe_batch_set_flather_tide(self._h, basin, SIDES[side], float(msl), len(a),
                                                   dptr(a), dptr(w), dptr(p), float(u_coef)))

    def run(self, steps):
        check(self._lib.swe_batch_run(self._h, int(steps)))

    def synchronize(self):
        """Wait for the ensemble; raises SweError (SWE_ETIMEOUT) when a
        work-queue wait ran past its limit since the last call."""
        check(self._lib.swe_batch_synchronize(self._h))

    @property
    def launch(self):
        """"queue": one persistent launch per step over a device work queue;
        "phases": a launch per phase of the step."""
        q = ctypes.c_int()
        check(self._lib.swe_batch_get_launch(self._h, ctypes.byref(q)))
        return "queue" if q.value else "phases"

    def set_launch(self, launch):
        check(self._lib.swe_batch_set_launch(self._h, {"phases": 0, "queue": 1}[launch]))

    def set_wait_limit(self, seconds):
        check(self._lib.swe_batch_set_wait_limit(self._h, float(seconds)))

    def debug_hold(self, basin=-1):
        """Test hook: never mark `basin`'s prepare done (-1: none)."""
        check(self._lib.swe_batch_debug_hold(self._h, int(basin)))

    def field(self, basin, name):
        W, H = self.dims[basin]
        out = np.zeros(W * H)
        check(self._lib.swe_batch_get_field(self._h, basin, FIELD[name], dptr(out)))
        return out

    def _scalar(self, basin, which):
        v = ctypes.c_double()
        check(self._lib.swe_batch_get_scalar(self._h, basin, _lib.SCALAR[which], ctypes.byref(v)))
        return v.value

    def t(self, basin):
        return self._scalar(basin, "t")

    def steps(self, basin):
        return int(self._scalar(basin, "steps"))

    @property
    def schedule(self):
        s = (ctypes.c_int * 4)()
        check(self._lib.swe_batch_get_schedule(self._h, s))
        return {"rows": s[0], "ctas": s[1], "order": s[2], "tiles": s[3]}

    def set_schedule(self, rows=0, ctas=0, order=0):
        """rows 0: the tiled stage pair (32 x 8 tiles); 4..64: fused row-marching
        tiles of that many rows.  ctas 0: one CTA per tile, else a persistent
        grid.  order 0 basin-major, 1 largest basin first, 2 round robin."""
        check(self._lib.swe_batch_set_schedule(self._h, int(rows), int(ctas), int(order)))

    def autotune(self, trial_steps=3, cache=None, key=None):
        """Choose the tile schedule by timing candidates (the state is kept).
        With `cache` (a JSON path) and `key`, a stored choice is reused."""
        if cache and key and os.path.exists(cache):
            with open(cache) as f:
                d = json.load(f)
            if key in d:
                self.set_schedule(**{k: d[key][k] for k in ("rows", "ctas", "order")})
                self.set_launch(d[key].get("launch", "phases"))
                return dict(d[key], cached=True)
        best = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        check(self._lib.swe_batch_autotune(self._h, int(trial_steps), best, ctypes.byref(ms)))
        res = {"rows": best[0], "ctas": best[1], "order": best[2], "tiles": best[3], "ms_per_step": ms.value,
               "launch": self.launch}
        if cache and key:
            d = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    d = json.load(f)
            d[key] = res
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(d, f, indent=1)
        return res

    def stream(self):
        p = ctypes.c_void_p()
        check(self._lib.swe_batch_get_stream(self._h, ctypes.byref(p)))
        return p.value
