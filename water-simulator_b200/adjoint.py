"""Gauge-misfit gradients with respect to the bed and the Manning-n field.

    J = sum over steps, gauges of (b + h - obs)^2

for a ShallowWater-style run (Cartesian; walls unless `boundaries` says
otherwise) of `steps` self-timed steps from still water eta0.  `forward()` runs the step kernels, records the dt
sequence and keeps a checkpoint every `checkpoint_every` steps;
`backward()` returns dJ/db and dJ/dn over the padded grid from the
hand-written reverse of every step (swe_adjoint_* in include/swe_b200.h).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import BC_KIND, LIMITERS, SIDES, check, dptr


class MisfitAdjoint:
    def __init__(self, nx, ny, dx, b, eta0, manning=0.025, manning_field=None, gauges=(), steps=1,
                 checkpoint_every=45, minDepth=1e-3, cfl=0.45, order=2, limiter="mc", coriolis=0.0, dy=None,
                 boundaries=None):
        lib = _lib.load()
        self._lib = lib
        o = _lib.SweOptions()
        lib.swe_options_init(ctypes.byref(o))
        o.nx, o.ny, o.dx, o.dy = int(nx), int(ny), float(dx), float(dy if dy is not None else dx)
        o.manning, o.min_depth, o.cfl, o.order = float(manning), float(minDepth), float(cfl), int(order)
        o.limiter, o.coriolis = LIMITERS[limiter], float(coriolis)
        self.W, self.H = o.nx + 4, o.ny + 4
        N = self.W * self.H
        self.b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
        e = np.full(N, float(eta0)) if np.isscalar(eta0) else np.ascontiguousarray(eta0, dtype=np.float64).reshape(-1)
        self.eta0 = e
        self.nfield = None if manning_field is None else np.ascontiguousarray(manning_field, dtype=np.float64).reshape(-1)
        g = np.ascontiguousarray(gauges, dtype=np.int32)
        self.gauges, self.steps = g, int(steps)
        h = ctypes.c_void_p()
        check(lib.swe_adjoint_create(ctypes.byref(o), dptr(self.b), dptr(self.eta0),
                                     dptr(self.nfield) if self.nfield is not None else None, len(g),
                                     g.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), self.steps,
                                     int(checkpoint_every), ctypes.byref(h)))
        self._h = h
        self.set_observations(np.zeros((self.steps, len(g))))
        for side, bc in (boundaries or {}).items():
            self.set_boundary(side, bc)

    def set_boundary(self, side, bc):
        """side: "west", "east", "south" or "north"; bc: "reflect", "outflow",
        "periodic", ("flather", eta_ext, u_ext) with a constant exterior
        state, or ("tide", msl, amps, omegas, phases_deg, u_coef): Flather
        with the exterior state of a tide (src/swe.mjs:1026-1126,
        src/tide.mjs:103-107)."""
        s = SIDES[side]
        usage = "reflect, outflow, periodic, ('flather', eta, u) or ('tide', msl, amps, omegas, phases, u_coef)"
        if isinstance(bc, str):
            if bc not in ("reflect", "outflow", "periodic"):
                raise ValueError(f"boundary {bc!r}: {usage}")
            check(self._lib.swe_adjoint_set_boundary(self._h, s, BC_KIND[bc]))
        elif bc[0] == "flather" and len(bc) == 3:
            check(self._lib.swe_adjoint_set_flather_values(self._h, s, float(bc[1]), float(bc[2])))
        elif bc[0] == "tide" and len(bc) == 6:
            amp, om, ph = (np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in bc[2:5])
            if not (len(amp) == len(om) == len(ph)):
                raise ValueError("tide: amps, omegas and phases differ in length")
            check(self._lib.swe_adjoint_set_flather_tide(self._h, s, float(bc[1]), len(amp), dptr(amp), dptr(om),
                                                         dptr(ph), float(bc[5])))
        else:
            raise ValueError(f"boundary {bc!r}: {usage}")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.swe_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_observations(self, obs):
        o = np.ascontiguousarray(obs, dtype=np.float64).reshape(self.steps, len(self.gauges))
        check(self._lib.swe_adjoint_set_observations(self._h, dptr(o)))

    def forward(self):
        """Returns (J, eta at the gauges after every step)."""
        J = ctypes.c_double()
        eta = np.zeros((self.steps, len(self.gauges)))
        check(self._lib.swe_adjoint_forward(self._h, ctypes.byref(J), dptr(eta)))
        return J.value, eta

    def backward(self):
        """Returns (dJ/db, dJ/dn) over the padded grid (ghost entries 0)."""
        N = self.W * self.H
        gb, gn = np.zeros(N), np.zeros(N)
        check(self._lib.swe_adjoint_backward(self._h, dptr(gb), dptr(gn)))
        return gb, gn

    def dt_sequence(self, fixed=None):
        out = np.zeros(self.steps)
        inp = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.float64)
        check(self._lib.swe_adjoint_dt_sequence(self._h, dptr(out), dptr(inp) if inp is not None else None))
        return out

    def stream(self):
        p = ctypes.c_void_p()
        check(self._lib.swe_adjoint_get_stream(self._h, ctypes.byref(p)))
        return p.value
