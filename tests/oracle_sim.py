"""Test-side Python wrapper of the CPU oracle (oracle/liboracle_swe.so).

TEST INFRASTRUCTURE: the checker the GPU library is compared with.  The
oracle restates src/swe.mjs + src/geometry.mjs of the reference in C++; this
wrapper gives it the same Python surface as water_simulator_b200.ShallowWater
(the reference's names), with the fields as numpy views onto the oracle's
own arrays, so tests can drive both the same way.
"""
import ctypes
import math
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle_swe.so")

_FIELDS = {"b": 0, "h": 1, "hu": 2, "hv": 3, "h0": 4, "hu0": 5, "hv0": 6, "rh": 7, "rhu": 8,
           "rhv": 9, "theta": 10, "manning": 11, "uu": 12, "vv": 13}
_GEOM = ["dxRow", "dyRowN", "dyRowS", "dyCFL", "area", "lx", "lyN", "lyS", "bedPhi", "phiC",
         "tanPhi", "fRow", "geoCoef"]
_SIDES = {"west": 0, "east": 1, "south": 2, "north": 3}
_LIM = {"mc": 0, "minmod": 1, "central": 2}


class OracleOptions(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("manning", ctypes.c_double), ("min_depth", ctypes.c_double),
                ("cfl", ctypes.c_double), ("coriolis", ctypes.c_double),
                ("order", ctypes.c_int), ("limiter", ctypes.c_int), ("sphere", ctypes.c_int),
                ("R", ctypes.c_double), ("lat0", ctypes.c_double), ("lat1", ctypes.c_double),
                ("omega", ctypes.c_double)]


_lib = None


def oracle_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            import subprocess
            subprocess.run(["python", os.path.join(ROOT, "oracle", "build.py")], check=True)
        lib = ctypes.CDLL(ORACLE_LIB)
        D, I, P, DP = ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        sig = {
            "oracle_create": ([ctypes.POINTER(OracleOptions), DP, DP, ctypes.POINTER(P)], I),
            "oracle_destroy": ([P], None),
            "oracle_last_error": ([], ctypes.c_char_p),
            "oracle_field": ([P, I], DP),
            "oracle_geom": ([P, I], DP),
            "oracle_get_scalar": ([P, I], D),
            "oracle_set_scalar": ([P, I, D], None),
            "oracle_set_threads": ([P, I], None),
            "oracle_set_boundary": ([P, I, I], I),
            "oracle_set_flather_values": ([P, I, D, D], I),
            "oracle_set_flather_tide": ([P, I, D, I, DP, DP, DP, D], I),
            "oracle_set_manning_field": ([P, DP], I),
            "oracle_set_sponge": ([P, I, I, D, D], I),
            "oracle_clear_sponge": ([P], I),
            "oracle_apply_bc": ([P], None),
            "oracle_residual": ([P, D], None),
            "oracle_max_dt": ([P], D),
            "oracle_apply_friction": ([P, D], None),
            "oracle_dry_clean": ([P], D),
            "oracle_step": ([P, D], D),
            "oracle_step_auto": ([P], D),
            "oracle_volume": ([P], D),
            "oracle_energy": ([P], D),
            "oracle_max_surface_deviation": ([P, D], D),
            "oracle_max_speed": ([P], D),
            "oracle_finite": ([P], I),
            "oracle_vel": ([P, D, D], D),
            "oracle_hllc": ([DP, D, D, D, D, D, D, D], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _jmax0(d):
    d = np.asarray(d, dtype=np.float64)
    return np.where(d > 0, d, np.where(np.isnan(d), d, 0.0))


def oracle_hllc(hL, huL, hvL, hR, huR, hvR, dry=1e-4):
    out = np.zeros(3)
    oracle_lib().oracle_hllc(_dp(out), hL, huL, hvL, hR, huR, hvR, dry)
    return out


class _Geom:
    def __init__(self, sim):
        self._sim = sim
        self.kind = "sphere" if sim._sphere else "cartesian"
        self.nx, self.ny, self.ng, self.H = sim.nx, sim.ny, 2, sim.H
        g = oracle_lib().oracle_get_scalar
        self.dx, self.dy, self.R = g(sim._p, 0), g(sim._p, 1), g(sim._p, 2)
        self.dlam, self.dphi, self.totalArea = g(sim._p, 3), g(sim._p, 4), g(sim._p, 5)

    def __getattr__(self, name):
        if name in _GEOM:
            ptr = oracle_lib().oracle_geom(self._sim._p, _GEOM.index(name))
            return np.ctypeslib.as_array(ptr, shape=(self._sim.H,))
        raise AttributeError(name)


class OracleSim:
    def __init__(self, nx, ny, dx=None, dy=None, bed=None, eta0=0, manning=0.025, minDepth=1e-3,
                 cfl=0.45, coriolis=0, order=2, limiter="mc", sphere=None, threads=1):
        lib = oracle_lib()
        o = OracleOptions()
        o.nx, o.ny = nx, ny
        o.dx = float(dx) if dx is not None else float("nan")
        o.dy = float(dy if dy is not None else (dx if dx is not None else float("nan")))
        o.manning, o.min_depth, o.cfl, o.coriolis = manning, minDepth, cfl, coriolis
        o.order, o.limiter = order, _LIM.get(limiter, -1)
        o.R, o.lat0, o.lat1, o.omega = 6371e3, -90.0, 90.0, 0.0
        self._sphere = bool(sphere)
        if sphere:
            o.sphere = 1
            o.R = float(sphere.get("R", 6371e3))
            o.lat0, o.lat1 = float(sphere.get("lat0", -90)), float(sphere.get("lat1", 90))
            o.omega = float(sphere.get("omega", 0))
        self.nx, self.ny, self.ng, self.W, self.H = nx, ny, 2, nx + 4, ny + 4
        self.N = self.W * self.H
        self.minDepth, self.cfl, self.manning = minDepth, cfl, manning
        p = ctypes.c_void_p()
        zero = np.zeros(self.N)
        if lib.oracle_create(ctypes.byref(o), _dp(zero), _dp(zero), ctypes.byref(p)) != 0:
            raise ValueError(lib.oracle_last_error().decode())
        self._p = p
        self.geom = _Geom(self)
        self.dx = None if sphere else dx
        self.dy = self.geom.dy if sphere else (dy if dy is not None else dx)
        lib.oracle_set_threads(p, threads)
        shape = (self.H, self.W)
        b = self._sample(bed if bed is not None else 0.0, shape)
        e = self._sample(eta0, shape)
        self.b[:] = b.reshape(-1)
        self.h[:] = _jmax0(e - b).reshape(-1)
        self._flather = {}
        self.forcing = None

    def _sample(self, fn, shape):
        if isinstance(fn, np.ndarray):
            return np.ascontiguousarray(fn, dtype=np.float64).reshape(shape).copy()
        if not callable(fn):
            return np.full(shape, float(fn))
        out = np.empty(shape)
        for j in range(shape[0]):
            for i in range(shape[1]):
                x, y = (self.cellLonLat(i - 2, j - 2) if self._sphere else self.cellCentre(i - 2, j - 2))
                out[j, i] = fn(x, y)
        return out

    def close(self):
        if getattr(self, "_p", None) is not None and self._p.value:
            oracle_lib().oracle_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # coordinates
    def cellCentre(self, i, j):
        return [(i + 0.5) * self.dx, (j + 0.5) * self.dy]

    def cellLonLat(self, i, j):
        lon = (i + 0.5) * self.geom.dlam * 180 / math.pi
        return [math.fmod(math.fmod(lon, 360) + 360, 360) - 180, self.geom.phiC[j + 2] * 180 / math.pi]

    def idx(self, i, j):
        return (j + 2) * self.W + (i + 2)

    def eta(self, i, j):
        k = self.idx(i, j)
        return float(self.b[k] + self.h[k])

    def depth(self, i, j):
        return float(self.h[self.idx(i, j)])

    def vel(self, hq, h):
        return oracle_lib().oracle_vel(self._p, hq, h)

    def _arr(self, name):
        ptr = oracle_lib().oracle_field(self._p, _FIELDS[name])
        if not ptr:
            return None
        return np.ctypeslib.as_array(ptr, shape=(self.N,))

    b = property(lambda s: s._arr("b"))
    h = property(lambda s: s._arr("h"))
    hu = property(lambda s: s._arr("hu"))
    hv = property(lambda s: s._arr("hv"))
    h0 = property(lambda s: s._arr("h0"))
    hu0 = property(lambda s: s._arr("hu0"))
    hv0 = property(lambda s: s._arr("hv0"))
    rh = property(lambda s: s._arr("rh"))
    rhu = property(lambda s: s._arr("rhu"))
    rhv = property(lambda s: s._arr("rhv"))
    theta = property(lambda s: s._arr("theta"))

    def field(self, name):
        return self._arr(name).copy()

    t = property(lambda s: oracle_lib().oracle_get_scalar(s._p, 6),
                 lambda s, v: oracle_lib().oracle_set_scalar(s._p, 6, v))
    steps = property(lambda s: int(oracle_lib().oracle_get_scalar(s._p, 7)))
    massFloored = property(lambda s: oracle_lib().oracle_get_scalar(s._p, 8))

    def set_boundaries(self, **kinds):
        """kinds: side -> 'reflect'|'outflow'|'periodic'|('flather', eta, u)|('tide', msl, amp, omega, phase, ucoef)."""
        lib = oracle_lib()
        for side, k in kinds.items():
            s = _SIDES[side]
            if isinstance(k, str):
                lib.oracle_set_boundary(self._p, s, {"reflect": 0, "outflow": 1, "periodic": 2}[k])
                self._flather.pop(side, None)
            elif k[0] == "flather":
                self._flather[side] = (k[1], k[2])
                lib.oracle_set_flather_values(self._p, s, 0.0, 0.0)
            elif k[0] == "tide":
                msl, amp, om, ph, uc = k[1:]
                amp, om, ph = (np.ascontiguousarray(x, dtype=np.float64) for x in (amp, om, ph))
                lib.oracle_set_flather_tide(self._p, s, msl, len(amp), _dp(amp), _dp(om), _dp(ph), uc)
                self._flather.pop(side, None)

    def _prep_flather(self):
        for side, (fe, fu) in self._flather.items():
            t = self.t
            oracle_lib().oracle_set_flather_values(self._p, _SIDES[side], float(fe(t)), float(fu(t)))

    def setManningField(self, n):
        if n is None:
            oracle_lib().oracle_set_manning_field(self._p, None)
            return self
        n = np.ascontiguousarray(n, dtype=np.float64).reshape(-1)
        if oracle_lib().oracle_set_manning_field(self._p, _dp(n)) != 0:
            raise ValueError(oracle_lib().oracle_last_error().decode())
        return self

    def setSponge(self, side="east", width=20, strength=0.06, etaRef=0.0):
        oracle_lib().oracle_set_sponge(self._p, _SIDES[side], int(width), float(strength), float(etaRef))

    def applyBC(self):
        self._prep_flather()
        oracle_lib().oracle_apply_bc(self._p)

    def residual(self, dt):
        oracle_lib().oracle_residual(self._p, dt)

    def maxDt(self):
        return oracle_lib().oracle_max_dt(self._p)

    def applyFriction(self, dt):
        oracle_lib().oracle_apply_friction(self._p, dt)

    def dryClean(self):
        return oracle_lib().oracle_dry_clean(self._p)

    def step(self, dt=None):
        self._prep_flather()
        if dt is None:
            return oracle_lib().oracle_step_auto(self._p)
        t0 = self.t
        taken = oracle_lib().oracle_step(self._p, dt)
        if taken and self.forcing is not None:
            self.forcing(self, taken, t0)
        return taken

    def volume(self):
        return oracle_lib().oracle_volume(self._p)

    def energy(self):
        return oracle_lib().oracle_energy(self._p)

    def maxSurfaceDeviation(self, ref):
        return oracle_lib().oracle_max_surface_deviation(self._p, ref)

    def maxSpeed(self):
        return oracle_lib().oracle_max_speed(self._p)

    def finite(self):
        return bool(oracle_lib().oracle_finite(self._p))
