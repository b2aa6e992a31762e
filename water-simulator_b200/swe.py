"""ShallowWater: the reference's JavaScript solver API over libswe_b200.so.

Mirrors `ShallowWater` of src/swe.mjs (Syntaxswine/water-simulator): the same
constructor options, fields and methods, with the reference's names, so code
written against the reference reads the same here.  Every field update runs
on the GPU through the C ABI; this module only samples the user's bed/eta0
callbacks on the host (as the reference's constructor does,
src/swe.mjs:222-232), keeps numpy mirrors of the fields coherent with the
device, and maps the built-in boundary functions onto device boundary kinds.

Field coherence: `sim.h`, `sim.hu`, `sim.hv`, `sim.b` (and the others) return
a numpy array refreshed from the device.  Because the caller may write into
it (tests do `sim.h[k] = ...`), a field handed out is uploaded again before
the next device call.  Re-read `sim.h` after a device call rather than
holding an old array.  `sim.field(name)` returns a read-only snapshot that is
never uploaded back.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import FIELD, GEOM_ROWS, SCALAR, SIDES, BC_KIND, LIMITERS, check, dptr

G = 9.80665                      # src/swe.mjs:85
R_EARTH = 6371e3                 # src/geometry.mjs:104
OMEGA_EARTH = 7.292115e-5        # src/geometry.mjs:106


# ---------------------------------------------------------------------------
# Built-in boundary conditions (src/swe.mjs:1026-1126).  They are applied on
# the device by applyBC()/step(); the objects identify the kind.
class _Boundary:
    def __init__(self, name):
        self.name = name
        self.kind = BC_KIND[name]

    def __call__(self, sim, i, j, side, g=0):
        raise NotImplementedError(
            f"{self.name}() is applied on the device for every ghost cell by sim.applyBC(); "
            "it is not callable per cell")

    def __repr__(self):
        return self.name


reflect = _Boundary("reflect")
outflow = _Boundary("outflow")
periodic = _Boundary("periodic")


class Flather:
    """flather(etaExt, uExt) of src/swe.mjs:1085-1115.

    etaExt/uExt are functions of t.  Before each step the host evaluates them
    at sim.t (both RK stages see the same t, src/swe.mjs:1093); a harmonic
    tide (tide.TideSignal) is instead evaluated on the device each step,
    which lets `run()` keep the whole loop on the GPU.
    """
    kind = BC_KIND["flather"]
    name = "flather"

    def __init__(self, etaExt, uExt=None):
        self.etaExt = etaExt
        self.uExt = uExt if uExt is not None else (lambda t: 0.0)
        # A harmonic tide with u = coef * eta (or u = 0) runs on the device.
        self._device_ucoef = None
        tide = getattr(etaExt, "tide", None)
        if tide is not None and getattr(etaExt, "coef", 1) is None:
            if uExt is None:
                self._device_ucoef = 0.0
            elif getattr(uExt, "tide", None) is tide and getattr(uExt, "coef", None) is not None:
                self._device_ucoef = float(uExt.coef)

    def __call__(self, sim, i, j, side, g=0):
        raise NotImplementedError("flather() is applied on the device by sim.applyBC()")


def flather(etaExt, uExt=None):
    return Flather(etaExt, uExt)


class Sponge:
    """makeSponge(sim, {side, width, strength, etaRef}), src/swe.mjs:1174-1198."""

    def __init__(self, side="east", width=20, strength=0.06, etaRef=0.0):
        if side not in SIDES:
            side = "south"                      # the reference's else-branch
        if callable(etaRef):
            raise NotImplementedError("a time-varying sponge reference is not supported on the device")
        self.side, self.width, self.strength, self.etaRef = side, int(width), float(strength), float(etaRef)

    def __call__(self, sim, dt):
        raise NotImplementedError("the sponge runs on the device inside step()")


def makeSponge(sim, side="east", width=20, strength=0.06, etaRef=0.0, **kw):
    if isinstance(side, dict):                  # makeSponge(sim, {...}) as in JS
        return Sponge(**side)
    return Sponge(side=side, width=width, strength=strength, etaRef=etaRef)


def hllc(out, hL, huL, hvL, hR, huR, hvR, dry=1e-4):
    """The exported Riemann solver (src/swe.mjs:975), evaluated on the GPU."""
    lib = _lib.load()
    inp = np.array([hL, huL, hvL, hR, huR, hvR, dry], dtype=np.float64)
    res = np.zeros(3)
    check(lib.swe_hllc_batch(1, dptr(inp), dptr(res)))
    if out is None:
        out = [0.0, 0.0, 0.0]
    out[0], out[1], out[2] = float(res[0]), float(res[1]), float(res[2])
    return out


def hllc_batch(inputs):
    """hllc over an (n, 7) array of (hL, huL, hvL, hR, huR, hvR, dry) rows."""
    lib = _lib.load()
    a = np.ascontiguousarray(inputs, dtype=np.float64).reshape(-1, 7)
    out = np.zeros((a.shape[0], 3))
    check(lib.swe_hllc_batch(a.shape[0], dptr(a), dptr(out)))
    return out


# ---------------------------------------------------------------------------
class Geometry:
    """The metric object of src/geometry.mjs:301-309: 13 per-row arrays and scalars."""

    def __init__(self, kind, nx, ny, ng, rows, scalars, extra):
        self.kind, self.nx, self.ny, self.ng, self.H = kind, nx, ny, ng, ny + 2 * ng
        self._rows = rows
        self._on_write = None
        self.dx, self.dy = scalars["dx"], scalars["dy"]
        self.R, self.totalArea = scalars["R"], scalars["totalArea"]
        if kind == "sphere":
            self.dlam, self.dphi = scalars["dlam"], scalars["dphi"]
            self.lat0, self.lat1, self.omega = extra["lat0"], extra["lat1"], extra["omega"]

    def __getattr__(self, name):
        rows = self.__dict__.get("_rows")
        if rows is not None and name in rows:
            cb = self.__dict__.get("_on_write")
            if cb is not None:
                cb(name)
            return rows[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        rows = self.__dict__.get("_rows")
        if rows is not None and name in rows:
            rows[name][:] = value
            cb = self.__dict__.get("_on_write")
            if cb is not None:
                cb(name)
            return
        object.__setattr__(self, name, value)


def _options(nx, ny, dx, dy, manning, minDepth, cfl, coriolis, order, limiter, sphere):
    o = _lib.SweOptions()
    _lib.load().swe_options_init(ctypes.byref(o))
    o.nx, o.ny = int(nx), int(ny)
    o.dx = float(dx) if dx is not None else float("nan")
    o.dy = float(dy if dy is not None else (dx if dx is not None else float("nan")))
    o.manning, o.min_depth, o.cfl, o.coriolis = float(manning), float(minDepth), float(cfl), float(coriolis)
    o.order = int(order)
    o.limiter = LIMITERS.get(limiter, -1)
    if sphere:
        o.sphere = 1
        o.R = float(sphere.get("R", R_EARTH))
        o.lat0 = float(sphere.get("lat0", -90))
        o.lat1 = float(sphere.get("lat1", 90))
        o.omega = float(sphere.get("omega", 0))
    return o


def _geometry_from_options(o, ng=2):
    lib = _lib.load()
    H = o.ny + 2 * ng
    rows = np.zeros(len(GEOM_ROWS) * H)
    sc = np.zeros(6)
    check(lib.swe_compute_geometry(ctypes.byref(o), dptr(rows), dptr(sc)))
    rowd = {name: rows[r * H:(r + 1) * H].copy() for r, name in enumerate(GEOM_ROWS)}
    scalars = {"dx": sc[0], "dy": sc[1], "R": sc[2], "dlam": sc[3], "dphi": sc[4], "totalArea": sc[5]}
    extra = {"lat0": o.lat0, "lat1": o.lat1, "omega": o.omega}
    return Geometry("sphere" if o.sphere else "cartesian", o.nx, o.ny, ng, rowd, scalars, extra)


def _jmax0(d):
    """Math.max(0, d) elementwise: NaN stays NaN, -0 becomes +0."""
    d = np.asarray(d, dtype=np.float64)
    return np.where(d > 0, d, np.where(np.isnan(d), d, 0.0))


def _sample(fn, coords, shape):
    """Sample a bed/eta0/n argument at every padded cell (src/swe.mjs:222-232)."""
    if isinstance(fn, np.ndarray):
        a = np.ascontiguousarray(fn, dtype=np.float64).reshape(shape)
        return a.copy()
    if not callable(fn):
        return np.full(shape, float(fn))
    out = np.empty(shape)
    H, W = shape
    for j in range(H):
        for i in range(W):
            x, y = coords(i, j)
            out[j, i] = fn(x, y)
    return out


class ShallowWater:
    """new ShallowWater({...}) of src/swe.mjs:170-244, on the GPU."""

    def __init__(self, nx, ny, dx=None, dy=None, bed=None, eta0=0, manning=0.025, minDepth=1e-3,
                 cfl=0.45, coriolis=0, order=2, limiter="mc", sphere=None, _gridlands_manning=False):
        lib = _lib.load()
        self._lib = lib
        if limiter not in LIMITERS:
            raise ValueError(f"unknown limiter {limiter}; have {','.join(['minmod', 'mc', 'central'])}")
        o = _options(nx, ny, dx, dy, manning, minDepth, cfl, coriolis, order, limiter, sphere)
        self._opts = o
        self.nx, self.ny = int(nx), int(ny)
        self.ng = 2
        self.W, self.H = self.nx + 4, self.ny + 4
        self.manning, self.minDepth, self.cfl = manning, minDepth, cfl
        self.eps4 = max(minDepth, 1e-12) ** 4
        self.coriolis, self.order = coriolis, order
        self.limiterName = limiter
        self.manningField = None
        self.forcing_ = None
        geom = _geometry_from_options(o)          # raises the reference's errors
        self.geom = geom
        if sphere:
            self.dx, self.dy = None, geom.dy
        else:
            self.dx, self.dy = dx, (dy if dy is not None else dx)
        shape = (self.H, self.W)
        if sphere:
            coords = lambda i, j: self.cellLonLat(i - 2, j - 2)
        else:
            coords = lambda i, j: self.cellCentre(i - 2, j - 2)
        if bed is None:
            bed = 0.0
        terrain = getattr(bed, "_gridlands", None)
        if terrain is not None and not sphere and getattr(eta0, "_gridlands", None) is terrain \
                and bed is terrain.bed and eta0 is terrain.eta0:
            # an imported gridlands terrain: sampled on the device from its layers
            from .gridlands import create_sim_handle
            self._h = create_sim_handle(o, terrain, manning_field=_gridlands_manning)
        else:
            b = _sample(bed, coords, shape).reshape(-1)
            e = _sample(eta0, coords, shape).reshape(-1)
            h = _jmax0(e - b)
            handle = ctypes.c_void_p()
            check(lib.swe_create(ctypes.byref(o), dptr(b), dptr(h), ctypes.byref(handle)))
            self._h = handle
        # host mirrors
        self._host = {}
        self._fresh = set()
        self._dirty = set()
        self._geom_dirty = set()
        self._keep_h0 = False
        geom._on_write = self._geom_dirty.add
        self._boundaries = _Boundaries(self, sphere is not None and sphere is not False)
        self._apply_boundaries_kinds()
        self._sponge = None

        if terrain is not None and _gridlands_manning:
            nf = np.empty(self.W * self.H)
            check(lib.swe_get_field(self._h, FIELD["manning"], dptr(nf)))
            self.manningField = nf

    @classmethod
    def fromGridlands(cls, t, manningField=False, **opts):
        """new ShallowWater({nx, ny, dx, dy from t.domain, bed: t.bed, eta0: t.eta0,
        manning: t.manning, ...opts}) for a terrain from gridlandsTerrain(), built
        on the device; with manningField, the export's per-cell n as well (the
        field tools/verify-gridlands.mjs:326-333 sets)."""
        d = t.domain
        kw = dict(nx=d["nx"], ny=d["ny"], dx=d["dx"], dy=d["dy"], manning=t.manning)
        kw.update(opts)
        return cls(bed=t.bed, eta0=t.eta0, _gridlands_manning=bool(manningField), **kw)

    # ---- lifetime -----------------------------------------------------------
    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.swe_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- coordinates (src/swe.mjs:246-279) ---------------------------------
    def cellCentre(self, i, j):
        if self.geom.kind == "sphere":
            raise ValueError("cellCentre is Cartesian-only; a spherical cell has no single "
                             "x in metres. Use cellLonLat(i, j).")
        return [(i + 0.5) * self.dx, (j + 0.5) * self.dy]

    def cellLonLat(self, i, j):
        g = self.geom
        if g.kind != "sphere":
            raise ValueError("cellLonLat is spherical-only")
        lon = (i + 0.5) * g.dlam * 180 / math.pi
        return [math.fmod(math.fmod(lon, 360) + 360, 360) - 180,
                g._rows["phiC"][j + self.ng] * 180 / math.pi]

    def idx(self, i, j):
        return (j + self.ng) * self.W + (i + self.ng)

    def eta(self, i, j):
        k = self.idx(i, j)
        return float(self.field("b")[k] + self.field("h")[k])

    def depth(self, i, j):
        return float(self.field("h")[self.idx(i, j)])

    def vel(self, hq, h):
        """src/swe.mjs:282-285, evaluated on the GPU (scalars or arrays)."""
        scalar = np.isscalar(hq) and np.isscalar(h)
        a = np.ascontiguousarray(np.atleast_1d(hq), dtype=np.float64)
        bh = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(h), a.shape), dtype=np.float64)
        out = np.zeros(a.shape)
        check(self._lib.swe_vel_batch(self._h, a.size, dptr(a), dptr(bh), dptr(out)))
        return float(out[0]) if scalar else out

    # ---- field mirrors ------------------------------------------------------
    def _download(self, name):
        arr = self._host.get(name)
        if arr is None:
            arr = np.zeros(self.W * self.H)
            self._host[name] = arr
        if name not in self._fresh:
            check(self._lib.swe_get_field(self._h, FIELD[name], dptr(arr)))
            self._fresh.add(name)
        return arr

    def _push(self):
        """Upload every field or metric row the caller may have written."""
        for name in list(self._dirty):
            if name in ("b", "h", "hu", "hv"):
                check(self._lib.swe_set_field(self._h, FIELD[name], dptr(self._host[name])))
        self._dirty.clear()
        for name in list(self._geom_dirty):
            row = np.ascontiguousarray(self.geom._rows[name], dtype=np.float64)
            check(self._lib.swe_set_geom(self._h, GEOM_ROWS.index(name), dptr(row)))
        self._geom_dirty.clear()

    def _stale(self, *names):
        for n in names:
            self._fresh.discard(n)

    def field(self, name):
        """Read-only snapshot of a field (never uploaded back)."""
        if name in self._dirty:
            return self._host[name]
        a = self._download(name).copy()
        a.flags.writeable = False
        return a

    def _writable(self, name):
        a = self._download(name)
        if name in ("b", "h", "hu", "hv"):
            self._dirty.add(name)
        return a

    def _set_field(self, name, value):
        a = self._download(name)
        a[:] = np.asarray(value, dtype=np.float64).reshape(-1)
        self._dirty.add(name)

    b = property(lambda s: s._writable("b"), lambda s, v: s._set_field("b", v))
    h = property(lambda s: s._writable("h"), lambda s, v: s._set_field("h", v))
    hu = property(lambda s: s._writable("hu"), lambda s, v: s._set_field("hu", v))
    hv = property(lambda s: s._writable("hv"), lambda s, v: s._set_field("hv", v))
    rh = property(lambda s: s._writable("rh"))
    rhu = property(lambda s: s._writable("rhu"))
    rhv = property(lambda s: s._writable("rhv"))
    theta = property(lambda s: s._writable("theta"))

    def get_rows(self, name, row0, nrows):
        """Rows [row0, row0 + nrows) of b, h, hu or hv over the padded grid,
        read from the device (the halo exchange of slabs.py)."""
        self._push()
        out = np.empty(int(nrows) * self.W)
        check(self._lib.swe_get_rows(self._h, FIELD[name], int(row0), int(nrows), dptr(out)))
        return out

    def set_rows(self, name, row0, values):
        """Write rows starting at row0 of b, h, hu or hv on the device."""
        self._push()
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if v.size % self.W:
            raise ValueError("set_rows: a whole number of rows of W values")
        check(self._lib.swe_set_rows(self._h, FIELD[name], int(row0), v.size // self.W, dptr(v)))
        self._stale(name)

    def _h0(self, name):
        if not self._keep_h0:
            check(self._lib.swe_set_keep_h0(self._h, 1))
            self._keep_h0 = True
        return self._writable(name)

    h0 = property(lambda s: s._h0("h0"))
    hu0 = property(lambda s: s._h0("hu0"))
    hv0 = property(lambda s: s._h0("hv0"))

    # ---- clock --------------------------------------------------------------
    def _scalar(self, name):
        v = ctypes.c_double()
        check(self._lib.swe_get_scalar(self._h, SCALAR[name], ctypes.byref(v)))
        return v.value

    @property
    def t(self):
        ft = getattr(self, "_forcing_t", None)
        return ft if ft is not None else self._scalar("t")

    @t.setter
    def t(self, v):
        check(self._lib.swe_set_scalar(self._h, SCALAR["t"], float(v)))

    @property
    def steps(self):
        return int(self._scalar("steps"))

    @steps.setter
    def steps(self, v):
        check(self._lib.swe_set_scalar(self._h, SCALAR["steps"], float(v)))

    @property
    def massFloored(self):
        return self._scalar("massFloored")

    # ---- boundaries and forcing ---------------------------------------------
    @property
    def boundaries(self):
        return self._boundaries

    @boundaries.setter
    def boundaries(self, value):
        for side in SIDES:
            if isinstance(value, dict):
                if side in value:
                    self._boundaries[side] = value[side]
            else:
                self._boundaries[side] = getattr(value, side)

    def _apply_boundaries_kinds(self):
        for side, s in SIDES.items():
            fn = self._boundaries[side]
            if isinstance(fn, Flather):
                continue               # set per step (or as a device tide) by _prepare_flather
            check(self._lib.swe_set_boundary(self._h, s, fn.kind))

    def _prepare_flather(self, t=None):
        for side, s in SIDES.items():
            fn = self._boundaries[side]
            if not isinstance(fn, Flather):
                continue
            table = getattr(fn.etaExt, "device_table", None)
            if table is not None and getattr(fn, "_device_ucoef", None) is not None:
                msl, amp, omega, phase = table()
                check(self._lib.swe_set_flather_tide(
                    self._h, s, msl, len(amp), dptr(amp), dptr(omega), dptr(phase), fn._device_ucoef))
                continue
            if t is None:
                t = self.t
            e0 = float(fn.etaExt(t))
            u0 = float(fn.uExt(t))
            check(self._lib.swe_set_flather_values(self._h, s, e0, u0))

    def _device_loop_ok(self):
        for side in SIDES:
            fn = self._boundaries[side]
            if isinstance(fn, Flather) and getattr(fn, "_device_ucoef", None) is None:
                return False
        return self.forcing_ is None or isinstance(self.forcing_, Sponge)

    @property
    def forcing(self):
        return self.forcing_

    @forcing.setter
    def forcing(self, fn):
        self.forcing_ = fn
        if isinstance(fn, Sponge):
            check(self._lib.swe_set_sponge(self._h, SIDES[fn.side], fn.width, fn.strength, fn.etaRef))
        else:
            check(self._lib.swe_clear_sponge(self._h))

    # ---- the hot path -------------------------------------------------------
    def applyBC(self):
        """src/swe.mjs:289-303"""
        self._push()
        self._prepare_flather()
        check(self._lib.swe_apply_bc(self._h))
        self._stale("b", "h", "hu", "hv")

    def residual(self, dt):
        """src/swe.mjs:308-629: fills rh, rhu, rhv and theta."""
        self._push()
        check(self._lib.swe_residual(self._h, float(dt)))
        self._stale("rh", "rhu", "rhv", "theta")

    def maxDt(self):
        """src/swe.mjs:632-647"""
        self._push()
        v = ctypes.c_double()
        check(self._lib.swe_max_dt(self._h, ctypes.byref(v)))
        return v.value

    def applyFriction(self, dt):
        """src/swe.mjs:659-704"""
        self._push()
        check(self._lib.swe_apply_friction(self._h, float(dt)))
        self._stale("hu", "hv")

    def setManningField(self, fn):
        """src/swe.mjs:714-731; fn(x, y) or (lon, lat), an array, or None."""
        self._push()
        if fn is None:
            check(self._lib.swe_set_manning_field(self._h, None))
            self.manningField = None
            return self
        if self.geom.kind == "sphere":
            coords = lambda i, j: self.cellLonLat(i - 2, j - 2)
        else:
            coords = lambda i, j: self.cellCentre(i - 2, j - 2)
        if isinstance(fn, np.ndarray):
            n = np.ascontiguousarray(fn, dtype=np.float64).reshape(-1).copy()
        else:
            n = np.empty(self.W * self.H)
            for j in range(self.H):
                for i in range(self.W):
                    x, y = coords(i, j)
                    v = fn(x, y)
                    if not (v >= 0) or not math.isfinite(v):
                        raise ValueError(f"setManningField: n = {v} at ({x}, {y}); "
                                         "Manning n must be finite and >= 0")
                    n[j * self.W + i] = v
        check(self._lib.swe_set_manning_field(self._h, dptr(n)))
        self.manningField = n
        return self

    def dryClean(self):
        """src/swe.mjs:734-745"""
        self._push()
        v = ctypes.c_double()
        check(self._lib.swe_dry_clean(self._h, ctypes.byref(v)))
        self._stale("h", "hu", "hv")
        return v.value

    def step(self, dt=None):
        """src/swe.mjs:754-814.  Returns the dt taken, 0 for a refused dt."""
        self._push()
        t0 = self.t
        self._prepare_flather(t0)
        v = ctypes.c_double()
        if dt is None:
            check(self._lib.swe_step_auto(self._h, ctypes.byref(v)))
        else:
            check(self._lib.swe_step(self._h, float(dt), ctypes.byref(v)))
        self._stale("b", "h", "hu", "hv", "h0", "hu0", "hv0")
        taken = v.value
        fn = self.forcing_
        if taken and fn is not None and not isinstance(fn, Sponge):
            # A user-supplied forcing is user code: it runs on the host
            # mirrors, after friction and before t advances (src/swe.mjs:809).
            self._forcing_t = t0
            try:
                fn(self, taken)
            finally:
                self._forcing_t = None
        return taken

    def run(self, n, dt=None, tEnd=math.inf):
        """n steps kept on the device (swe_run): dt fixed, or maxDt() each
        step, clamped to tEnd - t.  Equivalent to
        `for (...) sim.step(Math.min(dt ?? sim.maxDt(), tEnd - sim.t))`."""
        self._push()
        if not self._device_loop_ok():
            done = 0
            for _ in range(int(n)):
                d = self.maxDt() if dt is None else dt
                d = min(d, tEnd - self.t)
                if not self.step(d):
                    break
                done += 1
            return done
        self._prepare_flather()
        out = ctypes.c_int()
        check(self._lib.swe_run(self._h, int(n), float(dt) if dt else 0.0, float(tEnd), ctypes.byref(out)))
        self._stale("b", "h", "hu", "hv", "h0", "hu0", "hv0")
        return out.value

    # ---- diagnostics (src/swe.mjs:819-917) -----------------------------------
    def _diag(self, fn, *args):
        self._push()
        v = ctypes.c_double()
        check(fn(self._h, *args, ctypes.byref(v)))
        return v.value

    def volume(self):
        return self._diag(self._lib.swe_volume)

    def energy(self):
        return self._diag(self._lib.swe_energy)

    def maxSurfaceDeviation(self, ref):
        return self._diag(self._lib.swe_max_surface_deviation, float(ref))

    def maxSpeed(self):
        return self._diag(self._lib.swe_max_speed)

    def finite(self):
        self._push()
        v = ctypes.c_int()
        check(self._lib.swe_finite(self._h, ctypes.byref(v)))
        return bool(v.value)

    def synchronize(self):
        check(self._lib.swe_synchronize(self._h))


class _Boundaries:
    """sim.boundaries: attribute and item access; writes go to the device."""

    def __init__(self, sim, sphere):
        object.__setattr__(self, "_sim", sim)
        d = {"west": periodic, "east": periodic, "south": reflect, "north": reflect} if sphere else \
            {"west": reflect, "east": reflect, "south": reflect, "north": reflect}
        object.__setattr__(self, "_d", d)

    def __getitem__(self, side):
        return self._d[side]

    def __setitem__(self, side, fn):
        if side not in SIDES:
            raise KeyError(side)
        if not isinstance(fn, (_Boundary, Flather)):
            raise NotImplementedError(
                "boundaries must be reflect, outflow, periodic or flather(...): they run on the device")
        self._d[side] = fn
        if not isinstance(fn, Flather):
            check(self._sim._lib.swe_set_boundary(self._sim._h, SIDES[side], fn.kind))

    def __getattr__(self, side):
        if side in SIDES:
            return self._d[side]
        raise AttributeError(side)

    def __setattr__(self, side, fn):
        self[side] = fn


def cartesianGeometry(nx, ny, dx, dy=None, ng=2, coriolis=0):
    """src/geometry.mjs:163-176 (computed by the library's host-side set-up)."""
    if ng != 2:
        raise ValueError("the solver uses ng = 2")
    o = _options(nx, ny, dx, dy, 0.025, 1e-3, 0.45, coriolis, 2, "mc", None)
    return _geometry_from_options(o)


def sphericalGeometry(nx, ny, R=R_EARTH, lat0=-90, lat1=90, ng=2, omega=0):
    """src/geometry.mjs:190-299; raises the reference's errors."""
    if ng != 2:
        raise ValueError("the solver uses ng = 2")
    o = _options(nx, ny, None, None, 0.025, 1e-3, 0.45, 0, 2, "mc",
                 {"R": R, "lat0": lat0, "lat1": lat1, "omega": omega})
    try:
        return _geometry_from_options(o)
    except _lib.SweError as e:
        raise ValueError(str(e)) from None


def interiorArea(g):
    """src/geometry.mjs:325-329"""
    s = 0.0
    area = g._rows["area"]
    for j in range(g.ng, g.H - g.ng):
        s += area[j] * g.nx
    return s


def cellLonLat(g, i, j):
    """src/geometry.mjs:312-315"""
    if g.kind != "sphere":
        raise ValueError("cellLonLat is spherical-only")
    return [(i + 0.5) * g.dlam * 180 / math.pi - 180, g._rows["phiC"][j + g.ng] * 180 / math.pi]
