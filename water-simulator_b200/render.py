"""Headless frames of a simulation, computed on the device.

  renderMap(sim, ...)            the map panel of WaterView.draw() (src/render.mjs:220-247)
  globeCamera / buildGlobeLut /
  renderGlobe(out, sim, ...)     the orthographic globe of src/globe.mjs:460-812

Frames are RGBA bytes as the reference's ImageData holds them.  They are
written by kernels into a device buffer and copied to a numpy array, or
left on the device (`device_ptr`, e.g. a torch CUDA uint8 tensor's
data_ptr()) for a consumer that never needs them on the host.  The canvas
parts of the reference (the section panel's vector drawing, labels) are not
pixels of the state and are not rebuilt.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check

RAMP_N = 1025


def colourTables():
    """(RAMP as (1025, 3) float64 of src/render.mjs, CBYTES as (1025, 3) uint8 of src/globe.mjs)."""
    ramp = np.zeros(3 * RAMP_N)
    cb = np.zeros(3 * RAMP_N, dtype=np.uint8)
    check(_lib.load().swe_render_tables(ramp.ctypes.data, cb.ctypes.data))
    return ramp.reshape(RAMP_N, 3), cb.reshape(RAMP_N, 3)


def renderMap(sim, msl=0.0, scale=1.0, showBed=True, out=None, device_ptr=None):
    """WaterView.draw()'s map (nx x ny pixels, +y up).  Returns an (ny, nx, 4)
    uint8 array, or None when only `device_ptr` is given."""
    sim._push()
    if device_ptr is not None and out is None:
        check(_lib.load().swe_render_map(sim._h, float(msl), float(scale), 1 if showBed else 0, None,
                                         ctypes.c_void_p(device_ptr)))
        return None
    if out is None:
        out = np.empty((sim.ny, sim.nx, 4), dtype=np.uint8)
    assert out.dtype == np.uint8 and out.flags["C_CONTIGUOUS"] and out.size == 4 * sim.nx * sim.ny
    check(_lib.load().swe_render_map(sim._h, float(msl), float(scale), 1 if showBed else 0, out.ctypes.data,
                                     ctypes.c_void_p(device_ptr) if device_ptr is not None else None))
    return out


def globeCamera(size, tiltDeg=22, rotDeg=0, margin=0.94):
    """src/globe.mjs:460-466 (the fields the LUT depends on, plus rotDeg)."""
    return {"size": int(size), "tiltDeg": float(tiltDeg), "rotDeg": float(rotDeg), "margin": float(margin),
            "r": 0.5 * size * margin, "cx": 0.5 * size, "cy": 0.5 * size}


class GlobeLut:
    """The baked pixel -> cell table of buildGlobeLut(), resident on the device."""

    def __init__(self, handle, cam, sim):
        self._h = handle
        self._lib = _lib.load()
        self.size, self.tiltDeg, self.margin = cam["size"], cam["tiltDeg"], cam["margin"]
        c = (ctypes.c_int * 4)()
        check(self._lib.swe_globe_lut_get(self._h, c, None, None, None, None, None))
        self.count, self.inside, self.capped = c[0], c[1], c[2]
        self.key = f"{self.size}|{self.tiltDeg}|{self.margin}|{sim.nx}|{sim.ny}"

    def arrays(self):
        """The table as numpy arrays: px (byte offsets), lonBase, rowBase, lit (float32), bg."""
        n = self.count
        px = np.zeros(n, np.int32)
        lon = np.zeros(n)
        rb = np.zeros(n, np.int32)
        lit = np.zeros(n, np.float32)
        bg = np.zeros(4 * self.size * self.size, np.uint8)
        check(self._lib.swe_globe_lut_get(self._h, None, px.ctypes.data, lon.ctypes.data, rb.ctypes.data,
                                          lit.ctypes.data, bg.ctypes.data))
        return {"px": px, "lonBase": lon, "rowBase": rb, "lit": lit, "bg": bg}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.swe_globe_lut_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def buildGlobeLut(cam, sim, style=None):
    """src/globe.mjs:554-629 for the grid of a spherical sim."""
    style = style or {}

    def arr3(v):
        return None if v is None else (ctypes.c_double * 3)(*[float(x) for x in v])

    h = ctypes.c_void_p()
    check(_lib.load().swe_globe_lut_create(sim._h, cam["size"], cam["tiltDeg"], cam["margin"],
                                           arr3(style.get("sun")), arr3(style.get("bg")), arr3(style.get("halo")),
                                           ctypes.byref(h)))
    return GlobeLut(h, cam, sim)


def renderGlobe(out, sim, lut, rotDeg=0.0, scale=1.0, msl=0.0, landLight=True, device_ptr=None):
    """renderGlobe() (src/globe.mjs:770-812) into `out` (4 * size * size uint8,
    or None with `device_ptr`).  Returns the reference's frame statistics."""
    sim._push()
    st = (ctypes.c_double * 8)()
    host = None
    if out is not None:
        assert out.dtype == np.uint8 and out.flags["C_CONTIGUOUS"] and out.size == 4 * lut.size * lut.size
        host = out.ctypes.data
    check(_lib.load().swe_render_globe(sim._h, lut._h, float(rotDeg), float(scale), float(msl),
                                       1 if landLight else 0, host,
                                       ctypes.c_void_p(device_ptr) if device_ptr is not None else None, st))
    wet, dry = int(st[0]), int(st[1])
    return {"wet": wet, "dry": dry, "capped": int(st[2]), "inside": int(st[3]), "etaMin": st[4],
            "etaMax": st[5], "sat": int(st[6]), "satFrac": st[7], "scale": float(scale)}
