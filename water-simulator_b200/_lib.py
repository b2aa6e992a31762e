"""ctypes binding of libswe_b200.so (the C ABI in include/swe_b200.h).

Loading fails loudly when the library is missing: there is no other
implementation behind the Python API.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The exact build (-fmad=false, bit-identical to the oracle) by default;
# SWE_B200_ARITH=fma selects the build whose compiler fuses multiply-adds.
LIB_PATH = os.path.join(HERE, "libswe_b200_fma.so" if os.environ.get("SWE_B200_ARITH") == "fma"
                        else "libswe_b200.so")

SWE_OK, SWE_EINVAL, SWE_ECUDA, SWE_ENONFINITE, SWE_ETIMEOUT = 0, -1, -2, -3, -4

FIELD = {"b": 0, "h": 1, "hu": 2, "hv": 3, "h0": 4, "hu0": 5, "hv0": 6,
         "rh": 7, "rhu": 8, "rhv": 9, "theta": 10, "manning": 11}
GEOM_ROWS = ["dxRow", "dyRowN", "dyRowS", "dyCFL", "area", "lx", "lyN", "lyS",
             "bedPhi", "phiC", "tanPhi", "fRow", "geoCoef"]
SCALAR = {"dx": 0, "dy": 1, "R": 2, "dlam": 3, "dphi": 4, "totalArea": 5, "t": 6,
          "steps": 7, "massFloored": 8, "eps4": 9}
SIDES = {"west": 0, "east": 1, "south": 2, "north": 3}
BC_KIND = {"reflect": 0, "outflow": 1, "periodic": 2, "flather": 3}
LIMITERS = {"mc": 0, "minmod": 1, "central": 2}


class SweOptions(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("manning", ctypes.c_double), ("min_depth", ctypes.c_double),
                ("cfl", ctypes.c_double), ("coriolis", ctypes.c_double),
                ("order", ctypes.c_int), ("limiter", ctypes.c_int), ("sphere", ctypes.c_int),
                ("R", ctypes.c_double), ("lat0", ctypes.c_double), ("lat1", ctypes.c_double),
                ("omega", ctypes.c_double)]


class SweGridlands(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("cell_m", ctypes.c_double),
                ("flip_rows", ctypes.c_int),
                ("bed_b64", ctypes.c_char_p), ("bed_len", ctypes.c_size_t),
                ("surface_b64", ctypes.c_char_p), ("surface_len", ctypes.c_size_t),
                ("manning_b64", ctypes.c_char_p), ("manning_len", ctypes.c_size_t),
                ("bed_f32", ctypes.c_void_p), ("surface_f32", ctypes.c_void_p), ("manning_f32", ctypes.c_void_p),
                ("manning_field", ctypes.c_int)]


class SweError(RuntimeError):
    """A failure reported by the C ABI (status code + message)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "swe_set_device": [_I],
    "swe_options_init": [ctypes.POINTER(SweOptions)],
    "swe_create": [ctypes.POINTER(SweOptions), _DP, _DP, ctypes.POINTER(_P)],
    "swe_destroy": [_P],
    "swe_last_error": [],
    "swe_get_dims": [_P, _IP],
    "swe_get_field": [_P, _I, _DP],
    "swe_set_field": [_P, _I, _DP],
    "swe_get_rows": [_P, _I, _I, _I, _DP],
    "swe_set_rows": [_P, _I, _I, _I, _DP],
    "swe_get_rows_async": [_P, _I, _I, _I, _P],
    "swe_set_rows_async": [_P, _I, _I, _I, _P],
    "swe_max_dt_to": [_P, _P],
    "swe_step_dt_from": [_P, _P],
    "swe_get_geom": [_P, _I, _DP],
    "swe_set_geom": [_P, _I, _DP],
    "swe_get_scalar": [_P, _I, _DP],
    "swe_set_scalar": [_P, _I, _D],
    "swe_set_boundary": [_P, _I, _I],
    "swe_set_flather_values": [_P, _I, _D, _D],
    "swe_set_flather_tide": [_P, _I, _D, _I, _DP, _DP, _DP, _D],
    "swe_set_manning_field": [_P, _DP],
    "swe_set_sponge": [_P, _I, _I, _D, _D],
    "swe_clear_sponge": [_P],
    "swe_set_keep_h0": [_P, _I],
    "swe_apply_bc": [_P],
    "swe_residual": [_P, _D],
    "swe_max_dt": [_P, _DP],
    "swe_apply_friction": [_P, _D],
    "swe_dry_clean": [_P, _DP],
    "swe_step": [_P, _D, _DP],
    "swe_step_auto": [_P, _DP],
    "swe_run": [_P, _I, _D, _D, _IP],
    "swe_volume": [_P, _DP],
    "swe_energy": [_P, _DP],
    "swe_max_surface_deviation": [_P, _D, _DP],
    "swe_max_speed": [_P, _DP],
    "swe_set_diag_order": [_P, _I],
    "swe_eta_projection": [_P, _DP, _DP],
    "swe_finite": [_P, _IP],
    "swe_synchronize": [_P],
    "swe_get_stream": [_P, ctypes.POINTER(_P)],
    "swe_step_timed": [_P, _D, _DP],
    "swe_get_launch_config": [_P, _IP],
    "swe_compute_geometry": [ctypes.POINTER(SweOptions), _DP, _DP],
    "swe_hllc_batch": [_I, _DP, _DP],
    "swe_vel_batch": [_P, _I, _DP, _DP, _DP],
    "swe_max_dt_noalloc": [_I, _I, _P, _P, _P, _P, _P, _D, _D, _P, _P],
    "swe_gridlands_decode": [ctypes.c_char_p, ctypes.c_size_t, _I, _P],
    "swe_gridlands_create": [ctypes.POINTER(SweOptions), ctypes.POINTER(SweGridlands), ctypes.POINTER(_P)],
    "swe_gridlands_bodies": [_I, _I, _P, _P, _P],
    "swe_set_stage_kernels": [_P, _I],
    "swe_get_stage_kernels": [_P, _IP],
    "swe_render_map": [_P, _D, _D, _I, _P, _P],
    "swe_render_tables": [_P, _P],
    "swe_globe_lut_create": [_P, _I, _D, _D, _P, _P, _P, ctypes.POINTER(_P)],
    "swe_globe_lut_destroy": [_P],
    "swe_globe_lut_get": [_P, _P, _P, _P, _P, _P, _P],
    "swe_render_globe": [_P, _P, _D, _D, _D, _I, _P, _P, _P],
    "swe_batch_create": [_I, ctypes.POINTER(SweOptions), ctypes.POINTER(_DP), ctypes.POINTER(_DP), ctypes.POINTER(_P)],
    "swe_batch_destroy": [_P],
    "swe_batch_set_boundary": [_P, _I, _I, _I],
    "swe_batch_set_flather_tide": [_P, _I, _I, _D, _I, _DP, _DP, _DP, _D],
    "swe_batch_set_schedule": [_P, _I, _I, _I],
    "swe_batch_get_schedule": [_P, _IP],
    "swe_batch_autotune": [_P, _I, _IP, _DP],
    "swe_batch_run": [_P, _I],
    "swe_batch_synchronize": [_P],
    "swe_batch_set_launch": [_P, _I],
    "swe_batch_get_launch": [_P, _IP],
    "swe_batch_set_wait_limit": [_P, _D],
    "swe_batch_debug_hold": [_P, _I],
    "swe_batch_get_stream": [_P, ctypes.POINTER(_P)],
    "swe_batch_get_field": [_P, _I, _I, _DP],
    "swe_batch_get_scalar": [_P, _I, _I, _DP],
    "swe_adjoint_create": [ctypes.POINTER(SweOptions), _DP, _DP, _DP, _I, _IP, _I, _I, ctypes.POINTER(_P)],
    "swe_adjoint_destroy": [_P],
    "swe_adjoint_set_observations": [_P, _DP],
    "swe_adjoint_forward": [_P, _DP, _DP],
    "swe_adjoint_backward": [_P, _DP, _DP],
    "swe_adjoint_dt_sequence": [_P, _DP, _DP],
    "swe_adjoint_get_stream": [_P, ctypes.POINTER(_P)],
    "swe_adjoint_set_boundary": [_P, _I, _I],
    "swe_adjoint_set_flather_values": [_P, _I, _D, _D],
    "swe_adjoint_set_flather_tide": [_P, _I, _D, _I, _DP, _DP, _DP, _D],
}
_RESTYPES = {"swe_last_error": ctypes.c_char_p}

_lib = None


def load(path=LIB_PATH):
    """Load and bind the library once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with water-simulator_b200/build.py "
            "(nvcc, sm_100a). There is no CPU implementation to fall back to.")
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(rc):
    if rc != SWE_OK:
        msg = load().swe_last_error()
        raise SweError(rc, msg.decode() if msg else f"status {rc}")
    return rc


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array."""
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)
