"""Test helpers for the misfit's tangent-linear reference (the oracle run on
dual numbers, oracle_tlm_misfit) and for finite differences on the oracle."""
import ctypes

import numpy as np

from oracle_sim import OracleOptions, OracleSim, oracle_lib, _dp


SIDE_ORDER = ("west", "east", "south", "north")
KIND = {"reflect": 0, "outflow": 1, "periodic": 2, "flather": 3}


class TideSpec(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("msl", ctypes.c_double), ("u_coef", ctypes.c_double),
                ("amp", ctypes.POINTER(ctypes.c_double)), ("omega", ctypes.POINTER(ctypes.c_double)),
                ("phase_deg", ctypes.POINTER(ctypes.c_double))]


def boundary_arrays(bcs):
    """(kinds, flather eta, flather u, tides) in W, E, S, N order from a dict
    of side -> "reflect" | "outflow" | "periodic" | ("flather", eta, u) |
    ("tide", msl, amps, omegas, phases_deg, u_coef).  The tides array keeps
    its tables alive in ._keep."""
    kinds, fe, fu = [0] * 4, [0.0] * 4, [0.0] * 4
    tides = (TideSpec * 4)()
    keep = []
    for side, bc in (bcs or {}).items():
        q = SIDE_ORDER.index(side)
        if isinstance(bc, str):
            kinds[q] = KIND[bc]
        elif bc[0] == "flather":
            kinds[q], fe[q], fu[q] = KIND["flather"], float(bc[1]), float(bc[2])
        else:
            kinds[q] = KIND["flather"]
            tabs = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in bc[2:5]]
            keep += tabs
            tides[q] = TideSpec(len(tabs[0]), float(bc[1]), float(bc[5]), *[_dp(t) for t in tabs])
    tides._keep = keep
    return kinds, fe, fu, tides


def tlm_misfit(case, b, n, db, dn, steps, obs, threads=1, bcs=None):
    lib = oracle_lib()
    fn = lib.oracle_tlm_misfit_bc
    D, I, DP = ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    IP = ctypes.POINTER(ctypes.c_int)
    fn.argtypes = [ctypes.POINTER(OracleOptions), DP, DP, DP, DP, DP, I, IP, I, DP, I, IP, DP, DP,
                   ctypes.POINTER(TideSpec), ctypes.POINTER(D), ctypes.POINTER(D), DP]
    fn.restype = I
    o = OracleOptions()
    o.nx, o.ny, o.dx, o.dy = case["nx"], case["ny"], case["dx"], case["dx"]
    o.manning, o.min_depth, o.cfl, o.coriolis, o.order, o.limiter, o.sphere = 0.025, 1e-3, 0.45, 0.0, 2, 0, 0
    g = np.ascontiguousarray(case["gauges"], dtype=np.int32)
    arrs = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (b, case["eta0"], n, db, dn)]
    ob = np.ascontiguousarray(obs, dtype=np.float64).reshape(-1)
    J, dJ = D(), D()
    dts = np.zeros(steps)
    kinds, fe, fu, tides = boundary_arrays(bcs)
    ka = np.ascontiguousarray(kinds, dtype=np.int32)
    fe, fu = np.ascontiguousarray(fe), np.ascontiguousarray(fu)
    rc = fn(ctypes.byref(o), _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]), _dp(arrs[3]), _dp(arrs[4]), len(g),
            g.ctypes.data_as(IP), steps, _dp(ob), threads, ka.ctypes.data_as(IP), _dp(fe), _dp(fu), tides,
            ctypes.byref(J), ctypes.byref(dJ), _dp(dts))
    assert rc == 0, lib.oracle_last_error()
    return J.value, dJ.value, dts


def oracle_misfit(case, b, n, steps, obs, dts, bcs=None):
    """J on the oracle (doubles) with the dt sequence held fixed."""
    sim = OracleSim(nx=case["nx"], ny=case["ny"], dx=case["dx"], bed=np.asarray(b), eta0=case["eta0"], manning=0.025)
    sim.setManningField(n)
    if bcs:
        conv = {}
        for side, bc in bcs.items():
            if isinstance(bc, str) or bc[0] == "tide":
                conv[side] = bc
            else:
                e, u = float(bc[1]), float(bc[2])
                conv[side] = ("flather", lambda t, e=e: e, lambda t, u=u: u)
        sim.set_boundaries(**conv)
    J = 0.0
    g = case["gauges"]
    for s in range(steps):
        sim.step(float(dts[s]))
        hb = sim.b[g] + sim.h[g]
        for q in range(len(g)):
            r = hb[q] - obs[s][q]
            J += r * r
    sim.close()
    return J
