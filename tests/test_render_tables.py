"""The colour tables of the headless frames (built on the host, no GPU):
against a restatement of buildRamp / labToSrgbRaw (src/render.mjs:98-131) and
of CBYTES (src/globe.mjs:644-652), and against the figures the reference
measured on its own ramp (src/render.mjs:46-57): worst L* asymmetry 1.174e-4
exact and 0.4410 in 8 bits (1025 samples) on a 65.963 L* span, no step at
mean sea level, nothing out of gamut."""
import math

import numpy as np
import pytest

RAMP_N, MID = 1025, 512


def lab_to_srgb_raw(L, a, bb):
    fy = (L + 16) / 116
    fx, fz = fy + a / 500, fy - bb / 200

    def g(f):
        return f * f * f if f * f * f > 0.008856 else (f - 16 / 116) / 7.787

    X, Y, Z = 0.95047 * g(fx), g(fy), 1.08883 * g(fz)

    def enc(u):
        return 255 * (12.92 * u if u <= 0.0031308 else 1.055 * math.pow(max(u, 0), 1 / 2.4) - 0.055)

    return [enc(3.2406 * X - 1.5372 * Y - 0.4986 * Z), enc(-0.9689 * X + 1.8758 * Y + 0.0415 * Z),
            enc(0.0557 * X - 0.2040 * Y + 1.0570 * Z)]


def ramp_ref():
    T, M, C = [20, 8, -34], [53, -4, -14], [86, 6, 44]
    out = []
    for i in range(RAMP_N):
        t = -1 + (2 * i) / (RAMP_N - 1)
        e = C if t >= 0 else T
        q = abs(t)
        out.append(lab_to_srgb_raw(*[M[c] + (e[c] - M[c]) * q for c in range(3)]))
    return np.array(out)


def js_round(x):
    f = math.floor(x)
    return f + 1 if x - f >= 0.5 else f


def u8clamp(x):
    if not (x > 0):
        return 0
    if x >= 255:
        return 255
    f = math.floor(x)
    d = x - f
    if d > 0.5:
        return f + 1
    if d < 0.5:
        return f
    return f if f % 2 == 0 else f + 1


def surface_colour(ramp, v, scale):
    t = max(-1, min(1, v / scale))
    q = js_round(abs(t) * MID)
    return ramp[MID + q] if t >= 0 else ramp[MID - q]


def Lstar(c):
    def lin(u):
        u /= 255
        return u / 12.92 if u <= 0.04045 else math.pow((u + 0.055) / 1.055, 2.4)
    Y = 0.2126 * lin(c[0]) + 0.7152 * lin(c[1]) + 0.0722 * lin(c[2])
    return 116 * math.cbrt(Y) - 16 if Y > 0.008856 else 903.3 * Y


def ramp_symmetry(ramp, samples, round8):
    """rampSymmetry (src/render.mjs:164-191)."""
    q = (lambda c: [max(0, min(255, js_round(x))) for x in c]) if round8 else (lambda c: list(c))
    L0 = Lstar(q(surface_colour(ramp, 0, 1)))
    worst = 0.0
    for n in range(1, samples + 1):
        t = n / samples
        up = Lstar(q(surface_colour(ramp, t, 1))) - L0
        down = L0 - Lstar(q(surface_colour(ramp, -t, 1)))
        worst = max(worst, abs(up - down))
    zp, zn = q(surface_colour(ramp, 1e-12, 1)), q(surface_colour(ramp, -1e-12, 1))
    return {"worstAsym": worst, "jump": math.hypot(*[zp[c] - zn[c] for c in range(3)]),
            "span": Lstar(q(surface_colour(ramp, 1, 1))) - Lstar(q(surface_colour(ramp, -1, 1))),
            "outOfGamut": max(0.0, float(np.max(np.maximum(-ramp, ramp - 255))))}


def test_tables_match_the_restatement(swe):
    ramp, cb = swe.colourTables()
    ref = ramp_ref()
    assert np.array_equal(ramp, ref)
    want = np.array([[u8clamp(x) for x in surface_colour(ref, -1 + (2 * i) / (RAMP_N - 1), 1)]
                     for i in range(RAMP_N)], dtype=np.uint8)
    assert np.array_equal(cb, want)


def test_ramp_measures_as_the_reference_recorded(swe):
    ramp, _ = swe.colourTables()
    exact = ramp_symmetry(ramp, 257, False)
    assert exact["worstAsym"] == pytest.approx(1.174e-4, abs=5e-8)
    assert exact["jump"] == 0 and exact["outOfGamut"] == 0
    eight = ramp_symmetry(ramp, 1025, True)
    assert eight["worstAsym"] == pytest.approx(0.4410, abs=5e-5)
    assert eight["span"] == pytest.approx(65.963, abs=5e-4)
    assert eight["jump"] == 0
