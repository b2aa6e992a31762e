"""Structural rigs of the reference's verification suites, restated on the GPU.

Each rig's target is an exact identity or an analytic law of the equations,
so it needs no oracle: the solver under test (the CUDA library, through the
Python mirror of the C ABI) must meet it by itself.  Each test names the
reference rig it restates; the set-ups (grids, beds, states, step counts,
tolerances) are the rig's own, re-derived here.

  inertial oscillation   tools/verify-physics.mjs:140-212
  Manning spin-down      tools/verify-physics.mjs:221-310
  transpose symmetry     tools/verify-physics.mjs:710-766
  CFL formula            tools/verify-physics.mjs:1023-1059
  longitude rotation     tools/verify-sphere.mjs:1040-1078
  Flather absorption     tools/verify-tide.mjs:798-844
"""
import math

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

G_REF = 9.80665          # the test owns its constant (tools/verify.mjs:64-109)


def uniform(sim, h0, u0, v0):
    """Set every interior cell to (h0, h0 u0, h0 v0)."""
    h, hu, hv = sim.h, sim.hu, sim.hv
    for j in range(sim.ny):
        for i in range(sim.nx):
            k = sim.idx(i, j)
            h[k] = h0
            hu[k] = h0 * u0
            hv[k] = h0 * v0


def interior(sim, name):
    return np.asarray(sim.field(name)).reshape(sim.H, sim.W)[2:-2, 2:-2]


def non_uniformity(sim):
    m = 0.0
    for n in ("h", "hu", "hv"):
        a = interior(sim, n)
        m = max(m, float(np.max(np.abs(a - a[0, 0]))))
    return m


def test_constants_match(swe):
    assert swe.G == G_REF


# --------------------------------------------------------------- inertial circle
def test_inertial_oscillation(swe):
    """f-plane: a uniform current turns clockwise at f with no pressure
    gradient; period 2 pi / f to 1e-5, speed kept to 1e-7, the state exactly
    uniform, the trajectory a circle of radius U / f to 1e-4."""
    f, h0, U, N = 1e-4, 10.0, 0.5, 2000
    T = 2 * math.pi / f
    dt = T / N
    sim = swe.ShallowWater(nx=8, ny=8, dx=5000, bed=lambda x, y: -h0, eta0=0, manning=0, coriolis=f)
    sim.boundaries = {s: swe.periodic for s in ("west", "east", "south", "north")}
    uniform(sim, h0, U, 0.0)
    assert dt < sim.maxDt()
    k0 = sim.idx(4, 4)

    def uv():
        h = sim.field("h")[k0]
        return sim.vel(sim.field("hu")[k0], h), sim.vel(sim.field("hv")[k0], h)

    pu, pv = uv()
    spd0 = math.hypot(pu, pv)
    px = py = 0.0
    traj = [(0.0, 0.0)]
    ang, prev, quarter_v = 0.0, math.atan2(pv, pu), None
    for n in range(N):
        sim.step(dt)
        u, v = uv()
        px += 0.5 * (pu + u) * dt
        py += 0.5 * (pv + v) * dt
        traj.append((px, py))
        pu, pv = u, v
        d = math.atan2(v, u) - prev
        while d > math.pi:
            d -= 2 * math.pi
        while d < -math.pi:
            d += 2 * math.pi
        ang += d
        prev = math.atan2(v, u)
        if n == N // 4 - 1:
            quarter_v = v
    assert non_uniformity(sim) == 0
    period = T * 2 * math.pi / abs(ang)
    assert abs(period - T) <= 1e-5 * T
    assert ang < 0                                   # clockwise for f > 0
    assert abs(quarter_v + U) <= 2e-3 * U
    spd1 = math.hypot(*uv())
    assert abs(spd1 - spd0) <= 1e-7 * spd0
    tr = np.array(traj)
    c = tr.mean(axis=0)
    r = np.hypot(tr[:, 0] - c[0], tr[:, 1] - c[1])
    assert abs(0.5 * (r.min() + r.max()) - U / f) <= 1e-4 * U / f


# --------------------------------------------------------------- spin-down
@pytest.mark.parametrize("h0,n,u0", [(0.2, 0.05, 3.0), (1.5, 0.03, 2.0)])
def test_manning_spin_down_identity(swe, h0, n, u0):
    """The semi-implicit friction telescopes: 1/u - 1/u0 = g n^2 t / h^(4/3)
    for any dt, to round-off (1e-10 relative over 200 self-timed steps)."""
    A = G_REF * n * n / h0 ** (4.0 / 3.0)
    sim = swe.ShallowWater(nx=8, ny=4, dx=5, bed=lambda x, y: 0, eta0=h0, manning=n)
    sim.boundaries = {s: swe.periodic for s in ("west", "east", "south", "north")}
    uniform(sim, h0, u0, 0.0)
    k = sim.idx(3, 2)
    worst = 0.0
    for _ in range(200):
        assert sim.step() > 0
        u = sim.vel(sim.field("hu")[k], sim.field("h")[k])
        worst = max(worst, abs((1 / u - 1 / u0) - A * sim.t) / (A * sim.t))
    assert worst <= 1e-10, worst
    assert np.all(interior(sim, "h") == h0)


def test_manning_explicit_update_would_fail_the_identity():
    """Refutation on the host: an explicit friction update misses the
    identity by far more than the tolerance, so the check can see it."""
    h0, n, u0, dt = 0.2, 0.05, 3.0, 0.05
    A = G_REF * n * n / h0 ** (4.0 / 3.0)
    u, t = u0, 0.0
    worst = 0.0
    for _ in range(200):
        u = u - dt * A * abs(u) * u
        t += dt
        worst = max(worst, abs((1 / u - 1 / u0) - A * t) / (A * t))
    assert worst > 1e-3


# --------------------------------------------------------------- transpose
def _transpose_run(swe, T, dts=None, n=64, d=6, steps=200):
    def bedA(x, y):
        return (-6 + 1.8 * math.sin(x * 0.011) + 1.1 * math.cos(y * 0.019)
                + 2.2 * math.exp(-(((x - 150) / 70) ** 2) - (((y - 260) / 50) ** 2)))

    def etaA(x, y):
        return (0.4 * math.exp(-(((x - 90) / 60) ** 2) - (((y - 300) / 90) ** 2))
                - 0.25 * math.exp(-(((x - 320) / 80) ** 2) - (((y - 120) / 70) ** 2)))

    sim = swe.ShallowWater(nx=n, ny=n, dx=d, dy=d, bed=(lambda x, y: bedA(y, x)) if T else bedA,
                           eta0=(lambda x, y: etaA(y, x)) if T else etaA, manning=0.02)
    h, hu, hv = sim.h, sim.hu, sim.hv
    for j in range(n):
        for i in range(n):
            k = sim.idx(i, j)
            x = (j + 0.5) * d if T else (i + 0.5) * d
            y = (i + 0.5) * d if T else (j + 0.5) * d
            u, v = 0.6 * math.sin(x * 0.008), -0.35 * math.cos(y * 0.013)
            hu[k] = h[k] * (v if T else u)
            hv[k] = h[k] * (u if T else v)
    out = []
    if dts is None:
        for _ in range(steps):
            out.append(sim.step())
    else:
        for dt in dts:
            sim.step(dt)
    return sim, out


def test_transpose_symmetry(swe):
    """The same problem mirrored about y = x, driven with run A's dt
    sequence, is the transpose of run A to summation order: depth 1e-12,
    momentum 1e-11; without transposing the runs differ by > 1 cm."""
    A, dts = _transpose_run(swe, False)
    B, _ = _transpose_run(swe, True, dts=dts)
    hA, huA, hvA = (interior(A, f) for f in ("h", "hu", "hv"))
    hB, huB, hvB = (interior(B, f) for f in ("h", "hu", "hv"))
    plain = float(np.max(np.abs(hA - hB)))
    dh = float(np.max(np.abs(hA - hB.T)))
    dm = max(float(np.max(np.abs(huA - hvB.T))), float(np.max(np.abs(hvA - huB.T))))
    assert plain > 0.01
    assert dh <= 1e-12, dh
    assert dm <= 1e-11, dm


# --------------------------------------------------------------- CFL formula
@pytest.mark.parametrize("dx,dy", [(7, 11), (11, 7)])
def test_cfl_formula(swe, dx, dy):
    """maxDt = cfl / ((|u| + c)/dx + (|v| + c)/dy) to 1e-14 -- the sum of the
    two directions, not their maximum."""
    h0, u0, v0 = 3.0, 1.7, -0.9
    sim = swe.ShallowWater(nx=6, ny=5, dx=dx, dy=dy, bed=lambda x, y: -h0, eta0=0, manning=0)
    uniform(sim, h0, u0, v0)
    c = math.sqrt(G_REF * h0)
    want = sim.cfl / ((abs(u0) + c) / dx + (abs(v0) + c) / dy)
    mx = sim.cfl / max((abs(u0) + c) / dx, (abs(v0) + c) / dy)
    assert abs(sim.maxDt() - want) <= 1e-14 * want
    assert abs(mx - want) > 0.5 * want                 # the control is far away


def test_cfl_ignores_cells_at_or_below_min_depth(swe):
    h0, u0, v0, dx, dy = 3.0, 1.7, -0.9, 7, 11
    sim = swe.ShallowWater(nx=6, ny=5, dx=dx, dy=dy, bed=lambda x, y: -h0, eta0=0, manning=0)
    uniform(sim, h0, u0, v0)
    dt0 = sim.maxDt()
    k, hd = sim.idx(2, 2), 0.9 * sim.minDepth
    h, hu, hv = sim.h, sim.hu, sim.hv
    h[k], hu[k], hv[k] = hd, hd * 100, 0.0
    assert sim.maxDt() == dt0


# --------------------------------------------------------------- rotation
def _rotated(swe, deg, shift, steps=200):
    def bed_of(sh):
        return lambda lon, lat: S.bed_uneven(S.wrap180(lon - sh), lat)

    def eta_of(sh):
        def f(lon, lat):
            L = S.wrap180(lon - sh)
            return 2 * math.exp(-(S.wrap180(L - 40) ** 2 + (lat - 25) ** 2) / 200)
        return f

    A = S.sphere(swe.ShallowWater, bed_of(0.0), deg, eta0=eta_of(0.0), omega=S.OMEGA_REF)
    B = S.sphere(swe.ShallowWater, bed_of(shift * deg), deg, eta0=eta_of(shift * deg), omega=S.OMEGA_REF)
    dt = min(A.maxDt(), B.maxDt())
    assert A.run(steps, dt=dt) == steps and B.run(steps, dt=dt) == steps
    out = {}
    for f in ("h", "hu", "hv"):
        a, b = interior(A, f), interior(B, f)
        out[f] = (a, np.roll(b, -shift, axis=1))
    return out


def test_longitude_rotation_bit_identity(swe):
    """A 4-degree grid rotated by 23 cells (92 degrees, across the
    antimeridian): after 200 steps every cell is the same double as the
    unrotated run's -- the solver does not know where longitude 0 is."""
    r = _rotated(swe, 4, 23)
    for f, (a, b) in r.items():
        assert np.array_equal(a, b), f"{f}: max |d| = {np.max(np.abs(a - b))}"
    assert np.max(r["h"][0]) > 1000                  # an ocean, not an empty grid


def test_longitude_rotation_inexact_shift_bounded(swe):
    """3.6-degree cells: the shift is not exact in binary, so the two runs
    differ by round-off only (depth within 1e-11 of the largest depth)."""
    r = _rotated(swe, 3.6, 23)
    a, b = r["h"]
    assert float(np.max(np.abs(a - b))) / float(np.max(a)) <= 1e-11


# --------------------------------------------------------------- Flather
def _pulse_reflection(swe, bc):
    h, L, nx = 30.0, 60000.0, 600
    dx = L / nx
    sim = swe.ShallowWater(nx=nx, ny=1, dx=dx, bed=lambda x, y: -h, eta0=0, manning=0, cfl=0.4)
    c0 = math.sqrt(G_REF * h)
    A, x0, sig = 0.1, 20000.0, 2500.0
    hh, hu = sim.h, sim.hu
    for i in range(nx):
        x = (i + 0.5) * dx
        e = A * math.exp(-(((x - x0) / sig) ** 2))
        k = sim.idx(i, 0)
        hh[k] = h + e
        hu[k] = c0 * e                               # a purely right-going pulse
    sim.boundaries = {"west": swe.reflect, "east": bc, "south": swe.periodic, "north": swe.periodic}
    T = 1.9 * (L - x0) / c0
    sim.run(100000, tEnd=T)
    assert abs(sim.t - T) <= 1e-9 * T
    eta = interior(sim, "b")[0] + interior(sim, "h")[0]
    return float(np.max(np.abs(eta[10:nx - 40]))) / A


def test_flather_absorbs_normal_incidence(swe):
    """A long-wave pulse at normal incidence leaves through a Flather
    boundary (< 0.5 % returns) and bounces off a wall (> 50 %)."""
    r_flather = _pulse_reflection(swe, swe.flather(swe.Tide({}, msl=0.0).signal()))
    r_wall = _pulse_reflection(swe, swe.reflect)
    assert r_flather < 0.005, r_flather
    assert r_wall > 0.5, r_wall
