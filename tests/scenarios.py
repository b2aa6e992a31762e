"""Fixtures restated from the reference's verification suites (test data only).

Each helper names the reference lines it follows.  They build either the
product (`water_simulator_b200.ShallowWater`) or the oracle (`OracleSim`),
whichever class is passed as `cls`.
"""
import math

import numpy as np

G_REF = 9.80665
R_REF = 6371000.0
OMEGA_REF = 7.292115e-5
H_OCEAN = 4000.0
D = math.pi / 180
EPS = 2.220446049250313e-16


def wrap180(x):                      # tools/verify-sphere.mjs:158
    return math.fmod(math.fmod(x + 180, 360) + 360, 360) - 180


def bed_flat(lon, lat):              # tools/verify-sphere.mjs:161
    return -H_OCEAN


def bed_uneven(lon, lat):            # tools/verify-sphere.mjs:167-168
    return -H_OCEAN + 900 * math.sin(3 * lon * D) * math.cos(2 * lat * D) + 350 * math.sin(5 * lat * D)


def bed_piercing(lon, lat):          # tools/verify-sphere.mjs:174-177
    dl, dp = wrap180(lon - 30), lat - 20
    return bed_uneven(lon, lat) + 5000 * math.exp(-(dl * dl + dp * dp) / 128)


SPHERE_BEDS = {"flat": bed_flat, "uneven": bed_uneven, "piercing": bed_piercing}


def sphere(cls, bed, deg, eta0=0.0, lat0=-90, lat1=90, order=2, omega=0.0, cfl=0.45, **kw):
    """tools/verify-sphere.mjs:178-184"""
    nx, ny = round(360 / deg), round((lat1 - lat0) / deg)
    return cls(nx=nx, ny=ny, bed=bed, eta0=eta0, manning=0, cfl=cfl, order=order,
               sphere={"R": R_REF, "lat0": lat0, "lat1": lat1, "omega": omega}, **kw)


def dry_cells(sim):                  # tools/verify-sphere.mjs:185-189
    h = np.asarray(sim.field("h")).reshape(sim.H, sim.W)[2:-2, 2:-2]
    return int(np.count_nonzero(h <= sim.minDepth))


def legendre(n, x):                  # tools/verify-sphere.mjs:666-671
    p0, p1 = 1.0, x
    if n == 0:
        return 1.0
    for k in range(1, n):
        p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1)
        p0, p1 = p1, p2
    return p1


def merian(cls, n, deg, run_steps=None):
    """Period of the n-th zonal free mode of a flat 4000 m ocean
    (tools/verify-sphere.mjs:673-720).  run_steps(sim, dt, k) may advance k
    steps at once; the projection is sampled after every step."""
    omega = math.sqrt(G_REF * H_OCEAN * n * (n + 1) / (R_REF * R_REF))
    Tclosed = 2 * math.pi / omega
    sim = sphere(cls, bed_flat, deg, eta0=lambda lon, lat: legendre(n, math.sin(lat * D)))
    nx, ny = sim.nx, sim.ny
    area = np.asarray(sim.geom.area)
    pn = np.array([legendre(n, math.sin(sim.cellLonLat(0, j)[1] * D)) for j in range(ny)])
    w = pn * area[2:2 + ny]

    def proj():
        eta = (np.asarray(sim.field("b")) + np.asarray(sim.field("h"))).reshape(sim.H, sim.W)[2:-2, 2:-2]
        rows = np.cumsum(eta, axis=1)[:, -1]      # left-to-right running sums
        s = 0.0
        for j in range(ny):
            s += rows[j] * w[j]
        return s

    dt = sim.maxDt()
    tEnd = 1.3 * Tclosed
    zeros = []
    prev, tprev = proj(), 0.0
    t = 0.0
    while t < tEnd:
        sim.step(dt)
        t = sim.t
        c = proj()
        if (prev > 0 and c <= 0) or (prev < 0 and c >= 0):
            zeros.append(tprev + (t - tprev) * prev / (prev - c))
        prev, tprev = c, t
    T = 2 * (zeros[-1] - zeros[0]) / (len(zeros) - 1)
    return {"n": n, "deg": deg, "Tclosed": Tclosed, "T": T, "errPct": 100 * (T - Tclosed) / Tclosed,
            "steps": sim.steps}


LAKE_BEDS = {                        # tools/verify.mjs:124-129
    "smooth bump": lambda x: 0.8 * math.exp(-(((x - 500) / 120) ** 2)),
    "sharp step": lambda x: 1.2 if (480 < x < 620) else 0.1,
    "random rough": lambda x: 0.6 * (math.sin(x * 0.031) + math.sin(x * 0.0173) * math.cos(x * 0.0077)),
    "island (pierces)": lambda x: 2.6 * math.exp(-(((x - 500) / 90) ** 2)),
}


def lake(cls, name):
    """200 x 4 lake at eta = 2 m, walls W/E, periodic S/N (tools/verify.mjs:130-136)."""
    bf = LAKE_BEDS[name]
    return cls(nx=200, ny=4, dx=5, bed=lambda x, y: bf(x) + 0.15 * math.sin(y * 0.05), eta0=2.0, manning=0)


from water_simulator_b200.workloads import uniform_noise, bump_bed, beach_bed  # noqa: E402,F401
