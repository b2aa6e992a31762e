"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset exists for this path; every benchmark input is generated here
from a seed, so the same arrays are produced wherever it runs.
"""
import math

import numpy as np


def uniform_noise(seed, shape, lo, hi):
    """U(lo, hi) per cell from a counter-based hash (splitmix64 of seed, k)."""
    n = int(np.prod(shape))
    k = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = k + np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    return (lo + (hi - lo) * u).reshape(shape)


def _centres(nx, ny, dx, dy=None):
    dy = dx if dy is None else dy
    x = (np.arange(nx + 4) - 2 + 0.5) * dx
    y = (np.arange(ny + 4) - 2 + 0.5) * dy
    return np.meshgrid(x, y)


def bump_bed(nx, ny, dx, seed=1, height=1.5, sigma=40.0, rough=0.2):
    """Gaussian bump (height 1.5 m, sigma 40 m) at the domain centre plus
    seeded uniform roughness +/- 0.2 m, over the padded grid."""
    X, Y = _centres(nx, ny, dx)
    cx, cy = nx * dx / 2, ny * dx / 2
    b = height * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sigma * sigma))
    return b + uniform_noise(seed, X.shape, -rough, rough)


def beach_bed(nx, ny, dx, seed=2):
    """Sloping beach 1:50 plus smooth noise of amplitude 0.3 m:
    b = -10 + x/50 + 0.3 s(x, y), s the mean of 8 seeded plane sinusoids with
    wavelengths in [100, 1000] m (|s| <= 1)."""
    X, Y = _centres(nx, ny, dx)
    rng = np.random.default_rng(seed)
    s = np.zeros_like(X)
    for _ in range(8):
        lam = rng.uniform(100, 1000)
        ang = rng.uniform(0, 2 * math.pi)
        ph = rng.uniform(0, 2 * math.pi)
        kx, ky = 2 * math.pi / lam * math.cos(ang), 2 * math.pi / lam * math.sin(ang)
        s += np.sin(kx * X + ky * Y + ph)
    s /= 8
    return -10 + X / 50 + 0.3 * s


def _jmax0(d):
    return np.where(d > 0, d, np.where(np.isnan(d), d, 0.0))


def beach_dam_break(nx=2048, ny=2048, dx=2.0, seed=2, eta_left=5.0, x_dam=500.0):
    """The 2048 x 2048 wet/dry workload: dam break over the sloping beach,
    water at eta = 5 m for x < 500 m, dry land beyond (eta = 0 there, and the
    bed rises above 0 at x ~ 500 m).  Returns (b, h) over the padded grid.
    Manning n = 0.03, Flather(0, 0) on the west side, walls elsewhere."""
    b = beach_bed(nx, ny, dx, seed)
    X, _ = _centres(nx, ny, dx)
    eta = np.where(X < x_dam, eta_left, 0.0)
    return b, _jmax0(eta - b)


def bump_dam_break(nx=256, ny=256, dx=5.0, seed=1, still=False):
    """The plain 256 x 256 workload: bump + roughness under still water at
    eta = 2 m, or the dam-break variant (2 m left half, 0.5 m right half).
    Returns (b, eta0) over the padded grid."""
    b = bump_bed(nx, ny, dx, seed)
    X, _ = _centres(nx, ny, dx)
    eta = np.full_like(X, 2.0) if still else np.where(X < nx * dx / 2, 2.0, 0.5)
    return b, eta


def ensemble(n=256, seed=4, dx=5.0, amp=0.5, eta=2.0):
    """The batched-ensemble workload: n independent Cartesian basins of
    seeded uneven sizes, nx ~ U[64, 1024], ny ~ U[64, 512], each with its own
    bump-and-roughness bed (seeded per basin), still water at eta = 2 m,
    Manning n ~ U[0.015, 0.04] and a west Flather tide of amplitude 0.5 m
    (not given by the configuration; stated here) and period ~ U[2, 14] h.
    Returns a list of dicts: nx, ny, dx, b, eta0, manning, tide (msl, amp,
    omega, phase_deg)."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nx = int(rng.integers(64, 1025))
        ny = int(rng.integers(64, 513))
        manning = float(rng.uniform(0.015, 0.04))
        period_h = float(rng.uniform(2.0, 14.0))
        b = bump_bed(nx, ny, dx, seed=1000 + q)
        out.append({"nx": nx, "ny": ny, "dx": dx, "b": b, "eta0": np.full_like(b, eta),
                    "manning": manning,
                    "tide": {"msl": eta, "amp": [amp], "omega": [2 * math.pi / (period_h * 3600)],
                             "phase_deg": [0.0]}})
    return out


def adjoint_case(nx=1024, ny=1024, dx=10.0, n_gauges=32, seed=5, hump=0.5, noise=0.1, manning_lo=0.015,
                 manning_hi=0.04):
    """The adjoint workload: a bump-and-roughness bed (bump 1.5 m high,
    sigma 40 cells, roughness +/- 0.2 m) under still water at 2 m with a
    released Gaussian hump of `hump` m (sigma 25 cells) to set it moving;
    a per-cell Manning field ~ U[0.015, 0.04]; n_gauges seeded interior
    gauge cells; and the 'true' bed b + N(0, noise) that makes the synthetic
    observations.  Returns a dict with padded arrays b, b_true, eta0, n and
    the gauge indices k = j*W + i."""
    rng = np.random.default_rng(seed)
    W, H = nx + 4, ny + 4
    X, Y = _centres(nx, ny, dx)
    cx, cy = nx * dx / 2, ny * dx / 2
    s = 40 * dx
    b = 1.5 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s)) + uniform_noise(seed, X.shape, -0.2, 0.2)
    sh = 25 * dx
    hx, hy = 0.3 * nx * dx, 0.6 * ny * dx
    eta0 = 2.0 + hump * np.exp(-((X - hx) ** 2 + (Y - hy) ** 2) / (2 * sh * sh))
    n = rng.uniform(manning_lo, manning_hi, X.shape)
    gi = rng.integers(2, nx + 2, n_gauges)
    gj = rng.integers(2, ny + 2, n_gauges)
    gauges = (gj * W + gi).astype(np.int32)
    b_true = b + rng.normal(0.0, noise, X.shape)
    return {"nx": nx, "ny": ny, "dx": dx, "b": b, "b_true": b_true, "eta0": eta0, "n": n, "gauges": gauges}


def _legendre(n, x):
    """P_n(x) by Bonnet's recurrence (n + 1) P_{n+1} = (2n + 1) x P_n - n P_{n-1}."""
    p0, p1 = np.ones_like(x), x
    if n == 0:
        return p0
    for k in range(1, n):
        p0, p1 = p1, ((2 * k + 1) * x * p1 - k * p0) / (k + 1)
    return p1


def globe_tide(nx=1440, ny=720, lat0=-85.0, lat1=85.0, seed=3, land=0.30, depth=5000.0, land_height=50.0,
               modes=48):
    """The spherical tide workload: 1440 x 720 cells on the lat-lon grid
    (0.25 degrees in longitude) over the band lat0..lat1, whose south and
    north edges are the open boundaries the tide enters through (the whole
    sphere has none: longitude is periodic and the pole faces have zero
    length).  Bed: band-limited spherical noise, the sum of `modes` seeded
    terms P_k(sin lat) cos(m lon + p) with degrees k and zonal wavenumbers
    m in 1..12 (periodic across the seam), scaled so the ocean spans depths
    0..`depth` m; the `land` fraction of highest cells is land at
    +`land_height` m.  Still water at 0.  Returns padded arrays b, eta0 and
    the cell centres (lon, lat) in degrees, longitude wrapped into
    [-180, 180) as cellLonLat does."""
    W, H = nx + 4, ny + 4
    dlon, dlat = 360.0 / nx, (lat1 - lat0) / ny
    lon = -180.0 + (np.arange(W) - 2 + 0.5) * dlon
    lon = (lon + 180.0) % 360.0 - 180.0
    lat = lat0 + (np.arange(H) - 2 + 0.5) * dlat
    lam, mu = np.radians(lon), np.sin(np.radians(np.clip(lat, -90.0, 90.0)))
    rng = np.random.default_rng(seed)
    v = np.zeros((H, W))
    for _ in range(modes):
        m, k = int(rng.integers(1, 13)), int(rng.integers(1, 13))
        a = rng.normal(0.0, 1.0) / math.sqrt(m * m + k * k)
        p = rng.uniform(0, 2 * math.pi)
        v += a * np.outer(_legendre(k, mu), np.cos(m * lam + p))
    inner = v[2:-2, 2:-2]
    thr = float(np.quantile(inner, 1.0 - land))
    vmin = float(inner.min())
    b = np.where(v > thr, land_height, -depth * (thr - v) / (thr - vmin))
    eta0 = np.zeros((H, W))
    LON, LAT = np.meshgrid(lon, lat)
    return {"nx": nx, "ny": ny, "lat0": lat0, "lat1": lat1, "b": b, "eta0": eta0, "lon": LON, "lat": LAT}
