"""One grid cut into row slabs, each stepped by its own simulation (one per
GPU under torch.distributed, or several in one process).

The step (src/swe.mjs:754-814) is local: a stage changes a cell from the
state within 3 cells of it (slope -> face -> the upwind cell's positivity
limiter, src/swe.mjs:364-555), so a full SSP-RK2 step reaches 6 cells.  A
slab therefore holds its own interior rows plus HALO = 6 rows of each
neighbour.  Before every step the neighbours send each other the HALO rows
next to the cut; the slab then steps all of its rows with the global dt.
Its ghost rows at a cut are filled by its own boundary rule, and that
error, like the halo rows' missing neighbours, travels at most 3 rows per
stage: after the step it has reached the halo rows and no further, so
every owned row is the single grid's, bit for bit.

dt is the single grid's maxDt() (src/swe.mjs:632-647): cfl / (the largest
rate over wet interior cells).  At the start of a step a slab's interior
rows (owned + halo) hold the single grid's state, so the smallest of the
slabs' own maxDt() is cfl over the global largest rate, the same double
(cfl / x decreases with x and is correctly rounded).

On a spherical grid the metric differs row by row: a slab's simulation
takes the grid's own 13 metric rows over its padded rows (`copy_geometry`),
so that its arithmetic is the grid's, not that of a band recomputed from
its latitudes.

Limits: the global south and north boundaries may not be periodic (they
would wrap the slabs), and massFloored, volume() and the other
diagnostics of a slab count its halo rows too; take them from the owned
rows (`owned()`).  The cut is by rows, so each slab needs at least HALO
rows.
"""
import numpy as np

HALO = 6


def slab_rows(ny, n):
    """Interior rows [a, b) of each of n slabs of an ny-row grid: near-equal,
    the first ones one row longer."""
    if n < 1:
        raise ValueError("slab_rows: n >= 1")
    if ny < n * HALO:
        raise ValueError(f"slab_rows: {ny} rows cannot give {n} slabs of at least {HALO} rows")
    q, r = divmod(ny, n)
    out, a = [], 0
    for k in range(n):
        b = a + q + (1 if k < r else 0)
        out.append((a, b))
        a = b
    return out


class Slab:
    """Rows [a, b) of an ny-row grid, held with their halos.

    The slab's simulation covers interior rows [e0, e1) of the grid:
    e0 = max(0, a - HALO), e1 = min(ny, b + HALO); its padded row p is the
    grid's padded row p + e0 (both have two ghost rows on each side)."""

    def __init__(self, ny, a, b):
        if not (0 <= a < b <= ny) or b - a < HALO:
            raise ValueError(f"Slab: rows [{a}, {b}) of {ny} (at least {HALO} rows)")
        self.ny, self.a, self.b = ny, a, b
        self.e0, self.e1 = max(0, a - HALO), min(ny, b + HALO)
        self.rows = self.e1 - self.e0                # the slab simulation's ny
        self.south = a > 0                           # a neighbour below (lower rows)
        self.north = b < ny                          # a neighbour above

    def take(self, full):
        """The slab's padded rows of a grid field given as (ny + 4, W) or flat."""
        full = np.asarray(full, dtype=np.float64)
        W = full.size // (self.ny + 4)
        return np.ascontiguousarray(full.reshape(self.ny + 4, W)[self.e0:self.e1 + 4])

    # rows in the slab's padded indexing: (first row, count)
    def owned(self):
        return self.a - self.e0 + 2, self.b - self.a

    def send_south(self):
        return self.a - self.e0 + 2, HALO           # my lowest owned rows: the southern neighbour's upper halo

    def send_north(self):
        return self.b - HALO - self.e0 + 2, HALO    # my highest owned rows: the northern neighbour's lower halo

    def recv_south(self):
        return 2, self.a - self.e0                  # my lower halo

    def recv_north(self):
        return self.b - self.e0 + 2, self.e1 - self.b


GEOM_ROWS = ("dxRow", "dyRowN", "dyRowS", "dyCFL", "area", "lx", "lyN", "lyS", "bedPhi", "phiC", "tanPhi",
             "fRow", "geoCoef")


def copy_geometry(sim, slab, grid_geom):
    """Give a slab's simulation the grid's metric rows over the slab's padded
    rows (src/geometry.mjs:301-309); `grid_geom` is the grid's geometry
    object (or a mapping of row name to array)."""
    for name in GEOM_ROWS:
        full = grid_geom[name] if isinstance(grid_geom, dict) else getattr(grid_geom, name)
        getattr(sim.geom, name)[:] = np.asarray(full, dtype=np.float64)[slab.e0:slab.e1 + 4]


FIELDS = ("h", "hu", "hv")


def _pack(sim, rows):
    r0, n = rows
    return np.concatenate([sim.get_rows(f, r0, n) for f in FIELDS])


def _unpack(sim, rows, data):
    r0, n = rows
    parts = np.split(np.asarray(data, dtype=np.float64), len(FIELDS))
    for f, part in zip(FIELDS, parts):
        sim.set_rows(f, r0, part)


class LocalSlabs:
    """Several slabs of one grid stepped in one process (one device or the
    host): the halo exchange is a copy between the simulations.

    sims[k] is the simulation of slabs[k], made over slabs[k].rows rows with
    the slab's padded rows of every field (`Slab.take`); a simulation gives
    get_rows / set_rows / maxDt / step."""

    def __init__(self, slabs, sims):
        if len(slabs) != len(sims):
            raise ValueError("LocalSlabs: one simulation per slab")
        self.slabs, self.sims = list(slabs), list(sims)

    def exchange(self):
        out = []
        for k, (sl, sim) in enumerate(zip(self.slabs, self.sims)):
            out.append((_pack(sim, sl.send_south()) if sl.south else None,
                        _pack(sim, sl.send_north()) if sl.north else None))
        for k, (sl, sim) in enumerate(zip(self.slabs, self.sims)):
            if sl.south:
                _unpack(sim, sl.recv_south(), out[k - 1][1])
            if sl.north:
                _unpack(sim, sl.recv_north(), out[k + 1][0])

    def step(self):
        """One step of the grid: halos, the global maxDt(), every slab's step."""
        self.exchange()
        dt = min(sim.maxDt() for sim in self.sims)
        for sim in self.sims:
            sim.step(dt)
        return dt

    def gather(self, name):
        """The grid's interior rows of a field, from the slabs' owned rows
        ((ny, W); the ghost rows are each slab's own and are left out)."""
        parts = []
        for sl, sim in zip(self.slabs, self.sims):
            r0, n = sl.owned()
            parts.append(sim.get_rows(name, r0, n).reshape(n, -1))
        return np.concatenate(parts)


class DistributedSlab:
    """This rank's slab of a grid cut over the ranks of a torch.distributed
    group (rank k holds slab k): halos go to the neighbours by point-to-point
    messages, dt is the minimum of the ranks' maxDt() (all_reduce MIN).
    `device` is where the messages live: "cpu" for gloo, "cuda" for NCCL.
    On several GPUs each rank makes its slab's simulation on its own device
    (`swe_set_device(local rank)` before the handle is created)."""

    def __init__(self, slab, sim, dist, group=None, device="cpu"):
        self.slab, self.sim, self.dist, self.group, self.device = slab, sim, dist, group, device
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _tensor(self, a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def exchange(self):
        import torch
        sl, sim, dist = self.slab, self.sim, self.dist
        n = len(FIELDS) * HALO * sim.W
        reqs, recv = [], {}
        if sl.south:
            reqs.append(dist.isend(self._tensor(_pack(sim, sl.send_south())), self.rank - 1, group=self.group))
            recv["south"] = torch.empty(n, dtype=torch.float64, device=self.device)
            reqs.append(dist.irecv(recv["south"], self.rank - 1, group=self.group))
        if sl.north:
            reqs.append(dist.isend(self._tensor(_pack(sim, sl.send_north())), self.rank + 1, group=self.group))
            recv["north"] = torch.empty(n, dtype=torch.float64, device=self.device)
            reqs.append(dist.irecv(recv["north"], self.rank + 1, group=self.group))
        for r in reqs:
            r.wait()
        if "south" in recv:
            _unpack(sim, sl.recv_south(), recv["south"].cpu().numpy())
        if "north" in recv:
            _unpack(sim, sl.recv_north(), recv["north"].cpu().numpy())

    def step(self):
        self.exchange()
        t = self._tensor(np.array([self.sim.maxDt()], dtype=np.float64))
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        dt = float(t.cpu()[0])
        self.sim.step(dt)
        return dt

    def owned(self, name):
        r0, n = self.slab.owned()
        return self.sim.get_rows(name, r0, n).reshape(n, -1)
