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
would wrap the slabs; the classes refuse such simulations with a
ValueError), and massFloored, volume() and the other
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
_FIELD_ID = {"h": 1, "hu": 2, "hv": 3}


def check_cuttable(sim):
    """Refuse a simulation whose south or north boundary is periodic: the
    slabs would wrap onto each other and the exchange would not be the
    grid's.  Simulations without a `boundaries` mapping are taken as given."""
    bounds = getattr(sim, "boundaries", None)
    if bounds is None:
        return
    for side in ("south", "north"):
        fn = bounds[side]
        if getattr(fn, "name", None) == "periodic":
            raise ValueError(f"row slabs: the {side} boundary is periodic, which a cut into row slabs "
                             "cannot keep; use reflect, outflow or flather there")


def _pack(sim, rows):
    r0, n = rows
    return np.concatenate([sim.get_rows(f, r0, n) for f in FIELDS])


def _unpack(sim, rows, data):
    r0, n = rows
    parts = np.split(np.asarray(data, dtype=np.float64), len(FIELDS))
    for f, part in zip(FIELDS, parts):
        sim.set_rows(f, r0, part)


# ---- the device data plane --------------------------------------------------
# A slab's halo rows and its dt stay on the GPU: rows are copied between the
# simulation and device buffers on the simulation's own stream
# (swe_get_rows_async / swe_set_rows_async), maxDt() goes to device memory
# (swe_max_dt_to), the minimum over the slabs is taken on the device, and the
# step reads its dt from there (swe_step_dt_from).  No host round trip per
# step; torch provides the streams, events, buffers and collectives.
class _DeviceSim:
    """The async C-ABI calls of one product simulation, and its stream."""

    def __init__(self, sim, torch):
        import ctypes
        self.sim, self.torch = sim, torch
        self.lib = sim._lib
        sp = ctypes.c_void_p()
        self._check(self.lib.swe_get_stream(sim._h, ctypes.byref(sp)))
        self.stream = torch.cuda.ExternalStream(sp.value)
        self.W = sim.W

    def _check(self, rc):
        from ._lib import check
        check(rc)

    def pack(self, rows, buf):
        """Rows (r0, n) of h, hu, hv into the device buffer `buf` (3 n W doubles)."""
        r0, n = rows
        self.sim._push()
        for q, f in enumerate(FIELDS):
            self._check(self.lib.swe_get_rows_async(self.sim._h, _FIELD_ID[f], r0, n,
                                                    buf.data_ptr() + 8 * q * n * self.W))

    def unpack(self, rows, buf):
        r0, n = rows
        for q, f in enumerate(FIELDS):
            self._check(self.lib.swe_set_rows_async(self.sim._h, _FIELD_ID[f], r0, n,
                                                    buf.data_ptr() + 8 * q * n * self.W))
        self.sim._stale(*FIELDS)

    def max_dt_to(self, out):
        self.sim._push()
        self._check(self.lib.swe_max_dt_to(self.sim._h, out.data_ptr()))

    def step_dt_from(self, dt):
        self._check(self.lib.swe_step_dt_from(self.sim._h, dt.data_ptr()))
        self.sim._stale("b", "h", "hu", "hv", "h0", "hu0", "hv0")


class LocalSlabs:
    """Several slabs of one grid stepped in one process: the halo exchange is
    a copy between the simulations.

    sims[k] is the simulation of slabs[k], made over slabs[k].rows rows with
    the slab's padded rows of every field (`Slab.take`); a simulation gives
    get_rows / set_rows / maxDt / step.  With device=True (product
    simulations on one GPU) the exchange and dt stay on the device: each
    slab packs its edge rows into a device buffer on its own stream, its
    neighbours unpack them after an event, the slabs' maxDt() go to a device
    array whose minimum each step then reads."""

    def __init__(self, slabs, sims, device=False):
        if len(slabs) != len(sims):
            raise ValueError("LocalSlabs: one simulation per slab")
        for sim in sims:
            check_cuttable(sim)
        self.slabs, self.sims = list(slabs), list(sims)
        self.device = bool(device)
        if self.device:
            import torch
            self._torch = torch
            self._dev = [_DeviceSim(sim, torch) for sim in self.sims]
            n = len(FIELDS) * HALO
            self._send = [(torch.empty(n * d.W, dtype=torch.float64, device="cuda") if s.south else None,
                           torch.empty(n * d.W, dtype=torch.float64, device="cuda") if s.north else None)
                          for s, d in zip(self.slabs, self._dev)]
            self._rates = torch.empty(len(self.sims), dtype=torch.float64, device="cuda")
            self._dt = torch.empty(1, dtype=torch.float64, device="cuda")

    def exchange(self):
        if self.device:
            return self._exchange_device()
        out = []
        for k, (sl, sim) in enumerate(zip(self.slabs, self.sims)):
            out.append((_pack(sim, sl.send_south()) if sl.south else None,
                        _pack(sim, sl.send_north()) if sl.north else None))
        for k, (sl, sim) in enumerate(zip(self.slabs, self.sims)):
            if sl.south:
                _unpack(sim, sl.recv_south(), out[k - 1][1])
            if sl.north:
                _unpack(sim, sl.recv_north(), out[k + 1][0])

    def _exchange_device(self):
        torch = self._torch
        packed = []
        for sl, d, (ss, sn) in zip(self.slabs, self._dev, self._send):
            with torch.cuda.stream(d.stream):
                if sl.south:
                    d.pack(sl.send_south(), ss)
                if sl.north:
                    d.pack(sl.send_north(), sn)
                packed.append(torch.cuda.Event())
                packed[-1].record(d.stream)
        for k, (sl, d) in enumerate(zip(self.slabs, self._dev)):
            with torch.cuda.stream(d.stream):
                if sl.south:
                    d.stream.wait_event(packed[k - 1])
                    d.unpack(sl.recv_south(), self._send[k - 1][1])
                if sl.north:
                    d.stream.wait_event(packed[k + 1])
                    d.unpack(sl.recv_north(), self._send[k + 1][0])

    def step(self):
        """One step of the grid: halos, the global maxDt(), every slab's step.
        Returns dt (a float; with device=True a one-element device tensor,
        read without a host round trip until the caller asks for it)."""
        self.exchange()
        if not self.device:
            dt = min(sim.maxDt() for sim in self.sims)
            for sim in self.sims:
                sim.step(dt)
            return dt
        torch = self._torch
        rated = []
        for k, d in enumerate(self._dev):
            with torch.cuda.stream(d.stream):
                d.max_dt_to(self._rates[k:k + 1])
                rated.append(torch.cuda.Event())
                rated[-1].record(d.stream)
        cur = torch.cuda.current_stream()
        for ev in rated:
            cur.wait_event(ev)
        torch.amin(self._rates, dim=0, keepdim=True, out=self._dt)
        chosen = torch.cuda.Event()
        chosen.record(cur)
        for d in self._dev:
            with torch.cuda.stream(d.stream):
                d.stream.wait_event(chosen)
                d.step_dt_from(self._dt)
        return self._dt

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

    device="cpu" (gloo): the messages are host tensors, staged through the
    C ABI's row copies.  device="cuda" (NCCL, one GPU per rank, the slab's
    simulation made on this rank's device): the device data plane -- rows
    packed into device buffers on the simulation's stream, NCCL moves them,
    the all-reduce of dt runs on the device and the step reads its dt from
    there, with no host round trip per step.  Each exchange posts all of
    its sends and receives as one batch (batch_isend_irecv), so no rank's
    send waits on a receive its peer has not posted."""

    def __init__(self, slab, sim, dist, group=None, device="cpu"):
        check_cuttable(sim)
        self.slab, self.sim, self.dist, self.group, self.device = slab, sim, dist, group, device
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self._dev = None
        if device != "cpu":
            import torch
            self._torch = torch
            self._dev = _DeviceSim(sim, torch)
            n = len(FIELDS) * HALO * sim.W
            mk = lambda: torch.empty(n, dtype=torch.float64, device=device)  # noqa: E731
            self._bufs = {"send_s": mk(), "send_n": mk(), "recv_s": mk(), "recv_n": mk()}
            self._dt = torch.empty(1, dtype=torch.float64, device=device)

    def _peer(self, side):
        return self.dist.get_global_rank(self.group, self.rank + side) if self.group is not None \
            else self.rank + side

    def exchange(self):
        if self._dev is not None:
            with self._torch.cuda.stream(self._dev.stream):
                return self._exchange_on(self._bufs)
        import torch
        sl, sim = self.slab, self.sim
        n = len(FIELDS) * HALO * sim.W
        bufs = {"send_s": torch.from_numpy(_pack(sim, sl.send_south())) if sl.south else None,
                "send_n": torch.from_numpy(_pack(sim, sl.send_north())) if sl.north else None,
                "recv_s": torch.empty(n, dtype=torch.float64) if sl.south else None,
                "recv_n": torch.empty(n, dtype=torch.float64) if sl.north else None}
        self._exchange_on(bufs)
        if sl.south:
            _unpack(sim, sl.recv_south(), bufs["recv_s"].numpy())
        if sl.north:
            _unpack(sim, sl.recv_north(), bufs["recv_n"].numpy())

    def _exchange_on(self, bufs):
        sl, dist = self.slab, self.dist
        dev = self._dev
        if dev is not None:
            if sl.south:
                dev.pack(sl.send_south(), bufs["send_s"])
            if sl.north:
                dev.pack(sl.send_north(), bufs["send_n"])
        ops = []
        if sl.south:
            ops += [dist.P2POp(dist.irecv, bufs["recv_s"], self._peer(-1), self.group),
                    dist.P2POp(dist.isend, bufs["send_s"], self._peer(-1), self.group)]
        if sl.north:
            ops += [dist.P2POp(dist.irecv, bufs["recv_n"], self._peer(+1), self.group),
                    dist.P2POp(dist.isend, bufs["send_n"], self._peer(+1), self.group)]
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        if dev is not None:
            if sl.south:
                dev.unpack(sl.recv_south(), bufs["recv_s"])
            if sl.north:
                dev.unpack(sl.recv_north(), bufs["recv_n"])

    def step(self):
        """One step of this rank's slab with the grid's dt.  Returns dt: a
        float on gloo, a one-element device tensor with NCCL (read without a
        host round trip until the caller asks for it)."""
        self.exchange()
        if self._dev is None:
            import torch
            t = torch.tensor([self.sim.maxDt()], dtype=torch.float64)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
            dt = float(t[0])
            self.sim.step(dt)
            return dt
        with self._torch.cuda.stream(self._dev.stream):
            self._dev.max_dt_to(self._dt)
            self.dist.all_reduce(self._dt, op=self.dist.ReduceOp.MIN, group=self.group)
            self._dev.step_dt_from(self._dt)
        return self._dt

    def owned(self, name):
        r0, n = self.slab.owned()
        return self.sim.get_rows(name, r0, n).reshape(n, -1)
