"""One grid cut into row slabs (water-simulator_b200/slabs.py) steps bit for
bit like the grid itself: on the oracle in one process and over two `gloo`
ranks (CPU), and on the GPU with three slab handles in one process.  The
case moves across every cut: standing waves over a beach that rises to
the north (dry land over the last rows), Manning friction, Coriolis, and a
Flather boundary with a time-varying level on the west side."""
import json
import math
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NX, NY, DX = 24, 60, 5.0
STEPS = 25


def _slabs():
    sys.path.insert(0, ROOT)
    import __graft_entry__
    __graft_entry__.load_package()
    from water_simulator_b200 import slabs
    return slabs


def case(ny=NY):
    W, H = NX + 4, ny + 4
    rng = np.random.default_rng(5)
    y = (np.arange(H) - 2 + 0.5) * DX
    x = (np.arange(W) - 2 + 0.5) * DX
    b = (-2.0 + y / 125.0)[:, None] + 0.3 * np.exp(-((x[None, :] - 60) ** 2 + (y[:, None] - 120) ** 2) / 800.0)
    b = b + rng.uniform(-0.05, 0.05, (H, W))
    eta = 0.25 * np.sin(2 * np.pi * x / 60.0)[None, :] * np.cos(2 * np.pi * y / 80.0)[:, None]
    return b, eta


def eta_ext(t):
    return 0.1 * math.sin(2 * math.pi * t / 30.0)


def u_ext(t):
    return 0.0


KW = dict(dx=DX, manning=0.02, coriolis=1e-4)
BOUNDS = dict(west=("flather", eta_ext, u_ext), east="reflect", south="reflect", north="reflect")


class OracleRows:
    """The oracle with the row access of the product's simulation."""

    def __init__(self, **kw):
        from oracle_sim import OracleSim
        self.sim = OracleSim(**kw)
        self.W, self.H = self.sim.W, self.sim.H

    def get_rows(self, name, r0, n):
        return getattr(self.sim, name)[r0 * self.W:(r0 + n) * self.W].copy()

    def set_rows(self, name, r0, v):
        getattr(self.sim, name)[r0 * self.W:r0 * self.W + np.asarray(v).size] = v

    def maxDt(self):
        return self.sim.maxDt()

    def step(self, dt):
        return self.sim.step(dt)


def oracle_grid(ny, b, eta):
    o = OracleRows(nx=NX, ny=ny, bed=b, eta0=eta, **KW)
    o.sim.set_boundaries(**BOUNDS)
    return o


def reference_rows(steps=STEPS, ny=NY):
    """The grid itself on the oracle: its interior rows after `steps` and t."""
    b, eta = case(ny)
    ref = oracle_grid(ny, b, eta)
    for _ in range(steps):
        ref.step(ref.maxDt())
    out = {f: ref.get_rows(f, 2, ny).reshape(ny, -1) for f in ("h", "hu", "hv")}
    return out, ref.sim.t


def test_slab_rows_and_halos():
    sl = _slabs()
    assert sl.slab_rows(100, 3) == [(0, 34), (34, 67), (67, 100)]
    s = sl.Slab(100, 34, 67)
    assert (s.e0, s.e1, s.rows) == (28, 73, 45)
    assert s.owned() == (8, 33)
    assert s.send_south() == (8, 6) and s.send_north() == (35, 6)
    assert s.recv_south() == (2, 6) and s.recv_north() == (41, 6)
    edge = sl.Slab(100, 0, 34)
    assert (edge.south, edge.north, edge.e0, edge.recv_north()) == (False, True, 0, (36, 6))
    with pytest.raises(ValueError):
        sl.slab_rows(10, 2)                      # slabs shorter than the halo
    with pytest.raises(ValueError):
        sl.Slab(100, 10, 14)


def test_local_slabs_match_one_grid_on_the_oracle():
    sl = _slabs()
    b, eta = case()
    want, t_want = reference_rows()
    parts = sl.slab_rows(NY, 3)
    slabs = [sl.Slab(NY, a, c) for a, c in parts]
    sims = [oracle_grid(s.rows, s.take(b), s.take(eta)) for s in slabs]
    run = sl.LocalSlabs(slabs, sims)
    for _ in range(STEPS):
        run.step()
    for f in ("h", "hu", "hv"):
        got = run.gather(f)
        assert np.array_equal(got.view(np.uint64), want[f].view(np.uint64)), f
    assert all(s.sim.t == t_want for s in sims)
    # water moves across both cuts (rows 20 and 40), and the last rows are dry land
    hv = want["hv"][:, 2:-2]
    assert np.all(hv[14:46] != 0)
    assert np.count_nonzero(want["h"][NY - 4:, 2:-2] == 0) > 0


def test_slabs_as_short_as_the_halo():
    """Four slabs of 6 rows: each halo is a whole neighbouring slab, and the
    inner slabs' halos reach the grid's own walls."""
    sl = _slabs()
    ny = 24
    b, eta = case(ny)
    want, t_want = reference_rows(ny=ny)
    slabs = [sl.Slab(ny, a, c) for a, c in sl.slab_rows(ny, 4)]
    assert [s.b - s.a for s in slabs] == [6, 6, 6, 6]
    run = sl.LocalSlabs(slabs, [oracle_grid(s.rows, s.take(b), s.take(eta)) for s in slabs])
    for _ in range(STEPS):
        run.step()
    for f in ("h", "hu", "hv"):
        assert np.array_equal(run.gather(f).view(np.uint64), want[f].view(np.uint64)), f
    assert all(s.sim.t == t_want for s in run.sims)


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sl = _slabs()
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b, eta = case()
    a, c = sl.slab_rows(NY, world)[rank]
    slab = sl.Slab(NY, a, c)
    run = sl.DistributedSlab(slab, oracle_grid(slab.rows, slab.take(b), slab.take(eta)), dist)
    dts = [run.step() for _ in range(STEPS)]
    out = {f: run.owned(f).tolist() for f in ("h", "hu", "hv")}
    with open(os.path.join(out_dir, f"slab{rank}.json"), "w") as fh:
        json.dump({"rows": [a, c], "dts": dts, "fields": out}, fh)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_step_one_grid(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    want, _ = reference_rows()
    res = [json.load(open(tmp_path / f"slab{r}.json")) for r in range(world)]
    assert res[0]["dts"] == res[1]["dts"]
    for f in ("h", "hu", "hv"):
        got = np.concatenate([np.array(r["fields"][f]) for r in res])
        assert np.array_equal(got, want[f]), f


@pytest.mark.gpu
def test_local_slabs_match_one_grid_on_the_gpu():
    """Three slab handles on one GPU against one handle of the whole grid,
    bit for bit (uint64 patterns) after every step."""
    sl = _slabs()
    import __graft_entry__
    swe = __graft_entry__.load_package()
    b, eta = case()

    def make(ny, bb, ee):
        sim = swe.ShallowWater(nx=NX, ny=ny, bed=bb, eta0=ee, **KW)
        sim.boundaries = {"west": swe.flather(eta_ext, u_ext), "east": swe.reflect,
                          "south": swe.reflect, "north": swe.reflect}
        return sim

    whole = make(NY, b, eta)
    slabs = [sl.Slab(NY, a, c) for a, c in sl.slab_rows(NY, 3)]
    run = sl.LocalSlabs(slabs, [make(s.rows, s.take(b), s.take(eta)) for s in slabs])
    for step in range(STEPS):
        dt = run.step()
        assert whole.maxDt() == dt
        whole.step(dt)
        for f in ("h", "hu", "hv"):
            got = run.gather(f)
            want = whole.get_rows(f, 2, NY).reshape(NY, -1)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (step, f)
    for sim in run.sims + [whole]:
        sim.close()


# ---- a spherical band: every row has its own metric ------------------------
SNX, SNY, LAT0, LAT1 = 36, 48, -60.0, 60.0
SPHERE = {"R": 6371e3, "lat0": LAT0, "lat1": LAT1, "omega": 7.2921e-5}


def sphere_case():
    """Still water 0-4000 m deep over a bed with a continent (land at +50 m)
    in the northern slab, a released hump across the southern cut, Coriolis
    on; walls at the band's edges, longitude periodic."""
    W, H = SNX + 4, SNY + 4
    lon = (np.arange(W) - 2 + 0.5) * (360.0 / SNX)
    lat = LAT0 + (np.arange(H) - 2 + 0.5) * ((LAT1 - LAT0) / SNY)
    L, P = np.meshgrid(lon, lat)
    b = -4000.0 + 1500.0 * np.sin(np.radians(2 * L)) * np.cos(np.radians(3 * P))
    b = np.where((P > 25) & (L > 60) & (L < 140), 50.0, b)
    eta = 2.0 * np.exp(-((L - 200.0) ** 2 + (P + 20.0) ** 2) / 200.0)
    return b, eta


def sphere_bounds(**extra):
    return dict(west="periodic", east="periodic", south="reflect", north="reflect", **extra)


def band(slab):
    dphi = (LAT1 - LAT0) / SNY
    return dict(SPHERE, lat0=LAT0 + slab.e0 * dphi, lat1=LAT0 + slab.e1 * dphi)


def test_local_slabs_match_one_sphere_on_the_oracle():
    sl = _slabs()
    b, eta = sphere_case()
    whole = OracleRows(nx=SNX, ny=SNY, bed=b, eta0=eta, sphere=SPHERE, manning=0.025)
    whole.sim.set_boundaries(**sphere_bounds())
    slabs = [sl.Slab(SNY, a, c) for a, c in sl.slab_rows(SNY, 3)]
    sims = []
    for s in slabs:
        o = OracleRows(nx=SNX, ny=s.rows, bed=s.take(b), eta0=s.take(eta), sphere=band(s), manning=0.025)
        o.sim.set_boundaries(**sphere_bounds())
        sl.copy_geometry(o.sim, s, whole.sim.geom)
        sims.append(o)
    run = sl.LocalSlabs(slabs, sims)
    for _ in range(STEPS):
        dt = run.step()
        assert whole.maxDt() == dt
        whole.step(dt)
    for f in ("h", "hu", "hv"):
        want = whole.get_rows(f, 2, SNY).reshape(SNY, -1)
        assert np.array_equal(run.gather(f).view(np.uint64), want.view(np.uint64)), f
    hv = want  # the last field gathered: hv
    assert np.all(hv[14:34, 2:-2] != 0)                     # motion across both cuts (rows 16 and 32)
    assert np.count_nonzero(whole.get_rows("h", 2, SNY) == 0) > 0      # the continent stays dry


@pytest.mark.gpu
def test_local_slabs_match_one_sphere_on_the_gpu():
    """Three slab handles of a spherical band, each given the band's own
    metric rows, against one handle of the whole band after every step."""
    sl = _slabs()
    import __graft_entry__
    swe = __graft_entry__.load_package()
    b, eta = sphere_case()

    def make(ny, bb, ee, sphere):
        sim = swe.ShallowWater(nx=SNX, ny=ny, bed=bb, eta0=ee, sphere=sphere, manning=0.025)
        sim.boundaries = {"west": swe.periodic, "east": swe.periodic, "south": swe.reflect, "north": swe.reflect}
        return sim

    whole = make(SNY, b, eta, SPHERE)
    slabs = [sl.Slab(SNY, a, c) for a, c in sl.slab_rows(SNY, 3)]
    sims = []
    for s in slabs:
        sim = make(s.rows, s.take(b), s.take(eta), band(s))
        sl.copy_geometry(sim, s, whole.geom)
        sims.append(sim)
    run = sl.LocalSlabs(slabs, sims)
    for step in range(STEPS):
        dt = run.step()
        assert whole.maxDt() == dt
        whole.step(dt)
        for f in ("h", "hu", "hv"):
            want = whole.get_rows(f, 2, SNY).reshape(SNY, -1)
            assert np.array_equal(run.gather(f).view(np.uint64), want.view(np.uint64)), (step, f)
    for sim in run.sims + [whole]:
        sim.close()


def test_periodic_south_north_is_refused():
    """A cut into row slabs cannot keep a periodic south / north boundary."""
    sl = _slabs()

    class Fake:
        class _P:
            name = "periodic"

        class _R:
            name = "reflect"
        boundaries = {"west": _P, "east": _P, "south": _R, "north": _P}
    slab = sl.Slab(NY, 0, 30)
    with pytest.raises(ValueError, match="north boundary is periodic"):
        sl.LocalSlabs([slab], [Fake()])
    with pytest.raises(ValueError, match="north boundary is periodic"):
        sl.check_cuttable(Fake())


@pytest.mark.gpu
def test_device_slabs_match_one_grid_on_the_gpu():
    """The device data plane: three slab handles on one GPU exchange their
    halos through device buffers on their own streams and step with the
    minimum of their maxDt() taken on the device (no host round trip), bit
    for bit like one handle of the whole grid.  The Flather side is a
    device tide so nothing needs the host per step."""
    sl = _slabs()
    import __graft_entry__
    swe = __graft_entry__.load_package()
    b, eta = case()
    tide = swe.Tide({"X": [0.1, 90.0]}, periods_hours={"X": 30.0 / 3600})

    def make(ny, bb, ee):
        sim = swe.ShallowWater(nx=NX, ny=ny, bed=bb, eta0=ee, **KW)
        sim.boundaries = {"west": swe.flather(tide.signal()), "east": swe.reflect,
                          "south": swe.reflect, "north": swe.reflect}
        sim._prepare_flather()
        return sim

    whole = make(NY, b, eta)
    slabs = [sl.Slab(NY, a, c) for a, c in sl.slab_rows(NY, 3)]
    run = sl.LocalSlabs(slabs, [make(s.rows, s.take(b), s.take(eta)) for s in slabs], device=True)
    for step in range(STEPS):
        dt = run.step()
        t0 = whole.t
        assert whole.run(1) == 1
        assert float(dt.item()) == whole.t - t0 or run.sims[0].t == whole.t
        assert all(s.t == whole.t for s in run.sims)
        for f in ("h", "hu", "hv"):
            got = run.gather(f)
            want = whole.get_rows(f, 2, NY).reshape(NY, -1)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (step, f)
    assert all(s.t == whole.t for s in run.sims)
    for sim in run.sims + [whole]:
        sim.close()
