"""Every GPU parity case of test_parity_gpu.py again, with the stage run by
the two tiled kernels (k_split_faces, k_split_cells) instead of the fused
row-marching kernel: the same bit-for-bit comparison against the oracle."""
import pytest

from test_parity_gpu import *  # noqa: F401,F403  (the cases themselves)


@pytest.fixture(autouse=True)
def _stage_kernels(monkeypatch):
    monkeypatch.setenv("SWE_B200_STAGE", "split")


def test_the_handles_run_the_tiled_kernels(swe):
    import ctypes
    sim = swe.ShallowWater(nx=40, ny=30, dx=1.0, bed=-1.0, eta0=0.0)
    impl = ctypes.c_int(-1)
    swe._lib.check(swe.load_library().swe_get_stage_kernels(sim._h, ctypes.byref(impl)))
    assert impl.value == 1
    sim.close()


@pytest.mark.parametrize("case", ["beach", "sphere", "beach_sponge"])
def test_tiled_and_fused_give_the_same_bits(swe, case, monkeypatch):
    """Down to the sign of zero: the tiled pair (with its dry-tile skip and
    the tiles it settles to +0 without computing them) against the fused
    kernel, after many steps of a flooding beach, of a sphere with land, and
    of the beach with a sponge over its dry east end (the sponge pours water
    onto dry tiles, so no tile may settle under it)."""
    import numpy as np
    from water_simulator_b200 import workloads

    def make():
        if case in ("beach", "beach_sponge"):
            b, h = workloads.beach_dam_break(nx=256, ny=96, dx=8.0)
            sim = swe.ShallowWater(nx=256, ny=96, dx=8.0, bed=b, eta0=b + h, manning=0.03)
            sim.boundaries = {"west": swe.flather(lambda t: 0.0, lambda t: 0.0)}
            if case == "beach_sponge":
                eta_ref = float(np.max(b)) + 0.5
                sim.forcing = swe.makeSponge(sim, side="east", width=40, strength=0.05, etaRef=eta_ref)
            return sim
        c = workloads.globe_tide(nx=180, ny=90, lat0=-80.0, lat1=80.0, modes=12)
        return swe.ShallowWater(nx=180, ny=90, bed=c["b"], eta0=c["eta0"] + (c["b"] < 0) * 0.5,
                                sphere={"R": 6371e3, "lat0": -80.0, "lat1": 80.0, "omega": 7.2921e-5})

    out = {}
    for impl in ("fused", "split"):
        monkeypatch.setenv("SWE_B200_STAGE", impl)
        sim = make()
        assert sim.run(200) == 200
        out[impl] = [sim.field(f).view(np.uint64).copy() for f in ("h", "hu", "hv")] + [sim.t]
        sim.close()
    for a, b in zip(out["fused"][:3], out["split"][:3]):
        assert np.array_equal(a, b)
    assert out["fused"][3] == out["split"][3]


def test_dry_tile_flags_follow_host_writes(swe, monkeypatch):
    """The cell kernel records which tiles it left with h == 0 everywhere,
    and the next face kernel skips tiles whose 3 x 3 neighbourhood is so
    recorded.  Every other writer of the state clears those records: water
    poured onto dry land by the host, dryClean, friction, and a switch to
    the fused kernels and back.  Through all of them the tiled pair stays
    bit-identical (uint64 patterns) to the fused kernel."""
    import ctypes
    import numpy as np
    from water_simulator_b200 import workloads
    lib = swe.load_library()

    def scenario(impl):
        monkeypatch.setenv("SWE_B200_STAGE", impl)
        b, h = workloads.beach_dam_break(nx=256, ny=96, dx=8.0)
        sim = swe.ShallowWater(nx=256, ny=96, dx=8.0, bed=b, eta0=b + h, manning=0.03)
        sim.boundaries = {"west": swe.flather(lambda t: 0.0, lambda t: 0.0)}
        assert sim.run(40) == 40
        hh = np.array(sim.field("h")).reshape(sim.H, sim.W)
        assert (hh[30:70, 160:240] == 0).all()            # dry land, tiles deep inside it
        hh[40:60, 170:230] += 0.7                         # a pond poured onto it
        sim.h = hh.reshape(-1)
        assert sim.run(30) == 30
        sim.dryClean()
        assert sim.run(10) == 10
        sim.applyFriction(sim.maxDt())
        assert sim.run(10) == 10
        other = 0 if impl == "split" else 1               # there and back
        mine = 1 - other
        swe._lib.check(lib.swe_set_stage_kernels(sim._h, other))
        assert sim.run(5) == 5
        swe._lib.check(lib.swe_set_stage_kernels(sim._h, mine))
        assert sim.run(25) == 25
        out = [sim.field(f).view(np.uint64).copy() for f in ("h", "hu", "hv")] + [sim.t]
        sim.close()
        return out

    fused, split = scenario("fused"), scenario("split")
    for a, b in zip(fused[:3], split[:3]):
        assert np.array_equal(a, b)
    assert fused[3] == split[3]


@pytest.mark.parametrize("nx,ny", [(256, 96), (255, 97), (30, 9)])
def test_tensor_map_tile_copies_give_the_same_bits(swe, monkeypatch, nx, ny):
    """The face kernel's state tile and the cell kernel's face and depth
    tiles fetched by tensor-map copies (even padded width) against the
    per-element loads (SWE_B200_TMA=0): the same bits after 150 steps of a
    flooding beach with friction, tiles at every edge of the grid and tiles
    beside dry ones included (the copies fill outside the grid with zeros,
    and faces of dry tiles are read as +0 either way).  An odd padded width
    always takes the per-element loads."""
    import numpy as np
    from water_simulator_b200 import workloads

    def run(tma):
        monkeypatch.setenv("SWE_B200_TMA", "1" if tma else "0")
        b, h = workloads.beach_dam_break(nx=nx, ny=ny, dx=8.0 * 256 / nx)
        sim = swe.ShallowWater(nx=nx, ny=ny, dx=8.0 * 256 / nx, bed=b, eta0=b + h, manning=0.03)
        sim.boundaries = {"west": swe.flather(swe.Tide({}, msl=0.0).signal()), "north": swe.outflow}
        assert sim.run(150) == 150
        out = [sim.field(f).view(np.uint64).copy() for f in ("h", "hu", "hv")] + [sim.t]
        sim.close()
        return out

    a, b = run(True), run(False)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]


@pytest.mark.parametrize("nx,ny", [(256, 96), (512, 384)])
def test_face_tile_list_gives_the_same_bits(swe, monkeypatch, nx, ny):
    """The face kernel over the list of tiles that do not settle, on a grid
    of resident CTAs, against one CTA per tile (SWE_B200_FACE_LIST=0): the
    same bits after 150 steps of a flooding beach, where most tiles settle
    and the list changes as the water moves."""
    import numpy as np
    from water_simulator_b200 import workloads

    def run(on):
        monkeypatch.setenv("SWE_B200_FACE_LIST", "1" if on else "0")
        b, h = workloads.beach_dam_break(nx=nx, ny=ny, dx=8.0 * 256 / nx)
        sim = swe.ShallowWater(nx=nx, ny=ny, dx=8.0 * 256 / nx, bed=b, eta0=b + h, manning=0.03)
        sim.boundaries = {"west": swe.flather(swe.Tide({}, msl=0.0).signal())}
        assert sim.run(150) == 150
        out = [sim.field(f).view(np.uint64).copy() for f in ("h", "hu", "hv")] + [sim.t, sim.massFloored]
        sim.close()
        return out

    a, b = run(True), run(False)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3:] == b[3:]
