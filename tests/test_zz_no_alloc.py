"""swe_max_dt_noalloc: maxDt() for callers that cannot allocate device memory.

Some callers own every byte of device memory themselves (a fixed arena, a
hard memory cap, a region where allocation is forbidden), so they cannot
create a handle, whose constructor allocates.  They pass their own device
arrays; the library keeps the reduction scratch in a fixed array compiled
into it.  This checks, through the C ABI, that the result equals the handle
path's maxDt() exactly (the reduction is a max, so the tolerance is zero),
on two calls in a row and again after the state has moved, and that grids
taller than the fixed scratch are refused with a clear error.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_copies(torch, sim):
    dev = torch.device("cuda")
    f = {n: torch.from_numpy(np.array(sim.field(n))).to(dev) for n in ("h", "hu", "hv")}
    g = sim.geom._rows
    f["dxRow"] = torch.from_numpy(np.array(g["dxRow"])).to(dev)
    f["dyCFL"] = torch.from_numpy(np.array(g["dyCFL"])).to(dev)
    return f


def _call(lib, torch, sim, f, out, ny=None):
    stream = torch.cuda.current_stream().cuda_stream
    return lib.swe_max_dt_noalloc(sim.nx, sim.ny if ny is None else ny, f["h"].data_ptr(), f["hu"].data_ptr(),
                                  f["hv"].data_ptr(), f["dxRow"].data_ptr(), f["dyCFL"].data_ptr(),
                                  sim.minDepth, sim.cfl, out.data_ptr(), stream)


def test_noalloc_max_dt_matches_handle_path(swe):
    torch = pytest.importorskip("torch")
    from water_simulator_b200 import workloads
    lib = swe.load_library()
    nx, ny = 300, 180
    b, eta = workloads.bump_dam_break(nx, ny, 5.0)
    sim = swe.ShallowWater(nx=nx, ny=ny, dx=5.0, bed=b, eta0=eta, manning=0.025)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(2):                       # the state at t = 0, then after 7 steps
        want = sim.maxDt()
        f = _device_copies(torch, sim)
        for call in range(2):                # two calls in a row share the scratch
            out.fill_(-1.0)
            assert _call(lib, torch, sim, f, out) == 0, lib.swe_last_error()
            torch.cuda.synchronize()
            assert out.item() == want, (call, out.item(), want)
        for _ in range(7):
            sim.step()
    sim.close()


def test_noalloc_max_dt_all_dry_is_infinity(swe):
    """No wet cell: maxDt() is Infinity (src/swe.mjs:646), on both paths."""
    torch = pytest.importorskip("torch")
    lib = swe.load_library()
    sim = swe.ShallowWater(nx=40, ny=30, dx=2.0, bed=lambda x, y: 1.0, eta0=0.0)
    assert sim.maxDt() == float("inf")
    f = _device_copies(torch, sim)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(-1.0)
        assert _call(lib, torch, sim, f, out) == 0, lib.swe_last_error()
        torch.cuda.synchronize()
        assert out.item() == float("inf")
    sim.close()


def test_noalloc_max_dt_at_the_row_limit(swe):
    """ny = SWE_NOALLOC_MAX_ROWS: every scratch slot is used, and the result
    still equals the handle path's."""
    torch = pytest.importorskip("torch")
    lib = swe.load_library()
    nx, ny = 8, 16384
    rng = np.random.default_rng(3)
    eta = 1.0 + 0.5 * rng.uniform(0, 1, (ny + 4, nx + 4))
    sim = swe.ShallowWater(nx=nx, ny=ny, dx=1.5, bed=np.zeros((ny + 4, nx + 4)), eta0=eta)
    sim.step()
    want = sim.maxDt()
    f = _device_copies(torch, sim)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(-1.0)
        assert _call(lib, torch, sim, f, out) == 0, lib.swe_last_error()
        torch.cuda.synchronize()
        assert out.item() == want
    sim.close()


def test_noalloc_max_dt_rejects_oversized_grid(swe):
    torch = pytest.importorskip("torch")
    lib = swe.load_library()
    sim = swe.ShallowWater(nx=8, ny=6, dx=1.0, bed=lambda x, y: 0, eta0=1.0)
    f = _device_copies(torch, sim)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    assert _call(lib, torch, sim, f, out, ny=16385) == -1
    assert b"exceeds the fixed scratch" in lib.swe_last_error()
    sim.close()
