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
