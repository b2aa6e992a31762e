import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import __graft_entry__  # noqa: E402

__graft_entry__.load_package()   # registers water_simulator_b200 for module-level imports


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running oracle pin")


@pytest.fixture(scope="session")
def swe():
    """The product package (water-simulator_b200/)."""
    return __graft_entry__.load_package()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
