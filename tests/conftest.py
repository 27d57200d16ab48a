import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: long-running CPU check")


@pytest.fixture(scope="session")
def wtlib():
    """libwt.so, built in-tree if missing (nvcc cross-compiles without a GPU)."""
    from windtunnel_vis_b200 import abi, build

    if not os.path.exists(abi.LIB_PATH):
        build.build()
    return abi.load()


@pytest.fixture(scope="session")
def gpu(wtlib):
    """Skips when no CUDA device is visible; GPU tests run through libwt.so only."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device visible")
    return wtlib


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    return O
