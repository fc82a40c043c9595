import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def lib():
    from gpsm_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def gpu(lib):
    if not HAS_GPU:
        pytest.skip("no GPU")
    import gpsm_b200 as G
    G.init(0)
    return G


@pytest.fixture(scope="session")
def small_er():
    from gpsm_b200 import workloads as W
    return W.workload("small_er")
