import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU; run with -m gpu")


@pytest.fixture(scope="session")
def built_libs():
    """Build (or confirm up to date) the engine libraries and the oracle."""
    from gpu_cross_b200 import build

    import oracle

    build.build()
    oracle.build()
    return True


@pytest.fixture(scope="session")
def cuda(built_libs):
    import torch

    from gpu_cross_b200 import capi

    if not torch.cuda.is_available() or not capi.device_available():
        pytest.fail("GPU test collected on a machine without a usable sm_100 device")
    torch.cuda.init()
    return torch.device("cuda:0")
