import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and the built engine library")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="session")
def engine():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from astro_transit_gpu_b200.engine import BLSEngine
    return BLSEngine.get(0)
