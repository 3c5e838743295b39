import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and libmemphys_cuda.so")
    config.addinivalue_line("markers", "slow: larger sizes")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def mp_lib():
    """The CUDA library; GPU tests fail (not skip) when it is missing."""
    from memphys_b200 import build, capi
    if not os.path.exists(capi.LIB_PATH):
        build.build()
    L = capi.lib()
    capi.device_info()  # raises NO_DEVICE without a B200
    return L
