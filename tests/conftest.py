import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def device_lib():
    """The in-tree sm_100a library, built if missing; never a fallback."""
    from hpg_b200 import build as b
    b.build_device()
    import hpg_b200
    return hpg_b200.load()


@pytest.fixture(scope="session")
def gpu(device_lib):
    import hpg_b200
    if hpg_b200.device_count() < 1:
        pytest.fail("no CUDA device visible to libhpgb.so")
    return device_lib
