import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def controls():
    import clbool_b200 as cb
    if cb.device_count() == 0:
        pytest.fail("GPU test selected but no CUDA device is visible")
    return cb.create_controls(0, 0)
