import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine's kernels")
    config.addinivalue_line("markers", "slow: larger parity cases")


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def engine():
    import psiboil_b200 as pb
    pb.lib()
    if pb.device_count() < 1:
        pytest.fail("GPU test without a visible CUDA device")
    return pb
