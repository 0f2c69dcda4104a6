import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running full-size case")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O  # noqa: E402  (the CPU checker)
    O.lib()
    return O


@pytest.fixture(scope="session")
def gpu_lib():
    from salsaa_b200 import build
    build.build()
    import salsaa_b200
    return salsaa_b200.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but no CUDA device is visible")
    return torch
