import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hpc-and-climate-model_b200")
for p in (os.path.join(REPO, "oracle"), PKG, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.init_default()
    return o


@pytest.fixture(scope="session")
def uw():
    import uwshcu_b200 as u
    assert u.init_default() == 0
    return u


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return torch
