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
    """The oracle build pinned to the reference (glibc transcendentals)."""
    import oracle as o
    o.set_variant("glibc")
    o.init_default()
    return o


class _Variant:
    """Another build of the oracle (oracle.set_variant): every call selects that build and switches
    back to the glibc build afterwards."""

    def __init__(self, mod, variant):
        self.m = mod
        self.variant = variant

    def __getattr__(self, name):
        f = getattr(self.m, name)
        if not callable(f):
            return f

        def call(*a, **k):
            self.m.set_variant(self.variant)
            try:
                return f(*a, **k)
            finally:
                self.m.set_variant("glibc")
        return call


@pytest.fixture(scope="session")
def oracle_pm(oracle):
    """The oracle build with the host/device-identical math routines the CUDA path uses."""
    p = _Variant(oracle, "portable")
    p.init_default()
    return p


@pytest.fixture(scope="session")
def oracle_ftn(oracle):
    """The oracle build with the Fortran's own math: glibc exp/log/pow and CAM's CALERF erfc."""
    p = _Variant(oracle, "fortran")
    p.init_default()
    return p


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
