"""CUDA path against the fixtures produced by the reference's own drop-in (25 tracers)."""
import numpy as np
import pytest

from test_gpu_parity import _check
from test_oracle_pin import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture
def uw25(uw):
    yield uw
    assert uw.init_default() == 0


@pytest.mark.parametrize("path", GOLDEN, ids=[p.rsplit("/", 1)[-1] for p in GOLDEN])
def test_gpu_matches_reference_fixture(uw25, cuda, path):
    si, ref, qmin, wet, consts, estbl = load_golden(path)
    c = consts
    rc = uw25.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], 173.16, 375.16, 20.0, 1, c[14], c[15],
                   c[16], qmin, wet, 4, 5)
    assert rc == 0
    assert np.array_equal(uw25.estbl(), estbl)
    rc, out = uw25.compute_host(si, entry="bxcompute_uwshcu_inv_")
    assert rc == 0, uw25.last_cuda_error()
    _check(out, ref, si["ncol"], frac=1.0 - 1.0 / si["ncol"])
