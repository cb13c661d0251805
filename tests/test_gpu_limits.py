"""The FP64 CUDA path at the edges of its compiled instantiations, bit for bit against the oracle
build with the kernel's math routines: the largest level count of the 32-level unit (31 layers) and
the smallest of the 64-level unit (32), the library's limit of 63 layers, 63 layers with the limit
of 32 tracers, a 6-tracer call (the first to take the 32-tracer unit) and a 12-layer column set;
both level orders at the limits, and both worklist schedules."""
import numpy as np
import pytest

import soundings
from test_gpu_parity import _check

pytestmark = pytest.mark.gpu


def _init(uw, oracle_pm, ncnst):
    qmin = np.zeros(ncnst)
    qmin[0] = 1e-12
    wet = np.array([1] * 5 + [0] * (ncnst - 5), dtype=np.int32)
    c = oracle_pm.consts()
    assert uw.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], 173.16, 375.16, 20.0, 1, c[14], c[15], c[16],
                   qmin, wet, 4, 5) == 0
    oracle_pm.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], c[10], 173.16, 375.16, 20.0, 1, c[14], c[15],
                   c[16], qmin, wet, 4, 5)


@pytest.fixture
def uwn(uw, oracle_pm):
    yield uw
    assert uw.init_default() == 0
    assert uw.set_schedule(uw.SCHED_DEFAULT) == 0
    oracle_pm.init_default()


@pytest.mark.parametrize("mkx,ncnst,ncol,inv,sched", [
    (12, 5, 3000, 0, "sorted"),
    (31, 5, 1500, 0, "sorted"),
    (32, 5, 1500, 0, "sorted"),
    (63, 5, 1500, 1, "sorted"),
    (63, 32, 1500, 0, "sorted"),
    (63, 32, 1500, 1, "two_phase"),
    (30, 6, 1500, 0, "two_phase"),
])
def test_instantiation_edges_match_oracle(uwn, oracle_pm, cuda, mkx, ncnst, ncol, inv, sched):
    uw = uwn
    _init(uw, oracle_pm, ncnst)
    assert uw.set_schedule(uw.SCHED_SORTED if sched == "sorted" else uw.SCHED_TWO_PHASE) == 0
    s = soundings.make_soundings(ncol, mkx, seed=500 + mkx + ncnst, ncnst=ncnst, rh_pbl=(0.6, 0.95))
    ref = oracle_pm.compute(s, diag=False)
    assert np.sum(ref["cush"] != -1.0) >= 100
    if inv:
        rc, out = uw.compute_host(soundings.to_inv(s), entry="compute_uwshcu_inv_")
        ref = oracle_pm.compute(soundings.to_inv(s), inv=True, diag=False)
    else:
        rc, out = uw.compute_host(s)
    assert rc == ref["status"], uw.last_cuda_error()
    _check(out, ref, ncol, frac=1.0)
