"""The FP64 CUDA path at the edges of its compiled instantiations, bit for bit against the oracle
build with the kernel's math routines: the largest level count of the 32-level unit (31 layers) and
the smallest of the 64-level unit (32), the library's limit of 63 layers, 63 layers with the limit
of 32 tracers, a 6-tracer call (the first to take the 32-tracer unit) and a 12-layer column set;
both level orders at the limits, and both worklist schedules.  Also the calls at the edges of the
column count: none (iend = 0), one, none convecting and nearly all convecting."""
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


def test_empty_and_single_column_calls(uw, oracle_pm, cuda):
    """iend = 0 computes nothing and leaves the outputs as they were; iend = 1 (one column of a
    mix = 64 call) is the oracle's column, in both level orders."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(64, 30, seed=541, rh_pbl=(0.85, 0.95))
    ref = oracle_pm.compute(s, diag=False)
    i = int(np.flatnonzero(ref["cush"] != -1.0)[0])
    poison = uw.alloc_outputs(30, 5, 64, s["cush"])
    for v in poison.values():
        if v.dtype == np.float64:
            v.fill(7.0)
    before = {k: v.copy() for k, v in poison.items()}
    rc, out = uw.compute_host(s, iend=0, out=poison)
    assert rc == 0
    assert all(np.array_equal(out[k], before[k]) for k in out)
    # the convecting column moved to index 0, so that iend = 1 computes it
    s1 = {k: (np.ascontiguousarray(np.roll(v, -i, axis=-1)) if isinstance(v, np.ndarray) and v.shape[-1] == 64 else v)
          for k, v in s.items()}
    ref1 = oracle_pm.compute(s1, diag=False)
    assert ref1["cush"][0] != -1.0
    for inv in (0, 1):
        si = soundings.to_inv(s1) if inv else s1
        rc, out = uw.compute_host(si, iend=1, entry="compute_uwshcu_inv_" if inv else "compute_uwshcu_")
        assert rc == 0, uw.last_cuda_error()
        r = oracle_pm.compute(si, inv=bool(inv), diag=False)
        for k in out:
            if isinstance(out[k], np.ndarray) and out[k].ndim >= 1:
                assert np.array_equal(out[k][..., 0], r[k][..., 0]), (inv, k)


@pytest.mark.parametrize("rh,which", [((0.05, 0.10), "none"), ((0.97, 0.99), "most")])
def test_calls_with_no_or_mostly_convecting_columns(uw, oracle_pm, cuda, rh, which):
    """A call whose worklist is empty (dry boundary layers: no column passes the trigger) and one in
    which most columns convect, against the oracle, in both worklist schedules."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(4000, 30, seed=542, rh_pbl=rh)
    ref = oracle_pm.compute(s, diag=False)
    frac = float(np.mean(ref["cush"] != -1.0))
    assert (frac == 0.0) if which == "none" else (frac > 0.5), frac
    try:
        for sched in (uw.SCHED_SORTED, uw.SCHED_TWO_PHASE):
            assert uw.set_schedule(sched) == 0
            rc, out = uw.compute_host(s)
            assert rc == ref["status"], uw.last_cuda_error()
            _check(out, ref, 4000, frac=1.0)
    finally:
        assert uw.set_schedule(uw.SCHED_DEFAULT) == 0
