"""CUDA path on the fixtures produced by the reference's own drop-in (25 tracers, CAM level order,
bxcompute_uwshcu_inv_ entry): bit for bit against the portable-math oracle on the same inputs, and
within the conditioning bound of two libms against the fixture outputs themselves."""
import numpy as np
import pytest

from test_gpu_parity import _check
from test_oracle_pin import GOLDEN, init_oracle, load_golden
from util import conditioned_compare

pytestmark = pytest.mark.gpu


@pytest.fixture
def uw25(uw, oracle_pm):
    yield uw
    assert uw.init_default() == 0
    oracle_pm.init_default()


@pytest.mark.parametrize("path", GOLDEN, ids=[p.rsplit("/", 1)[-1] for p in GOLDEN])
def test_gpu_matches_reference_fixture(uw25, oracle_pm, cuda, path):
    si, ref, qmin, wet, consts, estbl = load_golden(path)
    c = consts
    rc = uw25.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], 173.16, 375.16, 20.0, 1, c[14], c[15],
                   c[16], qmin, wet, 4, 5)
    assert rc == 0
    assert np.array_equal(uw25.estbl(), estbl)
    rc, out = uw25.compute_host(si, entry="bxcompute_uwshcu_inv_")
    assert rc == 0, uw25.last_cuda_error()
    # against the reference's outputs: same decisions; values differ only by the amplified
    # last-bit differences of the two libms (bounded in test_oracle_variants on 12,000 columns)
    for f in ("cnt", "cnb"):
        assert np.array_equal(out[f], ref[f]), f
    w = conditioned_compare(out, ref)
    assert np.mean(w <= 1e-6) >= 0.95 and np.max(w) < 1e-2, (np.mean(w <= 1e-6), np.max(w))
    # against the portable-math oracle on the same inputs: bit for bit
    init_oracle(oracle_pm, qmin, wet)
    pm = oracle_pm.compute(si, inv=True)
    _check(out, pm, si["ncol"], frac=1.0)


@pytest.mark.parametrize("sched", ["sorted", "two_phase"])
def test_64_levels_25_tracers_match_oracle(uw25, oracle_pm, cuda, sched):
    """The (64-level, 32-tracer) instantiation: 51 levels and 25 tracers with the fixtures' tracer
    metadata, bit for bit against the portable-math oracle, in both worklist schedules."""
    import os
    import sys

    import soundings
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden

    qmin, wet = make_golden.config()
    c = oracle_pm.consts()
    assert uw25.init(c[0], c[3], c[1], c[4], c[5], c[6], c[7], 173.16, 375.16, 20.0, 1, c[14], c[15],
                     c[16], qmin, wet, 4, 5) == 0
    init_oracle(oracle_pm, qmin, wet)
    s = soundings.make_soundings(3000, 51, seed=131, ncnst=25, rh_pbl=(0.6, 0.95))
    ref = oracle_pm.compute(s, diag=False)
    assert np.mean(ref["cush"] != -1.0) > 0.2
    try:
        assert uw25.set_schedule(uw25.SCHED_SORTED if sched == "sorted" else uw25.SCHED_TWO_PHASE) == 0
        rc, out = uw25.compute_host(s)
    finally:
        uw25.set_schedule(uw25.SCHED_DEFAULT)
    assert rc == ref["status"], uw25.last_cuda_error()
    _check(out, ref, s["ncol"], frac=1.0)
