"""C ABI checks that need no GPU: the library loads, exports every entry point declared in
include/uwshcu.h, validates its arguments and builds the same saturation table as the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import soundings

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(REPO, "include", "uwshcu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|char|void)\s*\*?\s*(\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_expected_entries():
    names = _declared()
    for n in ("compute_uwshcu_", "compute_uwshcu_inv_", "bxcompute_uwshcu_inv_", "uwshcu_init",
              "uwshcu_compute_device"):
        assert n in names


def test_library_exports_every_declared_symbol(uw):
    L = uw.lib()
    for name in _declared():
        assert hasattr(L, name), name


def test_table_matches_oracle_bit_for_bit(uw, oracle):
    assert np.array_equal(uw.estbl(), oracle.estbl())


def test_bad_arguments_are_rejected(uw):
    L = uw.lib()
    ci = lambda v: ctypes.byref(ctypes.c_int(v))
    cd = ctypes.byref(ctypes.c_double(1800.0))
    nulls = [None] * 47
    # null arrays
    rc = L.compute_uwshcu_(ci(8), ci(30), ci(8), ci(5), cd, *nulls[:42], None, ci(0), None, None)
    assert rc == uw.ERR_BAD_ARGS
    # iend > mix, mkx out of range, ncnst not the initialised count
    s = soundings.make_soundings(8, 30, seed=1)
    for kw in ({"iend": 9},):
        rc, _ = uw.compute_host(s, **kw)
        assert rc == uw.ERR_BAD_ARGS
    s6 = soundings.make_soundings(8, 30, seed=1, ncnst=6)
    rc, _ = uw.compute_host(s6)
    assert rc == uw.ERR_BAD_ARGS
    assert L.uwshcu_set_block(ctypes.c_int(48)) == uw.ERR_BAD_ARGS
    assert L.uwshcu_set_precision(ctypes.c_int(7)) == uw.ERR_BAD_ARGS
    assert uw.set_schedule(3) == uw.ERR_BAD_ARGS
    assert uw.set_schedule(uw.SCHED_TWO_PHASE) == 0 and uw.set_schedule(uw.SCHED_DEFAULT) == 0
    assert uw.set_hand_slots(-1) == uw.ERR_BAD_ARGS
    assert uw.set_hand_slots(100) == 0 and uw.set_hand_slots(0) == 0
    assert L.uwshcu_compute_member(None, None) == uw.ERR_BAD_ARGS
    assert L.uwshcu_tangent_device(None, None, None) == uw.ERR_BAD_ARGS
    assert L.uwshcu_adjoint_device(None, None, None) == uw.ERR_BAD_ARGS
    assert uw.set_adjoint_rows(-1) == uw.ERR_BAD_ARGS and uw.set_adjoint_rows((1 << 19) + 1) == uw.ERR_BAD_ARGS
    assert uw.set_adjoint_rows(0) == 0
    assert uw.adjoint_release() == 0
    assert L.uwshcu_adjoint_device_checked(None, None, None, None) == uw.ERR_BAD_ARGS
    assert L.uwshcu_set_depth_order(ctypes.c_int(2)) == uw.ERR_BAD_ARGS
    assert uw.set_depth_order(True) == 0 and uw.set_depth_order(False) == 0
    assert L.uwshcu_set_pipeline(ctypes.c_int(-2), ctypes.c_int(0)) == uw.ERR_BAD_ARGS   # streams 1..8
    assert uw.set_pipeline(-65536, 2) == 0 and uw.set_pipeline(-1, 0) == 0
    assert L.uwshcu_fp64_peak(None, None) == uw.ERR_BAD_ARGS


def test_init_rejects_bad_tracer_metadata(uw):
    qmin = np.zeros(5)
    wet = np.ones(5, dtype=np.int32)
    rc = uw.init(2.501e6, 1004.64, 3.337e5, 0.6, 287.0, 9.8, 0.622, 173.16, 375.16, 20.0, 1, 0.622,
                 461.5, 273.15, qmin, wet, 7, 5)
    assert rc == uw.ERR_BAD_ARGS
    assert uw.init_default() == 0


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) not in ("", None) or
                    __import__("torch").cuda.is_available(), reason="a CUDA device is visible")
def test_compute_without_device_reports_no_device(uw):
    s = soundings.make_soundings(4, 30, seed=2)
    rc, _ = uw.compute_host(s)
    assert rc == uw.ERR_NO_DEVICE


def test_tuning_parameters(uw, oracle):
    """set_params validation (C ABI and oracle), and the oracle's result depends on the values."""
    import soundings as snd
    assert uw.init_default() == 0
    assert uw.set_params(-1.0, 0.1, 14.0, 0.7e-3) == uw.ERR_BAD_ARGS
    assert uw.set_params(10.0, 0.0, 14.0, 0.7e-3) == uw.ERR_BAD_ARGS
    assert uw.set_params(10.0, 0.1, 14.0, -1e-3) == uw.ERR_BAD_ARGS
    assert uw.set_params(10.0, 0.1, 14.0, 0.7e-3) == 0
    s = snd.make_soundings(256, 30, seed=5)
    try:
        a = oracle.compute(s, diag=False)
        assert oracle.set_params(10.0, 0.1, 18.0, 0.7e-3) == 0
        b = oracle.compute(s, diag=False)
        assert not np.array_equal(a["sten"], b["sten"])
        assert oracle.set_params(-1.0, 0.1, 14.0, 0.7e-3) == -1
    finally:
        oracle.init_default()
