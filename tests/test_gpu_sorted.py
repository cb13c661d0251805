"""The sorted schedule (UWSHCU_SCHED_SORTED).

Its worklist pass runs in two launches: the first computes iteration 1 of the implicit-CIN loop and
iteration 2 up to the CIN decision (uwshcu.F90:1759-1889); a column taking the implicit branch stores
its whole state and a second launch continues it, in warps sorted by iteration-1 updraft depth.
Each column computes the same operations in the same order whichever launch finishes it, so every
output and diagnostic must be the bits of the two-phase schedule: in the FP64, FAST and MIXED modes,
through the device entry with all diagnostics, through the host entries chunked over streams, for
30 and 51 levels, and with a slot cap small enough that most columns finish in the first launch.
"""
import numpy as np
import pytest

import soundings

pytestmark = pytest.mark.gpu

UW_L_DELCIN = 1 << 9


def _diff(a, b):
    return [k for k in a if not np.array_equal(a[k], b[k])]


def _settings(uw, sched, slots):
    assert uw.set_schedule(sched) == 0
    assert uw.set_hand_slots(slots) == 0


@pytest.mark.parametrize("prec", ["fp64", "fast", "mixed"])
@pytest.mark.parametrize("pver", [30, 51])
def test_device_entry_sorted_matches_two_phase(uw, cuda, prec, pver):
    assert uw.init_default() == 0
    mode = {"fp64": uw.PREC_FP64, "fast": uw.PREC_FAST, "mixed": uw.PREC_MIXED}[prec]
    s = soundings.make_soundings(12000, pver, seed=111 + pver, rh_pbl=(0.6, 0.95))
    out = {}
    try:
        assert uw.set_precision(mode) == 0
        first = None
        for name, sched, slots in (("two_phase", uw.SCHED_TWO_PHASE, 0), ("sorted", uw.SCHED_SORTED, 0),
                                   ("capped", uw.SCHED_SORTED, 64)):
            _settings(uw, sched, slots)
            case = uw.DeviceCase(s, diag=True, inputs=None if first is None else first.inp)
            first = first or case
            case.diag_level.fill_(-777.0)
            for _ in range(2):   # twice: the regions are reused, and their counters restart
                case.reset_cush()
                assert case.launch_member() == 0, uw.last_cuda_error()
                assert case.status() == 0
            out[name] = case.outputs_numpy()
    finally:
        _settings(uw, uw.SCHED_DEFAULT, 0)
        uw.set_precision(uw.PREC_FP64)
    ref = out["two_phase"]
    # the workload reaches the hand-off: convecting columns that took the implicit branch
    conv = ref["cush"] != -1.0
    implicit = conv & ((ref["diag_int"][1] & UW_L_DELCIN) == 0)
    assert implicit.sum() > 200, implicit.sum()
    assert not _diff(ref, out["sorted"]), _diff(ref, out["sorted"])
    assert not _diff(ref, out["capped"]), _diff(ref, out["capped"])


def test_host_entries_sorted_match_two_phase(uw, cuda):
    """Chunked host-array calls over several streams, each stream with its own hand-off region."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(9000, 30, seed=113, rh_pbl=(0.6, 0.95))
    try:
        for entry in ("compute_uwshcu_", "compute_uwshcu_inv_"):
            si = s if entry == "compute_uwshcu_" else soundings.to_inv(s)
            _settings(uw, uw.SCHED_TWO_PHASE, 0)
            rc0, o0 = uw.compute_host(si, entry=entry, iend=8800)
            for chunk, streams, slots in ((0, 1, 0), (2048, 3, 0), (1500, 2, 100)):
                assert uw.set_pipeline(chunk, streams) == 0
                _settings(uw, uw.SCHED_SORTED, slots)
                rc, o = uw.compute_host(si, entry=entry, iend=8800)
                assert rc == rc0
                assert not _diff(o0, o), (entry, chunk, streams, slots, _diff(o0, o))
    finally:
        _settings(uw, uw.SCHED_DEFAULT, 0)
        assert uw.set_pipeline(-1, 0) == 0


def test_sorted_schedule_matches_oracle(uw, oracle_pm, cuda):
    """Against the oracle build with the kernel's exp/log/pow/erfc: bit for bit."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(4096, 30, seed=117, rh_pbl=(0.6, 0.95))
    ref = oracle_pm.compute(s, diag=True)
    try:
        _settings(uw, uw.SCHED_SORTED, 0)
        case = uw.DeviceCase(s, diag=True)
        assert case.launch_member() == 0, uw.last_cuda_error()
        assert case.status() == ref["status"]
        out = case.outputs_numpy()
    finally:
        _settings(uw, uw.SCHED_DEFAULT, 0)
    same = [k for k in ("umf", "qvten", "sten", "precip", "cush", "cnt", "cnb", "diag_int", "diag_real",
                        "diag_level") if np.mean(np.all((out[k] == ref[k]).reshape(-1, s["ncol"]), axis=0)) < 0.9999]
    assert not same, same

