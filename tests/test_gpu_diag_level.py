"""Per-level diagnostics of uwshcu_compute_member (uwshcu_member.diag_level) against the oracle.

These are the history fields compute_uwshcu writes for every column: updraft fraction, total water,
liquid-water and virtual potential temperature, winds, net updraft mass flux, rain and snow fluxes on
interfaces; entrainment, detrainment and detrained condensate tendencies on layers
(uwshcu.F90:1945-1990 after the explicit-CIN fallback, :4383-4433 otherwise, zeros at :4484-4529).
The oracle build that shares the kernel's exp/log/pow/erfc gives the expected values; the bar is the
FP64 parity bar of the output fields (the expected result is bit for bit).
"""
import numpy as np
import pytest

import soundings
from util import compare

pytestmark = pytest.mark.gpu

TOL = 1e-11
FRAC = 0.9999
UW_L_DELCIN = 1 << 9


def _rows(dl, names):
    return {n: dl[j] for j, n in enumerate(names)}


def test_diag_level_matches_oracle(uw, oracle_pm, cuda):
    assert uw.init_default() == 0
    s = soundings.make_soundings(4096, 30, seed=91, rh_pbl=(0.6, 0.95))
    n = s["ncol"]
    ref = oracle_pm.compute(s, diag=True)
    # the workload reaches every writer: full runs, exits and the explicit-CIN fallback
    assert np.any(ref["cush"] != -1.0) and np.any(ref["diag_int"][0] != 0)
    assert np.any(ref["diag_int"][1] & UW_L_DELCIN)
    case = uw.DeviceCase(s, diag=True)
    case.diag_level.fill_(-777.0)
    assert case.launch_member() == 0, uw.last_cuda_error()
    assert case.status() == ref["status"]
    out = case.outputs_numpy()
    names = uw.DL_NAMES
    res, _ = compare(_rows(out["diag_level"], names), _rows(ref["diag_level"], names), tol=TOL,
                     fields=names, ncol=n)
    bad = {f: v for f, v in res.items() if v[0] < FRAC}
    assert not bad, bad
    same = np.mean(np.all(out["diag_level"] == ref["diag_level"], axis=(0, 1)))
    assert same >= FRAC, same
    # layer rows hold zero at the surface interface
    assert np.all(out["diag_level"][names.index("fer"):, 0, :] == 0.0)


def test_member_entry_matches_device_entry_in_both_level_orders(uw, cuda):
    """uwshcu_compute_member gives the bits of uwshcu_compute_device; with diag_level NULL it writes
    nothing there, and the top-down level order gives the same (bottom-up) per-level diagnostics."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(3000, 30, seed=92, rh_pbl=(0.6, 0.95))
    a = uw.DeviceCase(s, diag=True)
    assert a.launch() == 0 and a.status() == 0
    want = a.outputs_numpy()
    assert not np.any(want["diag_level"])
    b = uw.DeviceCase(s, diag=True, inputs=a.inp)
    assert b.launch_member() == 0 and b.status() == 0
    got = b.outputs_numpy()
    diff = [k for k in want if k != "diag_level" and not np.array_equal(want[k], got[k])]
    assert not diff, diff
    assert np.any(got["diag_level"])
    # without the optional arrays
    c = uw.DeviceCase(s, diag=False, inputs=a.inp)
    assert c.launch_member() == 0 and c.status() == 0
    oc = c.outputs_numpy()
    assert all(np.array_equal(oc[k], want[k]) for k in oc)
    # top-down inputs: outputs in that order, per-level diagnostics still bottom-up
    si = soundings.to_inv(s)
    d = uw.DeviceCase(si, diag=True)
    assert d.launch_member(inv=1) == 0 and d.status() == 0
    od = d.outputs_numpy()
    assert np.array_equal(od["diag_level"], got["diag_level"])
    assert np.array_equal(od["umf"][::-1], got["umf"])
