"""Non-finite inputs are flagged per column (no counterpart in the reference, where a NaN or Inf
propagates into the column's outputs or stops the model in findsp).

A column with a NaN or Inf in any input the scheme reads takes the exit path: the label-333 outputs
of uwshcu.F90:4448-4549 (zero tendencies and fluxes, cush = -1, cnt = 1, cnb = mkx), exit flag
UWSHCU_EXIT_NONFINITE in diag_int row 0, status UWSHCU_WARN_NONFINITE_INPUT.  Every other column is
bit for bit what the call gives without the bad columns."""
import numpy as np
import pytest

import soundings
from util import FIELDS

pytestmark = pytest.mark.gpu

EXIT_NONFINITE = 1 << 11
WARN_NONFINITE = 4

# (field, level or None, value): one bad value per poisoned column
POISON = [("t0", 3, np.nan), ("qv0", 0, np.inf), ("tke", 5, -np.inf), ("pblh", None, np.nan),
          ("u0", 29, np.nan), ("tr0", (3, 10), np.nan), ("ps0", 0, np.inf), ("cush", None, np.nan),
          ("z0", 12, np.nan), ("dp0", 7, np.inf)]


def _poison(s, cols):
    p = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in s.items()}
    for (field, lev, val), c in zip(POISON, cols):
        if lev is None:
            p[field][c] = val
        elif isinstance(lev, tuple):
            p[field][lev[0], lev[1], c] = val
        else:
            p[field][lev, c] = val
    return p


@pytest.mark.parametrize("entry", ["device", "host"])
def test_nonfinite_columns_take_the_exit_path(uw, oracle_pm, cuda, entry):
    s = soundings.make_soundings(4096, 30, seed=81)
    ref = oracle_pm.compute(s, diag=True)
    conv = np.flatnonzero(ref["cush"] != -1.0)
    cols = conv[:len(POISON)]                 # poison convecting columns: their outputs change most
    p = _poison(s, cols)
    if entry == "device":
        case = uw.DeviceCase(p, diag=True)
        assert case.launch() == 0
        assert case.status() == WARN_NONFINITE
        out = case.outputs_numpy()
        assert np.all(out["diag_int"][0, cols] & EXIT_NONFINITE)
        others = np.setdiff1d(np.arange(s["ncol"]), cols)
        assert not np.any(out["diag_int"][0, others] & EXIT_NONFINITE)
    else:
        rc, out = uw.compute_host(p)
        assert rc == WARN_NONFINITE
    mkx = s["mkx"]
    for f in FIELDS:
        a = out[f][..., cols]
        if f == "cush":
            assert np.all(a == -1.0)
        elif f == "cnt":
            assert np.all(a == 1.0)
        elif f == "cnb":
            assert np.all(a == float(mkx))
        else:
            assert np.all(a == 0.0), f
    keep = np.ones(s["ncol"], bool)
    keep[cols] = False
    for f in FIELDS:
        assert np.array_equal(out[f][..., keep], ref[f][..., keep]), f


def test_finite_inputs_report_no_flag(uw, cuda):
    s = soundings.make_soundings(1024, 30, seed=82)
    case = uw.DeviceCase(s, diag=True)
    assert case.launch() == 0 and case.status() == 0
    assert not np.any(case.outputs_numpy()["diag_int"][0] & EXIT_NONFINITE)
