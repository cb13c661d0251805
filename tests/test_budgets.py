"""Column energy and water budgets (check_energy_chng, check_energy.F90:321-395, as tphysbc.F90:446-447
applies it after the shallow scheme).  The scheme closes both to roundoff, so the budgets are a
size-independent property of every output: at the full benchmark size no column may exceed CAM's
flag thresholds (|te_rer| > 1e-14, |tw_rer| > 1e-10)."""
import numpy as np
import pytest

import soundings
from util import budgets

TE_MAX, TW_MAX = 1e-14, 1e-10


def _consts(oracle):
    c = oracle.consts()
    return c[0], c[1], c[6]   # latvap (xlv), latice (xlf), gravit


def test_oracle_closes_the_budgets(oracle):
    s = soundings.make_soundings(2048, 30, seed=91)
    o = oracle.compute(s, diag=False)
    te, tw = budgets(s, o, *_consts(oracle))
    assert np.max(np.abs(te)) <= TE_MAX and np.max(np.abs(tw)) <= TW_MAX


@pytest.mark.gpu
def test_budget_kernel_matches_restatement(uw, oracle, cuda):
    assert uw.init_default() == 0
    s = soundings.make_soundings(4096, 35, seed=92)
    case = uw.DeviceCase(s)
    assert case.launch() == 0
    te_d, tw_d = case.budgets()
    te_h, tw_h = budgets(s, case.outputs_numpy(), *_consts(oracle))
    assert np.array_equal(te_d, te_h) and np.array_equal(tw_d, tw_h)


@pytest.mark.gpu
@pytest.mark.parametrize("pver,rh", [(30, (0.675, 0.93)), (51, (0.75, 0.97))])
def test_budgets_close_at_full_size(uw, cuda, pver, rh):
    """259,200 columns, the benchmark workload (30 levels) and a 51-level, 60 %-convecting one."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(259_200, pver, seed=93, rh_pbl=rh)
    case = uw.DeviceCase(s)
    assert case.launch() == 0
    assert case.status() == 0
    te, tw = case.budgets()
    conv = int(np.sum(case.outputs_numpy()["cush"] != -1.0))
    assert conv > 0.3 * 259_200
    assert np.max(np.abs(te)) <= TE_MAX, (np.max(np.abs(te)), int(np.sum(np.abs(te) > TE_MAX)))
    assert np.max(np.abs(tw)) <= TW_MAX, (np.max(np.abs(tw)), int(np.sum(np.abs(tw) > TW_MAX)))
