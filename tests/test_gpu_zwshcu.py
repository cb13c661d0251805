"""compute_zwshcu (zwshcu.F90) on the GPU through the C ABI against the oracle build with the kernel's
math routines: bit for bit on every output, for the device entry (both level orders, 30 and 51
levels), the host entries compute_zwshcu_ and compute_zwshcu_inv_, and every option of the variant;
omega = 0 gives compute_uwshcu's bits."""
import numpy as np
import pytest

import soundings
from util import FIELDS

pytestmark = pytest.mark.gpu


def _same(out, ref):
    return [f for f in FIELDS if not np.array_equal(out[f], ref[f])]


def _bottom_up(out, mkx):
    """Outputs of a call in CAM's top-down order, put back in compute_zwshcu's bottom-up order."""
    b = {}
    for k, v in out.items():
        if k in ("cnt", "cnb"):
            b[k] = (mkx + 1) - v
        elif isinstance(v, np.ndarray) and v.ndim >= 2:
            b[k] = np.ascontiguousarray(v[..., ::-1, :])
        else:
            b[k] = v
    return b


@pytest.mark.parametrize("opts", [{}, {"ent": 1}, {"cloud_sh": 1}, {"lf": 0, "fwcrit": 0.7},
                                  {"ent": 1, "cloud_sh": 1, "ufrcz": 1.5}])
def test_device_entry_matches_oracle(uw, oracle_pm, cuda, opts):
    torch = cuda
    s = soundings.make_soundings(3000, 30, seed=21)
    om = soundings.make_omega(s, seed=21, mean=-0.5, sd=1.0)
    try:
        assert uw.set_zw_options(**opts) == 0
        oracle_pm.set_zw_options(**opts)
        ref = oracle_pm.compute(s, diag=True, omega=om)
        case = uw.DeviceCase(s, diag=True)
        assert case.launch(omega=torch.from_numpy(om).cuda()) == 0, uw.last_cuda_error()
        assert case.status() == ref["status"]
        out = case.outputs_numpy()
        assert not _same(out, ref)
        assert np.array_equal(out["diag_int"], ref["diag_int"])
    finally:
        assert uw.set_zw_options() == 0
        oracle_pm.set_zw_options()


@pytest.mark.parametrize("pver,inv", [(30, 1), (51, 0)])
def test_level_orders_and_counts(uw, oracle_pm, cuda, pver, inv):
    torch = cuda
    s = soundings.make_soundings(1500, pver, seed=22 + pver)
    om = soundings.make_omega(s, seed=22, mean=-0.5, sd=1.0)
    ref = oracle_pm.compute(s, diag=False, omega=om)
    si = soundings.to_inv(s) if inv else s
    omi = np.ascontiguousarray(om[::-1]) if inv else om
    case = uw.DeviceCase(si)
    assert case.launch(inv=inv, omega=torch.from_numpy(omi).cuda()) == 0
    out = case.outputs_numpy()
    if inv:
        out = _bottom_up(out, pver)
    assert not _same(out, ref)


def test_host_entries(uw, oracle_pm, cuda):
    s = soundings.make_soundings(5000, 30, seed=23)
    om = soundings.make_omega(s, seed=23, mean=-0.5, sd=1.0)
    ref = oracle_pm.compute(s, diag=False, omega=om)
    rc, out = uw.compute_host(s, entry="compute_zwshcu_", omega=om)
    assert rc == ref["status"] and not _same(out, ref)
    rc, outi = uw.compute_host(soundings.to_inv(s), entry="compute_zwshcu_inv_",
                               omega=np.ascontiguousarray(om[::-1]))
    assert rc == ref["status"]
    assert not _same(_bottom_up(outi, 30), ref)


def test_zero_omega_gives_compute_uwshcu(uw, cuda):
    torch = cuda
    s = soundings.make_soundings(2000, 30, seed=24)
    a = uw.DeviceCase(s)
    assert a.launch() == 0
    b = uw.DeviceCase(s, inputs=a.inp)
    assert b.launch(omega=torch.zeros((30, 2000), dtype=torch.float64, device="cuda")) == 0
    assert not _same(a.outputs_numpy(), b.outputs_numpy())
