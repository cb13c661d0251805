"""compute_zwshcu (zwshcu.F90), the CAS-ESM variant of the scheme, in the oracle: with omega = 0 it is
compute_uwshcu bit for bit (the variant's large-scale-forcing closure subtracts nothing), strong
large-scale ascent lowers wcrit and triggers more columns, descent changes nothing, and the
variant's entrainment and cloud-fraction options change the columns they act on."""
import numpy as np

import soundings
from util import FIELDS


def test_zero_omega_is_compute_uwshcu(oracle):
    s = soundings.make_soundings(3000, 30, seed=11)
    a = oracle.compute(s, diag=True)
    b = oracle.compute(s, diag=True, omega=np.zeros((30, 3000)))
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["diag_int"], b["diag_int"])


def test_large_scale_ascent_lowers_the_trigger_threshold(oracle):
    s = soundings.make_soundings(3000, 30, seed=12)
    om = soundings.make_omega(s, seed=12, mean=-1.0, sd=0.5)
    a = oracle.compute(s, diag=True)
    b = oracle.compute(s, diag=True, omega=om)
    assert (b["cush"] != -1.0).sum() > (a["cush"] != -1.0).sum()
    # descent (omega > 0) subtracts nothing (zwshcu.F90:2296: max(-omega, 0))
    c = oracle.compute(s, diag=True, omega=np.abs(om))
    assert all(np.array_equal(a[f], c[f]) for f in FIELDS)


def test_options_act(oracle):
    s = soundings.make_soundings(2000, 30, seed=13)
    om = soundings.make_omega(s, seed=13)
    base = oracle.compute(s, diag=True, omega=om)
    conv = base["cush"] != -1.0
    try:
        # the cloud-fraction option changes cufrc only
        oracle.set_zw_options(lf=1, cloud_sh=1)
        cs = oracle.compute(s, diag=True, omega=om)
        assert not np.array_equal(cs["cufrc"][:, conv], base["cufrc"][:, conv])
        assert all(np.array_equal(cs[f], base[f]) for f in FIELDS if f != "cufrc")
        # the buoyancy-based entrainment changes the updraft
        oracle.set_zw_options(lf=1, ent=1)
        en = oracle.compute(s, diag=True, omega=om)
        assert not np.array_equal(en["umf"], base["umf"])
        # the wcrit factor moves the closure
        oracle.set_zw_options(lf=0, fwcrit=0.5)
        fw = oracle.compute(s, diag=True, omega=om)
        assert not np.array_equal(fw["cbmf"], base["cbmf"])
    finally:
        oracle.set_zw_options()
    again = oracle.compute(s, diag=True, omega=om)
    assert all(np.array_equal(again[f], base[f]) for f in FIELDS)
