"""Property tests of the oracle's restatements of the uwshcu.F90 helpers (CPU only)."""
import ctypes

import numpy as np
import pytest

import soundings

D = ctypes.c_double
PD = ctypes.POINTER(ctypes.c_double)


def _out():
    return D(0.0)


def conden(L, p, thl, qt):
    th, qv, ql, qi, rv = D(), D(), D(), D(), D()
    idc = ctypes.c_int()
    L.uwo_conden(D(p), D(thl), D(qt), ctypes.byref(th), ctypes.byref(qv), ctypes.byref(ql),
                 ctypes.byref(qi), ctypes.byref(rv), ctypes.byref(idc))
    return th.value, qv.value, ql.value, qi.value, idc.value


def qsat(L, t, p):
    es, qs, gam = D(), D(), D()
    L.uwo_qsat(D(t), D(p), ctypes.byref(es), ctypes.byref(qs), ctypes.byref(gam))
    return es.value, qs.value, gam.value


@pytest.fixture(scope="module")
def L(oracle):
    return oracle.lib()


def test_table_knots_are_goff_gratch(oracle):
    t = 173.16 + np.arange(204)
    tbl = oracle.estbl()
    ref = soundings._esat(t)
    assert np.allclose(tbl[:204], ref, rtol=1e-12, atol=0)
    assert np.all(tbl[204:] == -99999.0)


def test_conden_conserves_qt_and_liquid_temperature(L, oracle):
    c = oracle.consts()
    xlv, xls, cp = c[0], c[2], c[3]
    rng = np.random.default_rng(0)
    for _ in range(400):
        p = rng.uniform(3e4, 1.02e5)
        t = rng.uniform(230.0, 305.0)
        ex = L.uwo_exnf(D(p))
        qs = qsat(L, t, p)[1]
        qt = qs * rng.uniform(0.5, 1.6)
        thl = t / ex
        th, qv, ql, qi, idc = conden(L, p, thl, qt)
        assert idc == 0
        assert qv + ql + qi == pytest.approx(qt, rel=1e-15, abs=1e-18)
        assert ql >= 0 and qi >= 0
        tt = th * ex
        # liquid-water temperature of the adjusted state equals the input to the Newton tolerance
        assert abs((tt - (xlv * ql + xls * qi) / cp) - thl * ex) < 2e-2
        if ql + qi > 0:
            assert qv == pytest.approx(qsat(L, tt, p)[1], rel=1e-6)


def test_roots_solves_the_quadratic(L):
    rng = np.random.default_rng(1)
    for _ in range(300):
        a, b, c = rng.normal(size=3)
        r1, r2, st = D(), D(), ctypes.c_int()
        L.uwo_roots(D(a), D(b), D(c), ctypes.byref(r1), ctypes.byref(r2), ctypes.byref(st))
        if b * b - 4 * a * c < 0:
            assert st.value == 3
            continue
        assert st.value == 0
        for r in (r1.value, r2.value):
            assert abs(a * r * r + b * r + c) <= 1e-9 * (abs(a * r * r) + abs(b * r) + abs(c) + 1e-300)
    r1, r2, st = D(5.0), D(6.0), ctypes.c_int()
    L.uwo_roots(D(0.0), D(0.0), D(1.0), ctypes.byref(r1), ctypes.byref(r2), ctypes.byref(st))
    assert st.value == 1 and r1.value == 5.0 and r2.value == 5.0     # r1 untouched, r2 = r1
    L.uwo_roots(D(1.0), D(0.0), D(1.0), ctypes.byref(r1), ctypes.byref(r2), ctypes.byref(st))
    assert st.value == 2


def test_slope_is_a_monotone_limiter(L):
    rng = np.random.default_rng(2)
    for _ in range(100):
        n = 30
        p = np.sort(rng.uniform(1e3, 1e5, n))[::-1].copy()
        f = np.cumsum(rng.normal(size=n))
        out = np.zeros(n)
        L.uwo_slope(ctypes.c_int(n), f.ctypes.data_as(PD), p.ctypes.data_as(PD), out.ctypes.data_as(PD))
        g = np.diff(f) / np.diff(p)
        for k in range(1, n - 1):
            lo, hi = g[k - 1], g[k]
            s = out[k]
            # limited to the smaller neighbouring gradient, zero at extrema
            if np.sign(lo) != np.sign(hi):
                assert s == 0.0
            else:
                assert abs(s) <= min(abs(lo), abs(hi)) + 1e-300
        assert out[-1] == out[-2]


def test_qsinvert_returns_the_saturation_pressure(L, oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        ps = rng.uniform(9.5e4, 1.02e5)
        t = rng.uniform(280.0, 303.0)
        rh = rng.uniform(0.3, 0.98)
        ex = L.uwo_exnf(D(ps))
        qt = rh * qsat(L, t, ps)[1]
        thl = t / ex
        plcl = L.uwo_qsinvert(D(qt), D(thl), D(ps))
        assert 3e4 < plcl <= ps
        tl = thl * L.uwo_exnf(D(plcl))
        assert qsat(L, tl, plcl)[1] == pytest.approx(qt, rel=2e-4)


def test_findsp_conserves_enthalpy(L, oracle):
    c = oracle.consts()
    s = soundings.make_soundings(64, 30, seed=4)
    n, k = 64, 30
    tsp = np.zeros((k, n))
    qsp = np.zeros((k, n))
    st = L.uwo_findsp(ctypes.c_int(n), ctypes.c_int(n), ctypes.c_int(k), s["qv0"].ctypes.data_as(PD),
                      s["t0"].ctypes.data_as(PD), s["p0"].ctypes.data_as(PD), tsp.ctypes.data_as(PD),
                      qsp.ctypes.data_as(PD))
    assert st == 0
    cp, xlv = c[3], c[0]
    hin = cp * s["t0"] + xlv * s["qv0"]
    hout = cp * tsp + xlv * qsp
    assert np.max(np.abs(hin - hout) / hin) < 2e-3
    # wet bulb is colder than the air and moister for sub-saturated air
    assert np.all(tsp <= s["t0"] + 1e-9)
    assert np.all(qsp >= s["qv0"] - 1e-12)


def test_fluxbelowinv_has_zero_surface_flux(L):
    ps0 = np.linspace(1.0e5, 3.0e4, 31)
    xflx = np.zeros(31)
    for kinv in (2, 5, 9):
        L.uwo_fluxbelowinv(D(0.02), ps0.ctypes.data_as(PD), ctypes.c_int(30), ctypes.c_int(kinv),
                           D(1800.0), D(0.012), D(0.010), D(0.006), D(0.011), xflx.ctypes.data_as(PD))
        assert xflx[0] == 0.0
        assert np.all(xflx[kinv:] == 0.0)


def test_positive_moisture_preserves_column_water(L, oracle):
    c = oracle.consts()
    rng = np.random.default_rng(5)
    for _ in range(50):
        n = 30
        dp = rng.uniform(500.0, 4000.0, n)
        qv = rng.uniform(1e-6, 1e-2, n)
        ql = rng.uniform(-1e-5, 1e-4, n)
        qi = rng.uniform(-1e-5, 1e-4, n)
        qv[rng.integers(0, n, 3)] = -1e-5
        s = np.full(n, 3.0e5)
        ten = [np.zeros(n) for _ in range(4)]
        before = np.sum((qv + ql + qi) * dp)
        args = [a.ctypes.data_as(PD) for a in (dp, qv, ql, qi, s, *ten)]
        L.uwo_positive_moisture_single(D(c[0]), D(c[2]), ctypes.c_int(n), D(1800.0), D(1e-12), D(0.0),
                                       D(0.0), *args)
        after = np.sum((qv + ql + qi) * dp)
        assert after == pytest.approx(before, rel=1e-10)
        assert np.all(ql >= 0) and np.all(qi >= 0)


def test_compute_alpha_is_the_implicit_fixed_point(L):
    for dcin, ke in ((5.0, 0.3), (40.0, 0.05), (0.5, 2.0)):
        a = L.uwo_compute_alpha(D(dcin), D(ke))
        assert a == pytest.approx(np.exp(-a * ke * dcin), rel=1e-12)
