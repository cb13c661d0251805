"""Seeded synthetic soundings for the UW shallow-cumulus driver.

The reference ships no input data (its benchmark drivers fill arrays with non-physical values such
as ``p0 = i + j + 2.1``, src/doubleGPUUWshcu/mpiuwshcu.cpp:6768-6802), so columns are generated here
with the distributions the workload definitions name:

* surface pressure ~ N(98500, 1500) Pa on a hybrid sigma-pressure grid defined below (the CAM
  hyai/hybi coefficients are not part of the reference tree);
* surface temperature ~ U(280, 303) K, 6.5 K/km lapse rate up to a 200 hPa tropopause, isothermal
  above; heights by hypsometric integration of the virtual temperature from z = 0 at the surface;
* relative humidity ~ U(rh_lo, rh_hi) inside the PBL, decaying linearly in pressure to 0.20 at
  300 hPa and 0.20 above; qv = RH * qs(T, p);
* ql, qi ~ U(0, 1e-4) kg/kg in a random 0-30 % of the levels (liquid where T > 248 K, ice where
  T < 268 K); number tracers nl = 1e8 * ql, ni = 1e6 * qi;
* u, v ~ N(0, 8) m/s; tke ~ U(0.1, 2) m2/s2 at interfaces below the PBL top and 0.01 above;
  pblh ~ U(300, 2000) m; cldfrct, concldfrct ~ U(0, 0.3); cush = 1000 m; dt = 1800 s.

Arrays are returned in the Fortran layout of compute_uwshcu (uwshcu.F90:529-550): numpy shape
(levels, ncol) in C order is the column-major (mix, levels) array with the column index fastest,
k = 0 at the surface (interfaces) or k = 1 at the lowest layer (layers, stored at row k-1).
Tracers are (ncnst, mkx, ncol).
"""
import numpy as np

# Physical constants (CESM shr_const values; the same ones the library is initialised with).
_BOLTZ = 1.38065e-23
_AVOGAD = 6.02214e26
_RGAS = _AVOGAD * _BOLTZ
_MWDAIR = 28.966
_MWWV = 18.016
RAIR = _RGAS / _MWDAIR
RH2O = _RGAS / _MWWV
ZVIR = RH2O / RAIR - 1.0
EPSILO = _MWWV / _MWDAIR
CPAIR = 1.00464e3
GRAVIT = 9.80616
TMELT = 273.15
LATVAP = 2.501e6
LATICE = 3.337e5

FIELDS_IFACE = ("ps0", "zs0", "tke")
FIELDS_LAYER = ("p0", "z0", "dp0", "u0", "v0", "qv0", "ql0", "qi0", "t0", "s0", "cldfrct",
                "concldfrct", "dpdry0")


def _esat(t):
    """Goff-Gratch saturation vapour pressure [Pa] with the 20 K water-ice transition below
    freezing (the same relationships gffgch.F90 tabulates)."""
    t = np.asarray(t, dtype=np.float64)
    ts = 373.16
    e1 = 11.344 * (1.0 - t / ts)
    e2 = -3.49149 * (ts / t - 1.0)
    f = (-7.90298 * (ts / t - 1.0) + 5.02808 * np.log10(ts / t)
         - 1.3816 * (10.0 ** e1 - 1.0) / 1.0e7 + 8.1328 * (10.0 ** e2 - 1.0) / 1.0e3
         + np.log10(1013.246))
    esw = 10.0 ** f * 100.0
    t0 = TMELT
    esi = 575.185606e10 * np.exp(-(2.01889049 / (t0 / t) + 3.56654 * np.log(t0 / t)
                                   + 20.947031 * (t0 / t)))
    w = np.clip((TMELT - t) / 20.0, 0.0, 1.0)
    return np.where(t >= TMELT, esw, w * esi + (1.0 - w) * esw)


def qsat(t, p):
    """Saturation specific humidity [kg/kg]."""
    es = _esat(t)
    return np.minimum(EPSILO * es / (p - (1.0 - EPSILO) * es), 1.0)


def hybrid_coefficients(pver, ptop=300.0, pref=1.0e5, eta_pure=0.2):
    """Interface coefficients (A, B) of a hybrid grid with pver layers, ordered surface (index 0)
    to model top (index pver): p_int = A * pref + B * ps.  Reference-pressure fractions follow
    eta(x) = ptop/pref + (1 - ptop/pref) * (x/2 + sin(pi x / 2)/2), x in [0, 1] top to bottom,
    which gives ~17 hPa layers near the ground; B rises from 0 at eta_pure to 1 at the surface."""
    x = np.linspace(0.0, 1.0, pver + 1)
    e0 = ptop / pref
    eta = e0 + (1.0 - e0) * (0.5 * x + 0.5 * np.sin(0.5 * np.pi * x))
    b = np.clip((eta - eta_pure) / (1.0 - eta_pure), 0.0, None) ** 1.5
    a = eta - b
    return a[::-1].copy(), b[::-1].copy()


def make_soundings(ncol, pver=30, seed=0, rh_pbl=(0.70, 0.95), ncnst=5, dt=1800.0):
    """Generate ncol independent columns.  Returns a dict of float64 arrays in the Fortran layout
    described in the module docstring, plus 'dt', 'mkx', 'ncnst', 'seed'."""
    if ncnst < 5:
        raise ValueError("ncnst must be >= 5 (qv, ql, qi, nl, ni)")
    rng = np.random.Generator(np.random.PCG64(seed))
    n, mkx = int(ncol), int(pver)
    a, b = hybrid_coefficients(mkx)
    ps = rng.normal(98500.0, 1500.0, n)
    ps0 = a[:, None] * 1.0e5 + b[:, None] * ps[None, :]            # (mkx+1, n), k = 0 surface
    p0 = 0.5 * (ps0[:-1] + ps0[1:])
    dp0 = ps0[:-1] - ps0[1:]
    tsfc = rng.uniform(280.0, 303.0, n)
    expo = RAIR * 6.5e-3 / GRAVIT
    ttrop = tsfc * (20000.0 / ps) ** expo
    t0 = np.where(p0 > 20000.0, tsfc[None, :] * (p0 / ps[None, :]) ** expo, ttrop[None, :])

    def heights(tv):
        zs = np.zeros_like(ps0)
        zs[1:] = np.cumsum(RAIR * tv / GRAVIT * np.log(ps0[:-1] / ps0[1:]), axis=0)
        z = zs[:-1] + RAIR * tv / GRAVIT * np.log(ps0[:-1] / p0)
        return zs, z

    zs0, z0 = heights(t0)
    pblh = rng.uniform(300.0, 2000.0, n)
    rh_sfc = rng.uniform(rh_pbl[0], rh_pbl[1], n)
    inpbl = z0 < pblh[None, :]
    # pressure at the PBL top: the lowest layer midpoint above pblh
    kt = np.argmax(~inpbl, axis=0)
    ptopbl = p0[kt, np.arange(n)]
    frac = np.clip((p0 - 30000.0) / np.maximum(ptopbl[None, :] - 30000.0, 1.0), 0.0, 1.0)
    rh = np.where(inpbl, rh_sfc[None, :], 0.20 + (rh_sfc[None, :] - 0.20) * frac)
    rh = np.where(p0 <= 30000.0, 0.20, rh)
    qv0 = rh * qsat(t0, p0)
    cloudy = rng.uniform(0.0, 0.3, n)
    liqmask = (rng.uniform(size=(mkx, n)) < cloudy[None, :]) & (t0 > 248.0)
    icemask = (rng.uniform(size=(mkx, n)) < cloudy[None, :]) & (t0 < 268.0)
    ql0 = np.where(liqmask, rng.uniform(0.0, 1.0e-4, (mkx, n)), 0.0)
    qi0 = np.where(icemask, rng.uniform(0.0, 1.0e-4, (mkx, n)), 0.0)
    tv = t0 * (1.0 + ZVIR * qv0 - ql0 - qi0)
    zs0, z0 = heights(tv)
    s0 = CPAIR * t0 + GRAVIT * z0
    u0 = rng.normal(0.0, 8.0, (mkx, n))
    v0 = rng.normal(0.0, 8.0, (mkx, n))
    tke = np.where(zs0 < pblh[None, :], rng.uniform(0.1, 2.0, (mkx + 1, n)), 0.01)
    cldfrct = rng.uniform(0.0, 0.3, (mkx, n))
    concldfrct = rng.uniform(0.0, 0.3, (mkx, n))
    qt = qv0 + ql0 + qi0
    dpdry0 = dp0 * (1.0 - qt)
    tr0 = np.zeros((ncnst, mkx, n))
    tr0[0], tr0[1], tr0[2] = qv0, ql0, qi0
    tr0[3] = 1.0e8 * ql0
    tr0[4] = 1.0e6 * qi0
    for m in range(5, ncnst):
        tr0[m] = rng.uniform(0.0, 1.0e-9, (mkx, n)) * (rng.uniform(size=(mkx, n)) < 0.9)
    cush = np.full(n, 1000.0)
    out = dict(ps0=ps0, zs0=zs0, p0=p0, z0=z0, dp0=dp0, u0=u0, v0=v0, qv0=qv0, ql0=ql0, qi0=qi0,
               t0=t0, s0=s0, tr0=tr0, tke=tke, cldfrct=cldfrct, concldfrct=concldfrct, pblh=pblh,
               cush=cush, dpdry0=dpdry0, massflx_sh=np.zeros(n))
    out = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in out.items()}
    out.update(dt=float(dt), mkx=mkx, ncnst=int(ncnst), seed=int(seed), ncol=n)
    return out


def make_omega(s, seed=0, mean=-0.05, sd=0.3):
    """Large-scale pressure velocity omega (mkx, ncol) [Pa/s] for compute_zwshcu, bottom-up like the
    other layer fields: a first-baroclinic-mode profile omega0 sin(pi (ps - p) / (ps - 10 kPa)) below
    100 hPa (zero above) with omega0 ~ N(mean, sd) per column (negative: ascent), plus N(0, 0.02)
    per level.  Every column's own surface pressure ps0[0]."""
    rng = np.random.default_rng(10_000 + seed)
    n, mkx = s["ncol"], s["mkx"]
    ps = s["ps0"][0]
    p = s["p0"]
    w0 = rng.normal(mean, sd, n)
    x = np.clip((ps - p) / (ps - 1.0e4), 0.0, 1.0)
    om = w0 * np.sin(np.pi * x) + rng.normal(0.0, 0.02, (mkx, n))
    om = np.where(p < 1.0e4, 0.0, om)
    return np.ascontiguousarray(om, dtype=np.float64)


def to_inv(s):
    """Return a copy of a sounding dict in CAM's top-down level order (compute_uwshcu_inv input
    layout, uwshcu.F90:274-297)."""
    out = dict(s)
    for k in FIELDS_IFACE + FIELDS_LAYER:
        out[k] = np.ascontiguousarray(s[k][::-1])
    out["tr0"] = np.ascontiguousarray(s["tr0"][:, ::-1])
    return out
