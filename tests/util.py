"""Comparison helpers shared by the parity tests."""
import numpy as np

FIELDS = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu", "qvten", "qlten", "qiten", "sten",
          "uten", "vten", "qrten", "qsten", "evapc", "cufrc", "qcu", "qlu", "qiu", "qc", "trten",
          "precip", "snow", "cbmf", "rliq", "cnt", "cnb", "cush")


def column_rel_err(a, b):
    """Norm-wise relative error per column: max_k |a-b| / max_k |b| (0 where both are all zero).
    Arrays have the column index last."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = b.shape[-1]
    a2 = a.reshape(-1, n)
    b2 = b.reshape(-1, n)
    num = np.max(np.abs(a2 - b2), axis=0)
    den = np.max(np.abs(b2), axis=0)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(den > 0, num / np.where(den > 0, den, 1.0), np.where(num > 0, np.inf, 0.0))
    return r


def compare(out, ref, tol=1e-11, fields=FIELDS, ncol=None):
    """Return {field: (fraction of columns within tol, max column error)} and the worst column
    errors over all fields."""
    res = {}
    worst = None
    for f in fields:
        a, b = out[f], ref[f]
        if ncol is not None:
            a, b = a[..., :ncol], b[..., :ncol]
        e = column_rel_err(a, b)
        worst = e if worst is None else np.maximum(worst, e)
        res[f] = (float(np.mean(e <= tol)), float(np.max(e)))
    return res, worst


def decisions(out):
    """Trigger (column convects), cloud-base and cloud-top interface indices."""
    return (out["cush"] != -1.0), out["cnb"], out["cnt"]


def conditioned_compare(out, ref, ncol=None, floor_rel=1e-9):
    """Column errors with a per-field absolute floor of floor_rel * max|ref field|: the measure for
    comparisons across two different (ulp-accurate) implementations of exp/log/pow/erfc, whose
    last-bit differences the scheme amplifies.  Returns the worst error per column."""
    worst = None
    for f in FIELDS:
        a = np.asarray(out[f], dtype=np.float64)
        b = np.asarray(ref[f], dtype=np.float64)
        if ncol is not None:
            a, b = a[..., :ncol], b[..., :ncol]
        n = b.shape[-1]
        a2, b2 = a.reshape(-1, n), b.reshape(-1, n)
        fl = floor_rel * float(np.abs(b2).max()) if b2.size else 0.0
        num = np.abs(a2 - b2).max(axis=0)
        den = np.maximum(np.abs(b2).max(axis=0), fl)
        with np.errstate(invalid="ignore", divide="ignore"):
            e = np.where(den > 0, num / np.where(den > 0, den, 1.0), np.where(num > 0, np.inf, 0.0))
        worst = e if worst is None else np.maximum(worst, e)
    return worst


def budgets(s, o, latvap, latice, g, inv=0):
    """check_energy_chng (check_energy.F90:321-395) as CAM applies it after the shallow scheme
    (tphysbc.F90:446-447), evaluated in CAM's level order with the expressions of the device
    budget kernel: relative energy and water errors te_rer, tw_rer per column."""
    dt = s["dt"]
    dp0, u0, v0, s0 = s["dp0"], s["u0"], s["v0"], s["s0"]
    qv0, ql0, qi0 = s["qv0"], s["ql0"], s["qi0"]
    mkx, n = dp0.shape
    te0, tw0, te1, tw1 = (np.zeros(n) for _ in range(4))
    for j in range(mkx):
        r = j if inv else mkx - 1 - j
        dp = dp0[r]
        u, v, sv, qv, ql, qi = u0[r], v0[r], s0[r], qv0[r], ql0[r], qi0[r]
        u1, v1, s1 = u + o["uten"][r] * dt, v + o["vten"][r] * dt, sv + o["sten"][r] * dt
        qv1, ql1, qi1 = qv + o["qvten"][r] * dt, ql + o["qlten"][r] * dt, qi + o["qiten"][r] * dt
        te0 = te0 + 0.5 * (u * u + v * v) * dp / g + sv * dp / g + (latvap + latice) * qv * dp / g + latice * ql * dp / g
        tw0 = tw0 + (qv + ql + qi) * dp / g
        te1 = te1 + 0.5 * (u1 * u1 + v1 * v1) * dp / g + s1 * dp / g + (latvap + latice) * qv1 * dp / g + latice * ql1 * dp / g
        tw1 = tw1 + (qv1 + ql1 + qi1) * dp / g
    flx_cnd = o["precip"] + o["rliq"]
    te_tnd = -(flx_cnd - o["snow"]) * 1000.0 * latice
    tw_tnd = -flx_cnd * 1000.0
    te_rer = ((te0 + te_tnd * dt) - te1) / te0
    with np.errstate(invalid="ignore", divide="ignore"):
        tw_rer = np.where(tw0 > 0.0, ((tw0 + tw_tnd * dt) - tw1) / tw0, 0.0)
    return te_rer, tw_rer
