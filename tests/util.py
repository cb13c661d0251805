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
