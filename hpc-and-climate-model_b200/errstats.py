"""Error of a reduced-precision run of compute_uwshcu against the FP64 path on the same inputs.

The FP64 path reproduces the oracle bit for bit, so these are errors against the FP64 oracle.
Reported per output field and for the three column quantities the precision targets name:
column heating  H = sum_k sten(k) dp0(k) / g       (W m-2)
column moistening M = sum_k qvten(k) dp0(k) / g     (kg m-2 s-1)
precipitation     P = precip                        (m s-1)
with the relative RMS  sqrt(mean((x - x64)^2)) / sqrt(mean(x64^2))  over all columns, the
largest relative column error, the count of columns whose trigger, cloud base or cloud top
decision differs, and the distribution of the columns' errors behind the RMS.
"""
import numpy as np

G = 9.80616
FIELDS = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu", "qvten", "qlten", "qiten", "sten",
          "uten", "vten", "qrten", "qsten", "evapc", "cufrc", "qcu", "qlu", "qiu", "qc", "trten",
          "precip", "snow", "cbmf", "rliq", "cush")


def column_quantities(out, dp0):
    return {"heating": (out["sten"] * dp0).sum(axis=0) / G,
            "moistening": (out["qvten"] * dp0).sum(axis=0) / G,
            "precipitation": np.asarray(out["precip"], dtype=np.float64)}


def rel_rms(a, b):
    den = float(np.sqrt(np.mean(np.square(b))))
    num = float(np.sqrt(np.mean(np.square(a - b))))
    return num / den if den > 0 else num


def report(out, ref, dp0):
    """Errors of `out` against `ref` (dicts of the ABI outputs, column index last)."""
    n = np.asarray(ref["precip"]).shape[-1]
    rep = {"columns": int(n)}
    fields = {}
    for f in FIELDS:
        a = np.asarray(out[f], dtype=np.float64).reshape(-1, n)
        b = np.asarray(ref[f], dtype=np.float64).reshape(-1, n)
        scale = float(np.abs(b).max()) or 1.0
        fields[f] = {"rel_rms": rel_rms(a, b), "max_abs_over_max": float(np.abs(a - b).max()) / scale}
    rep["fields"] = fields
    qa, qb = column_quantities(out, dp0), column_quantities(ref, dp0)
    rep["column"] = {}
    for k in qb:
        scale = float(np.abs(qb[k]).max()) or 1.0
        rep["column"][k] = {"rel_rms": rel_rms(qa[k], qb[k]),
                            "max_abs_over_max": float(np.abs(qa[k] - qb[k]).max()) / scale}
    trig_a, trig_b = out["cush"] != -1.0, ref["cush"] != -1.0
    rep["flips"] = {"trigger": int(np.sum(trig_a != trig_b)),
                    "cloud_base": int(np.sum(out["cnb"] != ref["cnb"])),
                    "cloud_top": int(np.sum(out["cnt"] != ref["cnt"])),
                    "convecting_columns": int(np.sum(trig_b))}
    rep["worst_column_rel_rms"] = max(v["rel_rms"] for v in rep["column"].values())
    same = ((trig_a == trig_b) & (np.asarray(out["cnb"]) == np.asarray(ref["cnb"])) &
            (np.asarray(out["cnt"]) == np.asarray(ref["cnt"])))
    rep["distribution"] = distribution(qa, qb, same & trig_b)
    return rep


def distribution(qa, qb, sel):
    """How the relative RMS of each column quantity is made: percentiles (50, 90, 99, 99.9) of the
    columns' relative errors |x - x64| / max(|x64|, 1e-3 rms(x64)) over the columns in `sel` (the
    convecting columns whose trigger, cloud base and cloud top are the FP64 path's), and the share
    of the summed squared error that the worst 0.1 % and 1 % of all columns carry."""
    res = {}
    for k in qb:
        a, b = np.asarray(qa[k], dtype=np.float64), np.asarray(qb[k], dtype=np.float64)
        rms = float(np.sqrt(np.mean(np.square(b)))) or 1.0
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * rms)
        d2 = np.sort(np.square(a - b))[::-1]
        tot = float(d2.sum())
        n = d2.size
        res[k] = {"rel_percentiles_same_decisions": [float(np.percentile(rel[sel], p)) if np.any(sel) else 0.0
                                                     for p in (50, 90, 99, 99.9)],
                  "sq_error_share_worst_0.1pct": float(d2[: max(1, n // 1000)].sum() / tot) if tot > 0 else 0.0,
                  "sq_error_share_worst_1pct": float(d2[: max(1, n // 100)].sum() / tot) if tot > 0 else 0.0}
    return res
