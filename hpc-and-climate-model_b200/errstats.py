"""Error of a reduced-precision run of compute_uwshcu against the FP64 path on the same inputs.

The FP64 path reproduces the oracle bit for bit, so these are errors against the FP64 oracle.
Reported per output field and for the three column quantities the precision targets name:
column heating  H = sum_k sten(k) dp0(k) / g       (W m-2)
column moistening M = sum_k qvten(k) dp0(k) / g     (kg m-2 s-1)
precipitation     P = precip                        (m s-1)
with the relative RMS  sqrt(mean((x - x64)^2)) / sqrt(mean(x64^2))  over all columns, the
largest relative column error, and the count of columns whose trigger, cloud base or cloud top
decision differs.
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
    return rep
