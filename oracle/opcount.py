"""Algorithmic FP64 operations per column of compute_uwshcu, counted by the operation-counting
oracle build (opcount.hpp: + - * / sqrt and one per exp/log/pow/erfc/log10) on seeded synthetic
soundings of each benchmark workload (TEST AND MEASUREMENT INFRASTRUCTURE; the product never loads
it).  Writes profiles/flops_per_column.json, which bench.py reads for its FP64 roofline:
per workload the mean operations of a convecting and of a non-convecting column.

    python oracle/opcount.py [--sample 8192]
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(REPO, "hpc-and-climate-model_b200")]
import oracle  # noqa: E402
import soundings  # noqa: E402

# (name, total columns of the workload, levels, PBL RH draw, seed): the sample is the first
# `sample` columns of the workload as bench.py generates it
WORKLOADS = (
    ("fp64_259200x30", 259_200, 30, (0.675, 0.93), 1),
    ("batched_member_30L_5pct", 262_144, 30, (0.55, 0.757), 100),
    ("batched_member_35L_25pct", 262_144, 35, (0.625, 0.86), 101),
    ("batched_member_51L_45pct", 262_144, 51, (0.662, 0.912), 102),
    ("batched_member_30L_60pct", 262_144, 30, (0.75, 0.97), 103),
)
KINDS = ("add", "mul", "div", "sqrt", "tr")


def subset(s, idx):
    o = dict(s)
    n = s["ncol"]
    for k, v in s.items():
        if isinstance(v, np.ndarray) and v.shape[-1] == n:
            o[k] = np.ascontiguousarray(v[..., idx])
    o["ncol"] = int(len(idx))
    return o


def count(s):
    oracle.set_variant("ops")
    oracle.init_default()
    L = oracle.lib()
    buf = (ctypes.c_ulonglong * 5)()
    L.uwo_opcount(buf, 1)
    oracle.compute(s, diag=False, nthreads=1)
    L.uwo_opcount(buf, 1)
    return dict(zip(KINDS, (int(x) for x in buf)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sample", type=int, default=8192)
    ap.add_argument("--out", default=os.path.join(REPO, "profiles", "flops_per_column.json"))
    args = ap.parse_args()
    res = {"what": "algorithmic FP64 operations per column (+ - * / sqrt, one per exp/log/pow/erfc), "
                   "counted by the oracle's operation-counting build on the first columns of each "
                   "workload; generated by oracle/opcount.py", "workloads": {}}
    for name, n, pver, rh, seed in WORKLOADS:
        s = soundings.make_soundings(n, pver, seed=seed, rh_pbl=rh)
        s = subset(s, np.arange(min(args.sample, n)))
        oracle.set_variant("glibc")
        oracle.init_default()
        conv = oracle.compute(s, diag=False)["cush"] != -1.0
        cc = count(subset(s, np.where(conv)[0]))
        cn = count(subset(s, np.where(~conv)[0]))
        nc, nn = int(conv.sum()), int((~conv).sum())
        per = lambda c, m: {k: c[k] / max(m, 1) for k in KINDS}
        pc, pn = per(cc, nc), per(cn, nn)
        res["workloads"][name] = {
            "levels": pver, "sample_columns": nc + nn, "convecting_fraction": nc / (nc + nn),
            "ops_per_convecting_column": sum(pc.values()), "ops_per_other_column": sum(pn.values()),
            "convecting_breakdown": pc, "other_breakdown": pn}
        print(name, "convecting %.3f  ops/convecting column %.4g  ops/other column %.4g" % (
            nc / (nc + nn), sum(pc.values()), sum(pn.values())), flush=True)
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    oracle.set_variant("glibc")


if __name__ == "__main__":
    main()
