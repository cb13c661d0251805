#!/usr/bin/env python
"""Benchmark of the UW shallow-cumulus driver compute_uwshcu on B200.

Workload: 1,048,576 independent columns x 30 levels, 5 tracers (qv, ql, qi, nl, ni), dt = 1800 s,
seeded synthetic soundings (hpc-and-climate-model_b200/soundings.py) with the PBL relative humidity
drawn from U(0.675, 0.93) so that about 40 % of the columns convect.  A step is one compute_uwshcu
call over all columns.  Metric: columns per second.

  value : device-resident throughput of the FP64 path (inputs already in HBM,
          uwshcu_compute_device), CUDA events on the launching stream around exactly K steps;
          inputs (4.6 GB) exceed the 126 MB L2.
  e2e   : the same metric through the reference-facing C ABI compute_uwshcu_ with host arrays:
          the timed region includes the host->device copy of each step's inputs and the
          device->host copy of its outputs.
  mixed : the mixed-precision path on the same columns: columns/s, speed-up over FP64, relative
          RMS error of column heating, moistening and precipitation against the FP64 path (which is
          the FP64 oracle bit for bit), and the columns whose decisions change; fast: the same for
          the fast-FP64 mode.
  adjoint: the adjoint model against the forward pass on 65,536 x 30 columns (cost ratio, tape).
  batched: the batched uneven workload (4 x 262,144 columns, 30/35/51/30 levels) as one plan.
  zwshcu: compute_zwshcu (zwshcu.F90, the CAS-ESM variant) on the same columns with a synthetic
          large-scale pressure velocity.
  parity: the FP64 path on the 259,200 x 30 grid (720 x 360) against the oracle builds: decision
          agreement and the fraction of columns within 1e-11 on every output.
  --impl reference : the reference algorithm's CPU implementation (the C restatement in
          oracle/, compiled with -O2 -ffp-contract=off, OpenMP over all host cores) on a bounded
          sample of the same workload.

Multi-GPU (torchrun): every rank processes its own 1,048,576 columns (different seeds); columns
are independent, so there is no collective on the data path ("scaling": "weak").  Timing is the max
over ranks of the device time.  The mixed, adjoint and parity legs run at N = 1 only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "hpc-and-climate-model_b200")
sys.path.insert(0, PKG)

NCOL = 1_048_576
NCOL_GRID = 259_200       # the 720 x 360 grid of the parity leg
PVER = 30
NCNST = 5
RH_PBL = (0.675, 0.93)
METRIC = "columns/s (compute_uwshcu, FP64, 1,048,576 x 30 levels)"
G = 9.80616


# From the ncu capture of the worklist pass on the 65,536-column case of this workload (29,956
# worklist columns; summary in profiles/uwshcu_fp64_kernel_bench65k.txt, correctly rounded math,
# non-finite check fused into the loads): DRAM bytes read + written per worklist column by its two
# launches (UW_MODE_LIST1 7.420 GB + UW_MODE_RESUME 3.876 GB), and FP64 operations executed per
# worklist column (2 x DFMA + DADD + DMUL thread instructions per cycle x cycles of each launch:
# 707.70 x 17,051,704 + 561.79 x 14,282,396; the Newton steps of the IEEE divisions included).  Both
# scale with the columns a launch processes.  Constants of one capture: a change to the column code
# needs a new capture (the command is in the summary).
NCU_DRAM_BYTES_PER_LIST_COLUMN = 11.295961e9 / 29_956
NCU_FP64_OPS_PER_LIST_COLUMN = (707.70 * 17_051_704 + 561.79 * 14_282_396) / 29_956
FP64_DFMA_PER_CYCLE = 9472    # ncu sm__sass_thread_inst_executed_op_dfma_pred_on.sum.peak_sustained
# Algorithmic FP64 operations per convecting / other column of each workload, counted by the
# oracle's operation-counting build (written by oracle/opcount.py; a data file, read as text).
FLOPS_JSON = os.path.join(REPO, "profiles", "flops_per_column.json")


def algorithmic_ops(workload, ncol, convecting_fraction):
    """FP64 operations of one step over ncol columns of `workload`, or None."""
    try:
        with open(FLOPS_JSON) as f:
            w = json.load(f)["workloads"][workload]
    except (OSError, KeyError, ValueError):
        return None
    return ncol * (convecting_fraction * w["ops_per_convecting_column"] +
                   (1.0 - convecting_fraction) * w["ops_per_other_column"])


def bytes_per_column(mkx=PVER, ncnst=NCNST):
    """Algorithmic bytes of one column: inputs read + outputs written (FP64)."""
    n_in = 3 * (mkx + 1) + 10 * mkx + ncnst * mkx + 2
    n_out = 6 * (mkx + 1) + 14 * mkx + ncnst * mkx + 7
    return 8 * n_in, 8 * n_out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def shard_seed(rank):
    """Seed of rank `rank`'s columns: every rank generates and computes its own columns (the
    columns are independent, so there is no exchange step and no collective on the data path)."""
    return 1 + rank


def max_over_ranks(dist, value, device):
    """The largest `value` over all ranks (device times are reported as the max over ranks)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, ncol_per_rank, seconds):
    """Whole-job columns/s: the columns of all ranks over the slowest rank's time (weak scaling)."""
    return world * ncol_per_rank / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_reference(args):
    """CPU arm: the oracle (C restatement of the reference algorithm) on host cores."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    import soundings
    oracle.init_default()
    cores = os.cpu_count() or 1
    sample = int(args.cpu_sample)
    s = soundings.make_soundings(sample, PVER, seed=shard_seed(0), rh_pbl=RH_PBL)
    for _ in range(args.warmup if args.warmup < 1 else 1):
        oracle.compute(s, nthreads=cores, diag=False)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.compute(s, nthreads=cores, diag=False)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    val = sample / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "columns/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded soundings)",
        "config": {"workload": "compute_uwshcu 1,048,576 x 30 levels, 5 tracers, dt=1800 s; each "
                               "step a %d-column sample" % sample,
                   "ncol_sample": sample, "pver": PVER, "ncnst": NCNST},
        "cpu_baseline": {"value": val, "unit": "columns/s", "cores": cores, "kind": "port",
                         "sample": "the first %d columns of the 1,048,576-column workload "
                                   "per step" % sample},
        "e2e": {"value": val, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


OUT_FIELDS = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu", "qvten", "qlten", "qiten",
              "sten", "uten", "vten", "qrten", "qsten", "evapc", "cufrc", "qcu", "qlu", "qiu", "qc",
              "trten", "precip", "snow", "cbmf", "rliq", "cnt", "cnb", "cush")


def _column_errors(out, ref):
    """Worst norm-wise relative column error over all outputs (max_k |a-b| / max_k |b| per field)
    and the per-field fraction of columns within 1e-11."""
    worst, per = None, {}
    for f in OUT_FIELDS:
        a = np.asarray(out[f], dtype=np.float64)
        b = np.asarray(ref[f], dtype=np.float64)
        n = b.shape[-1]
        a, b = a.reshape(-1, n), b.reshape(-1, n)
        num = np.abs(a - b).max(axis=0)
        den = np.abs(b).max(axis=0)
        with np.errstate(invalid="ignore", divide="ignore"):
            e = np.where(den > 0, num / np.where(den > 0, den, 1.0), np.where(num > 0, np.inf, 0.0))
        per[f] = float(np.mean(e <= 1e-11))
        worst = e if worst is None else np.maximum(worst, e)
    return worst, per


def grid_case(uw):
    """The FP64 path on the 259,200-column grid (seed 0) with diagnostics: inputs and outputs."""
    import soundings
    s = soundings.make_soundings(NCOL_GRID, PVER, seed=0, rh_pbl=RH_PBL)
    case = uw.DeviceCase(s, diag=True)
    rc = case.launch()
    st = case.status()
    out = case.outputs_numpy()
    del case
    return s, out, rc, st


def cpu_baseline_leg(s, gpu_out):
    """The oracle (the C restatement of the reference algorithm, OpenMP over all host cores) timed
    on the 259,200-column grid, and, as the checker, compared with the FP64 path's outputs of the
    same inputs (gpu_out): the glibc build (pinned to the reference's C++ drop-in), the build with
    the Fortran's own math (glibc exp/log/pow, CALERF erfc) and the build with the kernel's math
    routines.  Returns (cpu_baseline, parity)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    n = s["ncol"]
    parity, base = {"workload": "259,200 columns (720 x 360) x 30 levels, seed 0, ~40 % convecting",
                    "column_error": "max_k |gpu - oracle| / max_k |oracle| per output field"}, None
    try:
        for name in ("glibc", "fortran", "portable"):
            oracle.set_variant(name)
            oracle.init_default()
            t0 = time.perf_counter()
            ref = oracle.compute(s, nthreads=cores, diag=True)
            sec = time.perf_counter() - t0
            if name == "glibc":
                base = {"value": n / sec, "unit": "columns/s", "cores": cores, "kind": "port",
                        "sample": "one pass over the %d-column grid (%.1f s); the 1,048,576-column "
                                  "workload has the same column distribution" % (n, sec)}
            worst, per = _column_errors(gpu_out, ref)
            trig = float(np.mean((gpu_out["cush"] != -1.0) == (ref["cush"] != -1.0)))
            parity[name] = {
                "columns_within_1e-11_all_outputs": float(np.mean(worst <= 1e-11)),
                "columns_bit_identical": float(np.mean(worst == 0.0)),
                "trigger_agree": trig, "cloud_base_agree": float(np.mean(gpu_out["cnb"] == ref["cnb"])),
                "cloud_top_agree": float(np.mean(gpu_out["cnt"] == ref["cnt"])),
                "level_indices_agree": float(np.mean(np.all(gpu_out["diag_int"][2:] == ref["diag_int"][2:], axis=0))),
                "worst_fields_within_1e-11": dict(sorted(per.items(), key=lambda kv: kv[1])[:3])}
            del ref
    finally:
        oracle.set_variant("glibc")
    parity["builds"] = {"glibc": "exp/log/pow/erfc from glibc; pinned bit for bit to the reference's "
                                 "C++ drop-in (bxcompute_uwshcu_inv.cpp) built for the host",
                        "fortran": "glibc exp/log/pow and CAM's CALERF erfc: the functions a Fortran "
                                   "build of uwshcu.F90 calls",
                        "portable": "the kernel's own math routines (correctly rounded exp/log/pow, "
                                    "CALERF erfc): expected bit for bit"}
    return base, parity


def column_quantities_dev(case):
    """Column heating, moistening and precipitation and the decisions of the last call, on the
    device (errstats.py's definitions)."""
    o, dp0 = case.out, case.inp["dp0"]
    return {"heating": (o["sten"] * dp0).sum(0) / G, "moistening": (o["qvten"] * dp0).sum(0) / G,
            "precipitation": o["precip"].clone(), "cnt": o["cnt"].clone(), "cnb": o["cnb"].clone(),
            "trigger": o["cush"] != -1.0}


def precision_leg(uw, case, stream, steps, warmup, fp64_ms, mode):
    """A reduced-precision mode (uw.PREC_MIXED or uw.PREC_FAST) on the columns of `case`, whose
    outputs hold the FP64 path's: speed and the error of column heating, moistening and
    precipitation against FP64.  Every device operation runs on `stream`, in order.  Leaves the
    FP64 outputs in `case` again."""
    import torch

    def step():
        case.out["cush"].copy_(case.cush0, non_blocking=True)
        rc = case.launch(stream=stream)
        if rc != 0:
            raise RuntimeError("precision %d: %d %s" % (mode, rc, uw.last_cuda_error()))

    with torch.cuda.stream(stream):
        ref = column_quantities_dev(case)
        assert uw.set_precision(mode) == 0
        try:
            for _ in range(warmup):
                step()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            q = column_quantities_dev(case)
        finally:
            assert uw.set_precision(uw.PREC_FP64) == 0
            step()                       # the FP64 outputs again, after q is taken
        stream.synchronize()
        ms = e0.elapsed_time(e1) / steps
        err, err_kept = {}, {}
        # the columns whose trigger, cloud-base and cloud-top decisions are the FP64 path's
        kept = (q["trigger"] == ref["trigger"]) & (q["cnb"] == ref["cnb"]) & (q["cnt"] == ref["cnt"])
        for k in ("heating", "moistening", "precipitation"):
            a, b = q[k].double(), ref[k].double()
            err[k] = float(torch.sqrt(torch.mean((a - b) ** 2)) / torch.sqrt(torch.mean(b ** 2)))
            err_kept[k] = float(torch.sqrt(torch.mean((a[kept] - b[kept]) ** 2)) / torch.sqrt(torch.mean(b[kept] ** 2)))
        import errstats
        dist = errstats.distribution({k: q[k].double().cpu().numpy() for k in ("heating", "moistening", "precipitation")},
                                     {k: ref[k].double().cpu().numpy() for k in ("heating", "moistening", "precipitation")},
                                     (kept & ref["trigger"]).cpu().numpy())
        flips = {"trigger": int((q["trigger"] != ref["trigger"]).sum()),
                 "cloud_base": int((q["cnb"] != ref["cnb"]).sum()),
                 "cloud_top": int((q["cnt"] != ref["cnt"]).sum()),
                 "convecting_columns": int(ref["trigger"].sum())}
        same = float(kept.double().mean())
    n = case.n
    return {"value": n / (ms * 1e-3), "unit": "columns/s", "ms_per_step": ms,
            "speedup_vs_fp64": fp64_ms / ms, "column_rel_rms_vs_fp64": err,
            "column_rel_rms_vs_fp64_same_decisions": err_kept, "columns_with_same_decisions": same,
            "column_error_distribution": dist,
            "flips": flips, "targets": "mixed precision: >= 2x the FP64 path at <= 1e-4 relative RMS"}


def depth_order_leg(uw, case, stream, nsteps=4, dt=1800.0, cp=1004.64):
    """uwshcu_set_depth_order on a state that evolves: each step applies the last step's tendencies
    for dt (temperature, dry static energy, water species, wind) and computes the columns once in
    trigger order and once ordered by the previous step's keys (the same bits).  Changes the inputs of
    `case`; run last on it."""
    import torch
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    t_off, t_on = [], []
    with torch.cuda.stream(stream):
        for step in range(nsteps + 1):
            for on, acc in ((False, t_off), (True, t_on)):
                assert uw.set_depth_order(on) == 0
                case.out["cush"].copy_(case.cush0, non_blocking=True)
                e0, e1 = ev()
                e0.record(stream)
                rc = case.launch(stream=stream)
                e1.record(stream)
                if rc != 0:
                    raise RuntimeError("depth order: %d %s" % (rc, uw.last_cuda_error()))
                e1.synchronize()
                if step > 0:   # step 0 only writes the first keys
                    acc.append(e0.elapsed_time(e1))
            o, i = case.out, case.inp
            i["t0"].add_(dt * o["sten"] / cp)
            i["s0"].add_(dt * o["sten"])
            for a, b in (("qv0", "qvten"), ("ql0", "qlten"), ("qi0", "qiten")):
                i[a].add_(dt * o[b]).clamp_(min=0.0)
            i["u0"].add_(dt * o["uten"])
            i["v0"].add_(dt * o["vten"])
            case.cush0.copy_(o["cush"])
    stream.synchronize()
    assert uw.set_depth_order(False) == 0
    return {"steps": nsteps, "ms_trigger_order": t_off, "ms_depth_order": t_on,
            "time_saved": 1.0 - sum(t_on) / sum(t_off),
            "workload": "the benchmark columns, advanced by their own tendencies every step (dt = 1800 s)"}


def zwshcu_leg(uw, case, s, stream, steps, warmup):
    """compute_zwshcu (zwshcu.F90), the CAS-ESM variant, on the columns of `case` with a synthetic
    large-scale pressure velocity (soundings.make_omega): FP64 columns/s and the trigger fraction.
    Leaves the compute_uwshcu outputs in `case` again."""
    import torch
    import soundings
    om = torch.from_numpy(soundings.make_omega(s, seed=1)).cuda()

    def step(omega):
        case.out["cush"].copy_(case.cush0, non_blocking=True)
        rc = case.launch(stream=stream, omega=omega)
        if rc != 0:
            raise RuntimeError("compute_zwshcu_device: %d %s" % (rc, uw.last_cuda_error()))

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step(om)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(om)
        e1.record(stream)
        trig = float((case.out["cush"] != -1.0).double().mean())
        step(None)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"value": case.n / (ms * 1e-3), "unit": "columns/s", "ms_per_step": ms, "steps": steps,
            "trigger_fraction": trig,
            "workload": "the same columns with omega = omega0 sin(pi (ps - p) / (ps - 10 kPa)), "
                        "omega0 ~ N(-0.05, 0.3) Pa/s (soundings.make_omega, seed 1); the variant's "
                        "default options (large-scale forcing on)"}


def adjoint_leg(uw, steps, warmup, n=65_536):
    """The adjoint model against the forward pass on n x 30 columns (random cotangents on every
    differentiable output): cost ratio and tape size."""
    import torch
    import soundings
    s = soundings.make_soundings(n, PVER, seed=301, rh_pbl=RH_PBL)
    case = uw.DeviceCase(s)
    g = torch.Generator(device="cpu").manual_seed(11)
    cot = {k: torch.randn(v.shape, generator=g, dtype=torch.float64).cuda() for k, v in case.out.items()
           if k in uw.ADJ_OUTPUTS}
    stream = torch.cuda.Stream()

    def timed(fn, k):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                case.reset_cush()
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                case.reset_cush()
                fn()
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    def adjoint(defect=False):
        rc, _ = uw.adjoint_launch(case, cot, stream=stream, defect=defect)
        if rc != 0:
            raise RuntimeError("adjoint: %d %s" % (rc, uw.last_cuda_error()))

    fwd = timed(lambda: case.launch(stream=stream), steps)
    ka = max(1, min(steps, 5))
    adj = timed(adjoint, ka)
    rows = uw.adjoint_last_records()
    checked = timed(lambda: adjoint(True), ka)
    conv = int((case.out["cush"] != -1.0).sum())
    uw.adjoint_release()
    del case, cot
    torch.cuda.empty_cache()
    return {"value": adj / fwd, "unit": "adjoint ms / forward ms", "forward_ms": fwd,
            "adjoint_ms": adj, "checked_adjoint_ms": checked, "steps": ka, "workload": "%s columns x 30 levels (seed 301)" % f"{n:,}",
            "convecting_columns": conv, "tape_rows_per_warp": rows,
            "tape_bytes_per_convecting_column": rows * 32,
            "target": "adjoint: <= 4x the forward"}


# Batched uneven workload: 4 members of 262,144 columns (1,048,576 in all) with 30, 35, 51 and 30
# levels; the PBL relative-humidity draws give trigger fractions of about 5, 25, 45 and 60 %.
BATCH_MEMBERS = ((262_144, 30, (0.55, 0.757)), (262_144, 35, (0.625, 0.86)),
                 (262_144, 51, (0.662, 0.912)), (262_144, 30, (0.75, 0.97)))


def batched_leg(uw, steps, warmup):
    """The batched uneven workload in FP64 (4 members of 262,144 columns, 30/35/51/30 levels, ~5/25/
    45/60 % convecting): one plan, autotuned launch shape, replays of its captured CUDA graph; every
    device operation on one stream."""
    import torch
    import soundings
    cases = []
    for j, (n, pver, rh) in enumerate(BATCH_MEMBERS):
        s = soundings.make_soundings(n, pver, seed=100 + j, rh_pbl=rh)
        cases.append(uw.DeviceCase(s))
        del s
    stream = torch.cuda.Stream()
    plan = uw.BatchPlan(cases)
    try:
        tuned = plan.autotune(stream)
        assert plan.capture(stream) == 0, uw.last_cuda_error()

        def step():
            for c in cases:
                c.out["cush"].copy_(c.cush0, non_blocking=True)
            rc = plan.run(stream)
            if rc != 0:
                raise RuntimeError("uwshcu_batch_run: %d %s" % (rc, uw.last_cuda_error()))

        with torch.cuda.stream(stream):
            for _ in range(warmup):
                step()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            trig = [float((c.out["cush"] != -1.0).double().mean()) for c in cases]
        e1.synchronize()
        st = plan.status(stream)
    finally:
        plan.close()
    ms = e0.elapsed_time(e1) / steps
    ncol = sum(m[0] for m in BATCH_MEMBERS)
    del cases
    torch.cuda.empty_cache()
    return {"value": ncol / (ms * 1e-3), "unit": "columns/s", "ms_per_step": ms, "steps": steps,
            "workload": "4 members x 262,144 columns, pver 30/35/51/30, FP64, sorted schedule",
            "trigger_fraction": trig, "status": st,
            "launch": "CUDA graph replay; autotuned block %d, %d column(s) per lane per task" % (tuned[0], tuned[2])}


def run_batched(args):
    """One step = one replay of the captured batch plan over all members, inputs resident in HBM:
    per level class a trigger launch and the worklist pass (sorted schedule, the default: a
    persistent first worklist launch, the per-member sort of the handed-off columns, a persistent
    resume launch; --schedule two-phase: one persistent worklist launch)."""
    import torch
    import soundings
    import uwshcu_b200 as uw

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    assert uw.init_default() == 0
    sorted_plan = args.schedule == "sorted"
    assert uw.set_schedule(uw.SCHED_SORTED if sorted_plan else uw.SCHED_TWO_PHASE) == 0
    cases = []
    for j, (n, pver, rh) in enumerate(BATCH_MEMBERS):
        s = soundings.make_soundings(n, pver, seed=100 + 10 * rank + j, rh_pbl=rh)
        cases.append(uw.DeviceCase(s))
        del s
    stream = torch.cuda.Stream()
    plan = uw.BatchPlan(cases)
    tuned = plan.autotune(stream)
    assert plan.capture(stream) == 0, uw.last_cuda_error()

    def step():
        for c in cases:
            c.out["cush"].copy_(c.cush0, non_blocking=True)
        rc = plan.run(stream)
        if rc != 0:
            raise RuntimeError("uwshcu_batch_run: %d %s" % (rc, uw.last_cuda_error()))

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    st = plan.status(stream)
    trig = [float((c.out["cush"] != -1.0).float().mean().item()) for c in cases]
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    ncol = sum(m[0] for m in BATCH_MEMBERS)
    nclass = len({(m[1] + 1) <= 32 for m in BATCH_MEMBERS})
    names = ("batched_member_30L_5pct", "batched_member_35L_25pct", "batched_member_51L_45pct",
             "batched_member_30L_60pct")
    ops = [algorithmic_ops(nm, m[0], t) for nm, m, t in zip(names, BATCH_MEMBERS, trig)]
    fp64_alg = None
    if all(o is not None for o in ops) and clk is not None and clk.summary().get("sm_mhz"):
        pk = 2 * FP64_DFMA_PER_CYCLE * clk.summary()["sm_mhz"] * 1e6 / 1e12
        ach = sum(ops) / (ms * 1e-3) / 1e12
        fp64_alg = {"ops_per_step": sum(ops), "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                    "frac": ach / pk, "t_roof_ms": sum(ops) / (pk * 1e12) * 1e3}
    # the same members in the reduced-precision modes, side by side with FP64: speed and error
    G = 9.80616

    def col_quantities():
        return [((c.out["sten"] * c.inp["dp0"]).sum(0) / G, (c.out["qvten"] * c.inp["dp0"]).sum(0) / G,
                 c.out["precip"].clone(), c.out["cnt"].clone(), (c.out["cush"] != -1.0)) for c in cases]

    ref_q = col_quantities()
    plan.close()
    others = {}
    for name, mode in (("fast", uw.PREC_FAST), ("mixed", uw.PREC_MIXED)):
        assert uw.set_precision(mode) == 0
        p2 = uw.BatchPlan(cases)
        tuned2 = p2.autotune(stream)
        assert p2.capture(stream) == 0, uw.last_cuda_error()
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                for c in cases:
                    c.out["cush"].copy_(c.cush0, non_blocking=True)
                assert p2.run(stream) == 0
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                for c in cases:
                    c.out["cush"].copy_(c.cush0, non_blocking=True)
                assert p2.run(stream) == 0
            e1.record(stream)
        e1.synchronize()
        ms2 = e0.elapsed_time(e1) / args.steps
        q = col_quantities()
        err = {}
        for j, nm in enumerate(("heating", "moistening", "precipitation")):
            a = torch.cat([x[j] for x in q]).double()
            b = torch.cat([x[j] for x in ref_q]).double()
            err[nm] = float(torch.sqrt(torch.mean((a - b) ** 2)) / torch.sqrt(torch.mean(b ** 2)))
        flips_top = int(sum(int((x[3] != y[3]).sum()) for x, y in zip(q, ref_q)))
        flips_trig = int(sum(int((x[4] != y[4]).sum()) for x, y in zip(q, ref_q)))
        others[name] = {"value": ncol / (ms2 * 1e-3), "ms_per_step": ms2, "speedup_vs_fp64": ms / ms2,
                        "column_rel_rms_vs_fp64": err, "cloud_top_flips": flips_top,
                        "trigger_flips": flips_trig, "autotuned": list(tuned2)}
        p2.close()
    assert uw.set_precision(uw.PREC_FP64) == 0
    line = {
        "metric": "columns/s (batched uneven compute_uwshcu, FP64, 4 members x 262,144 columns)",
        "value": ncol / (ms * 1e-3), "unit": "columns/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded soundings, seeds 100..103)",
        "config": {"workload": "batched uneven launch: 4 members x 262,144 columns, pver 30/35/51/30, "
                               "5 tracers, dt=1800 s", "pver": [m[1] for m in BATCH_MEMBERS],
                   "trigger_fraction": trig, "l2": "inputs larger than L2",
                   "launch": ("CUDA graph: per level class one trigger launch, a persistent first "
                              "worklist launch (4 blocks/SM) and a persistent resume launch (5 blocks/SM), "
                              "3 sort kernels per member; autotuned block %d, %d column(s) per lane per "
                              "task" % (tuned[0], tuned[2])
                              if sorted_plan else
                              "CUDA graph: per level class one trigger launch + one persistent worklist "
                              "launch; autotuned block %d, register cap %d blocks/SM, %d column(s) "
                              "per lane per task" % tuned),
                   "schedule": args.schedule},
        "gpu_launches": args.steps * ((3 * nclass + 3 * len(BATCH_MEMBERS)) if sorted_plan else 2 * nclass),
        "status": st,
        "roofline": {"fp64_algorithmic": fp64_alg},
        "precisions": others,
    }
    if clk is not None:
        line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def run_tangent(args):
    """Cost of the tangent-linear model against the forward pass: 65,536 columns x 30 levels, one
    direction in t0, qv0, tke and pblh and all four tuning parameters."""
    import torch
    import soundings
    import uwshcu_b200 as uw

    torch.cuda.set_device(0)
    assert uw.init_default() == 0
    n = 65_536
    s = soundings.make_soundings(n, PVER, seed=301, rh_pbl=RH_PBL)
    case = uw.DeviceCase(s)
    rng = np.random.default_rng(7)
    dirs = {k: torch.from_numpy(np.ascontiguousarray(s[k] * rng.uniform(-1e-3, 1e-3, s[k].shape))).cuda()
            for k in ("t0", "qv0", "tke", "pblh")}
    dparams = (1e-2, 1e-4, 1.4e-2, 7e-7)
    stream = torch.cuda.Stream()

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                case.reset_cush()
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                case.reset_cush()
                fn()
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / args.steps

    fwd = timed(lambda: case.launch(stream=stream))
    assert uw.set_schedule(uw.SCHED_SINGLE_PASS) == 0
    fwd1 = timed(lambda: case.launch(stream=stream))
    assert uw.set_schedule(uw.SCHED_DEFAULT) == 0
    tl = timed(lambda: uw.tangent_launch(case, dirs, dparams, stream=stream))
    line = {"metric": "tangent-linear cost / forward cost (compute_uwshcu, 65,536 x 30, FP64)",
            "value": tl / fwd, "unit": "ratio", "higher_is_better": False, "n_gpus": 1,
            "steps": args.steps, "warmup": max(args.warmup, 3), "dtype": "f64", "data": "synthetic",
            "config": {"workload": "65,536 columns x 30 levels, one direction in t0/qv0/tke/pblh and "
                                   "rpen/rle/rkm/criqc"},
            "forward_ms": fwd, "forward_single_pass_ms": fwd1, "tangent_ms": tl,
            "tangent_vs_single_pass": tl / fwd1,
            "memory": "tangent: 54 KB stack per thread (forward 27 KB), 26 extra output arrays"}
    print(json.dumps(line), flush=True)


def run_adjoint(args):
    """Cost of the adjoint model against the forward pass: 65,536 columns x 30 levels, cotangents on
    every differentiable output, gradients in t0, qv0, tke, pblh and the four tuning parameters."""
    import torch
    import soundings
    import uwshcu_b200 as uw

    torch.cuda.set_device(0)
    assert uw.init_default() == 0
    n = args.columns
    s = soundings.make_soundings(n, PVER, seed=301, rh_pbl=RH_PBL)
    case = uw.DeviceCase(s)
    g = torch.Generator(device="cpu").manual_seed(11)
    cot = {k: torch.randn(v.shape, generator=g, dtype=torch.float64).cuda() for k, v in case.out.items()
           if k in uw.ADJ_OUTPUTS}
    stream = torch.cuda.Stream()

    def timed(fn, steps):
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                case.reset_cush()
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                case.reset_cush()
                fn()
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def adjoint():
        rc, _ = uw.adjoint_launch(case, cot, stream=stream)
        assert rc == 0, (rc, uw.last_cuda_error())

    fwd = timed(lambda: case.launch(stream=stream), args.steps)
    adj = timed(adjoint, max(1, min(args.steps, 5)))
    line = {"metric": "adjoint cost / forward cost (compute_uwshcu, %s x 30, FP64)" % f"{n:,}",
            "value": adj / fwd, "unit": "ratio", "higher_is_better": False, "n_gpus": 1,
            "steps": max(1, min(args.steps, 5)), "warmup": max(args.warmup, 3), "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "%s columns x 30 levels, random cotangents on every differentiable "
                                   "output" % f"{n:,}"},
            "forward_ms": fwd, "adjoint_ms": adj, "tape_rows_per_warp": uw.adjoint_last_records()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncol", type=int, default=NCOL)
    ap.add_argument("--columns", type=int, default=65536,
                    help="columns of the tangent and adjoint cost configs (65,536 by default)")
    ap.add_argument("--cpu-sample", type=int, default=262144,
                    help="columns of the workload the reference arm computes per step")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision, adjoint and parity legs of the default run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--schedule", default="sorted", choices=["two-phase", "sorted", "single-pass"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fast", "mixed"],
                    help="fp64: bit-exact (default); fast: FP64 with the early-stopping conden; "
                         "mixed: FP32 bulk with FP64 islands")
    ap.add_argument("--config", default="fp64", choices=["fp64", "batched", "tangent", "adjoint"],
                    help="fp64: the 1,048,576-column workload (default); batched: 4 uneven members")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "tangent":
        return run_tangent(args)
    if args.config == "adjoint":
        return run_adjoint(args)

    import torch
    import soundings
    import uwshcu_b200 as uw

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    assert uw.init_default() == 0
    prec = {"fp64": uw.PREC_FP64, "fast": uw.PREC_FAST, "mixed": uw.PREC_MIXED}[args.precision]
    assert uw.set_precision(prec) == 0, "precision %s not available" % args.precision
    two_phase = args.schedule in ("two-phase", "sorted")
    sorted_pass = args.schedule == "sorted"
    assert uw.set_schedule({"two-phase": uw.SCHED_TWO_PHASE, "sorted": uw.SCHED_SORTED,
                            "single-pass": uw.SCHED_SINGLE_PASS}[args.schedule]) == 0
    n = args.ncol
    s = soundings.make_soundings(n, PVER, seed=shard_seed(rank), rh_pbl=RH_PBL)
    case = uw.DeviceCase(s)
    stream = torch.cuda.Stream()
    nbytes_in, nbytes_out = bytes_per_column()

    def step():
        case.out["cush"].copy_(case.cush0, non_blocking=True)
        rc = case.launch(stream=stream)
        if rc != 0:
            raise RuntimeError("uwshcu_compute_device: %d %s" % (rc, uw.last_cuda_error()))

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    stream.synchronize()
    st = case.status(stream)
    trig = float((case.out["cush"] != -1.0).float().mean().item())
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    uw.set_profiling(two_phase)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    phases = None
    if two_phase:
        calls, trig_ms, list_ms, ncand = uw.profile_read()
        uw.set_profiling(False)
        phases = {"trigger_ms": trig_ms / max(calls, 1), "worklist_ms": list_ms / max(calls, 1),
                  "worklist_columns": ncand, "calls": calls}
    ms = max_over_ranks(pg, ms, "cuda")
    value = job_throughput(world, n, ms * 1e-3)
    # the dominant kernel: the worklist launch of the two-phase schedule, else the single pass
    kernel_ms = phases["worklist_ms"] if phases else ms

    # end-to-end through compute_uwshcu_ with host arrays
    e2e = None
    if not args.no_e2e:
        keep = []

        def pinned(x):
            # a page-locked copy (the library then copies each level plane straight to the device)
            t = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
            keep.append(t)
            return t.numpy()

        def host_steps(sd, out):
            for _ in range(2):
                out["cush"][:] = sd["cush"]
                rc, _ = uw.compute_host(sd, out=out)
            if pg:
                pg.barrier()
            ksteps = max(1, min(args.steps, 5))
            t0 = time.perf_counter()
            for _ in range(ksteps):
                out["cush"][:] = sd["cush"]
                rc, _ = uw.compute_host(sd, out=out)
            sec = (time.perf_counter() - t0) / ksteps
            return max_over_ranks(pg, sec, "cuda"), rc

        sp = {k: pinned(v) if isinstance(v, np.ndarray) else v for k, v in s.items()}
        outp = {k: pinned(v) for k, v in uw.alloc_outputs(PVER, NCNST, n, s["cush"]).items()}
        sec, rc = host_steps(sp, outp)
        e2e = {"value": job_throughput(world, n, sec), "unit": "columns/s",
               "h2d_bytes_per_step": int(n * (nbytes_in + 8 * PVER)),
               "d2h_bytes_per_step": int(n * nbytes_out), "ms_per_step": sec * 1e3,
               "host_memory": "page-locked caller arrays (torch pin_memory)", "status": int(rc)}
        if world == 1:
            # pageable arrays too (one GPU only: eight ranks' extra host copies would not fit the
            # host's memory beside their page-locked ones)
            sec_pg, rc_pg = host_steps(s, uw.alloc_outputs(PVER, NCNST, n, s["cush"]))
            e2e["pageable"] = {"value": job_throughput(world, n, sec_pg), "ms_per_step": sec_pg * 1e3,
                               "status": int(rc_pg),
                               "host_memory": "pageable numpy arrays, packed through pinned staging"}
        del keep

    # column energy and water budgets of the last step (CAM's check_energy_chng thresholds)
    te_r, tw_r = case.budgets(stream=stream)
    budget = {"te_rer_max": float(np.max(np.abs(te_r))), "tw_rer_max": float(np.max(np.abs(tw_r))),
              "columns_over_cam_thresholds": int(np.sum((np.abs(te_r) > 1e-14) | (np.abs(tw_r) > 1e-10)))}
    err = None
    if prec != uw.PREC_FP64:
        import errstats
        out_r = case.outputs_numpy()
        assert uw.set_precision(uw.PREC_FP64) == 0
        case.reset_cush()
        assert case.launch(stream=stream) == 0
        stream.synchronize()
        rep = errstats.report(out_r, case.outputs_numpy(), s["dp0"])
        assert uw.set_precision(prec) == 0
        err = {"vs": "FP64 path (bit-identical to the FP64 oracle), same inputs",
               "column_rel_rms": {k: v["rel_rms"] for k, v in rep["column"].items()},
               "flips": rep["flips"],
               "field_rel_rms_max": max(v["rel_rms"] for v in rep["fields"].values())}

    extras = rank == 0 and world == 1 and not args.no_extras and prec == uw.PREC_FP64
    mixed = fast = adjoint = batched = zw = dord = None
    if extras:
        mixed = precision_leg(uw, case, stream, args.steps, max(args.warmup, 3), ms, uw.PREC_MIXED)
        fast = precision_leg(uw, case, stream, args.steps, max(args.warmup, 3), ms, uw.PREC_FAST)
        zw = zwshcu_leg(uw, case, s, stream, args.steps, max(args.warmup, 3))
        # last on these columns: it advances their state
        dord = depth_order_leg(uw, case, stream)
    if extras or (rank == 0 and world == 1 and not args.no_cpu_baseline):
        # free the large workload before the grid run, the adjoint buffer and the oracle
        del case
        torch.cuda.empty_cache()
        if extras:
            # the adjoint first: its tape buffer takes most of the free device memory
            adjoint = adjoint_leg(uw, args.steps, max(args.warmup, 3))
            batched = batched_leg(uw, args.steps, max(args.warmup, 3))
        grid_s, grid_out, grid_rc, grid_st = grid_case(uw)

    peak, peak_kind = peaks()
    # the FP64 pipe's throughput, measured here (a loop of independent fused multiply-adds)
    fp64_rc, fp64_meas = uw.fp64_peak()
    ncols_dom = phases["worklist_columns"] if phases else n
    fp64 = None
    fp64_alg = None
    # operation counts per convecting / other column of this column distribution (counted on the
    # 259,200-column grid of the same generator)
    ops = algorithmic_ops("fp64_259200x30", world * n, trig) if PVER == 30 else None
    pk_derived = (2 * FP64_DFMA_PER_CYCLE * clk.summary()["sm_mhz"] * 1e6 / 1e12
                  if clk is not None and clk.summary().get("sm_mhz") else None)
    if fp64_rc == 0 and fp64_meas > 0:
        pk, pk_kind = fp64_meas, "measured: uwshcu_fp64_peak (independent DFMA chains, two full waves)"
    else:
        pk, pk_kind = pk_derived, "derived: 2 x 9472 DFMA/cycle x median SM clock"
    if ops and pk:
        ach = ops / (ms * 1e-3) / 1e12
        fp64_alg = {"ops_per_step": ops, "achieved": ach, "peak": pk, "peak_kind": pk_kind,
                    "peak_derived": pk_derived, "unit": "TFLOP/s",
                    "frac": ach / pk, "t_roof_ms": ops / (pk * 1e12) * 1e3,
                    "what": "algorithmic FP64 operations of the whole step (oracle operation count "
                            "per convecting / other column x columns) / step time"}
    if phases and sorted_pass and prec == uw.PREC_FP64 and pk:
        ach = NCU_FP64_OPS_PER_LIST_COLUMN * ncols_dom / (kernel_ms * 1e-3) / 1e12
        fp64 = {"achieved": ach, "peak": pk, "peak_kind": pk_kind, "peak_derived": pk_derived,
                "unit": "TFLOP/s", "frac": ach / pk,
                "what": "executed FP64 ops (ncu count per worklist column) / live kernel time"}
    # algorithmic bytes of the dominant launch: the columns it processes x bytes per column
    alg = ncols_dom * (nbytes_in + nbytes_out)
    achieved = alg / (kernel_ms * 1e-3) / 1e9
    line = {
        "metric": "columns/s (compute_uwshcu, %s, %s x 30 levels)" % (
            "FP64" if prec == uw.PREC_FP64 else args.precision, f"{n:,}"),
        "value": value, "unit": "columns/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec == uw.PREC_MIXED else "f64",
        "data": "synthetic (seeded soundings, PCG64 seed 1+rank)",
        "config": {"workload": "compute_uwshcu %s columns x 30 levels, 5 tracers, dt=1800 s, ~40%% "
                               "convecting" % f"{n:,}", "ncol_per_gpu": n, "pver": PVER,
                   "ncnst": NCNST, "trigger_fraction": trig,
                   "l2": "inputs (%.1f GB) larger than L2" % (n * nbytes_in / 1e9),
                   "parallelism": "column shards, %d rank(s), no collective" % world},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (NCU_DRAM_BYTES_PER_LIST_COLUMN * ncols_dom)
                                if (phases and sorted_pass and prec == uw.PREC_FP64) else None,
                     "peak_kind": peak_kind,
                     "kernel": "uwshcu_%s_kernel<32,5,%s>" % ({"fp64": "fp64", "fast": "fast", "mixed": "mixed"}[args.precision],
                                                              ("UW_MODE_LIST1 + UW_MODE_RESUME" if sorted_pass else "UW_MODE_LIST")
                                                              if phases else "UW_MODE_ALL"),
                     "kernel_ms": kernel_ms, "columns_per_launch": ncols_dom,
                     "fp64": fp64, "fp64_algorithmic": fp64_alg,
                     "note": "branchy FP64 column physics: neither HBM nor the FP64 pipe is the bound "
                             "(issue latency is); algorithmic bytes = %d B/column; traffic = ncu DRAM "
                             "bytes per worklist column x columns (the per-thread stack of level "
                             "profiles spills out of L1/L2)" % (nbytes_in + nbytes_out)},
        "schedule": args.schedule,
        "precision": args.precision,
        "phases": phases,
        # trigger + worklist; sorted: trigger, first worklist launch, 3 sort kernels, second launch
        "gpu_launches": args.steps * ((6 if sorted_pass else 2) if two_phase else 1),
        "status": st,
    }
    if e2e is not None:
        line["e2e"] = e2e
    if err is not None:
        line["error_vs_fp64"] = err
    line["budgets"] = budget
    if clk is not None:
        line["clocks"] = clk.summary()
    if mixed is not None:
        line["mixed"] = mixed
    if fast is not None:
        line["fast"] = fast
    if adjoint is not None:
        line["adjoint"] = adjoint
    if batched is not None:
        line["batched"] = batched
    if zw is not None:
        line["zwshcu"] = zw
    if dord is not None:
        line["depth_order"] = dord
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, parity = cpu_baseline_leg(grid_s, grid_out)
        parity["gpu_status"] = [int(grid_rc), int(grid_st)]
        line["cpu_baseline"] = base
        line["parity"] = parity
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
