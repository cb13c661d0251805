"""Batched uneven launches (uwshcu_batch_*): members with different level counts and trigger
fractions in one trigger launch and one persistent worklist launch per level class.  Every member's
outputs, per-level diagnostics included, must be the bits uwshcu_compute_member gives for that
member alone, for a plain run, a CUDA-graph replay and a run with the autotuned launch shape."""
import ctypes

import numpy as np
import pytest

import soundings

# (columns, levels, PBL relative-humidity draw): trigger fractions of about 5, 25, 45 and 60 %
MEMBERS = ((2048, 30, (0.55, 0.757)), (1536, 35, (0.625, 0.86)), (1024, 51, (0.662, 0.912)),
           (1800, 30, (0.75, 0.97)))


def _cases(uw):
    ref, bat = [], []
    for j, (n, pver, rh) in enumerate(MEMBERS):
        s = soundings.make_soundings(n, pver, seed=40 + j, rh_pbl=rh)
        r = uw.DeviceCase(s, diag=True)
        ref.append(r)
        bat.append(uw.DeviceCase(s, diag=True, inputs=r.inp))
    return ref, bat


def _same(a, b):
    return [k for k in a if not np.array_equal(a[k], b[k])]


def _poison(case):
    for t in case.out.values():
        t.fill_(-777.0)
    case.diag_int.fill_(-7)
    case.diag_real.fill_(-777.0)
    case.diag_level.fill_(-777.0)
    case.reset_cush()


@pytest.mark.gpu
@pytest.mark.parametrize("sched", ["sorted", "two_phase"])
@pytest.mark.parametrize("prec", ["fp64", "fast", "mixed"])
def test_batch_matches_single_member_calls(uw, cuda, prec, sched):
    """In every precision mode and both worklist schedules (a plan takes the schedule in force when
    it is created: sorted plans hand each member's implicit-CIN columns to its own region and resume
    them in depth order): the reduced-precision conden iterations stop per lane, so a column's
    result does not depend on which columns share its warp and the batch reproduces the single calls."""
    import torch

    assert uw.init_default() == 0
    mode = {"fp64": uw.PREC_FP64, "fast": uw.PREC_FAST, "mixed": uw.PREC_MIXED}[prec]
    assert uw.set_precision(mode) == 0
    assert uw.set_schedule(uw.SCHED_SORTED if sched == "sorted" else uw.SCHED_TWO_PHASE) == 0
    ref, bat = _cases(uw)
    want = []
    for r in ref:
        assert r.launch_member() == 0, uw.last_cuda_error()
        assert r.status() == 0
        want.append(r.outputs_numpy())
    trig = [float(np.mean(w["cush"] != -1.0)) for w in want]
    assert trig[0] < trig[1] < trig[2] < trig[3], trig

    plan = uw.BatchPlan(bat)
    stream = torch.cuda.Stream()
    try:
        # plain run
        assert plan.run(stream) == 0, uw.last_cuda_error()
        assert plan.status(stream) == 0
        for j, b in enumerate(bat):
            assert not _same(b.outputs_numpy(), want[j]), (j, _same(b.outputs_numpy(), want[j]))
        # CUDA-graph replay, twice
        assert plan.capture(stream) == 0, uw.last_cuda_error()
        for _ in range(2):
            for b in bat:
                _poison(b)
            torch.cuda.synchronize()
            assert plan.run(stream) == 0, uw.last_cuda_error()
            assert plan.status(stream) == 0
            for j, b in enumerate(bat):
                assert not _same(b.outputs_numpy(), want[j]), ("graph", j)
        # autotuned launch shape
        block, regcap_blocks, chunk = plan.autotune(stream)
        assert block in (64, 128) and regcap_blocks in ((3, 4, 6) if prec == "fp64" else (4,)) and chunk in (1, 2)
        for b in bat:
            _poison(b)
        torch.cuda.synchronize()
        assert plan.run(stream) == 0, uw.last_cuda_error()
        assert plan.status(stream) == 0
        for j, b in enumerate(bat):
            assert not _same(b.outputs_numpy(), want[j]), ("tuned", j)
    finally:
        plan.close()
        uw.set_precision(uw.PREC_FP64)
        uw.set_schedule(uw.SCHED_DEFAULT)


def test_batch_rejects_bad_plans_before_touching_the_device(uw):
    assert uw.init_default() == 0
    L = uw.lib()
    h = ctypes.c_void_p()
    assert L.uwshcu_batch_create(ctypes.c_int(0), None, ctypes.byref(h)) == uw.ERR_BAD_ARGS
    m = (uw.Member * (uw.MAX_MEMBERS + 1))()
    assert L.uwshcu_batch_create(ctypes.c_int(uw.MAX_MEMBERS + 1), m, ctypes.byref(h)) == uw.ERR_BAD_ARGS
    # members with valid sizes but NULL arrays
    for x in m:
        x.mix = x.iend = 64
        x.mkx = 30
        x.dt = 1800.0
    assert L.uwshcu_batch_create(ctypes.c_int(2), m, ctypes.byref(h)) == uw.ERR_BAD_ARGS
    m[0].mkx = 99
    assert L.uwshcu_batch_create(ctypes.c_int(1), m, ctypes.byref(h)) == uw.ERR_BAD_ARGS
    assert L.uwshcu_batch_run(None, None) == uw.ERR_BAD_ARGS
    assert L.uwshcu_batch_destroy(None) == uw.ERR_BAD_ARGS


# the batched uneven workload at full size: 4 members of 262,144 columns, 1,048,576 in all
MEMBERS_FULL = ((262_144, 30, (0.55, 0.757)), (262_144, 35, (0.625, 0.86)),
                (262_144, 51, (0.662, 0.912)), (262_144, 30, (0.75, 0.97)))


def _columns(s, idx):
    """The columns idx of a sounding dict (columns are independent)."""
    n = s["ncol"]
    out = {k: (np.ascontiguousarray(v[..., idx]) if isinstance(v, np.ndarray) and v.shape[-1] == n else v)
           for k, v in s.items()}
    out["ncol"] = len(idx)
    return out


@pytest.mark.gpu
def test_full_size_batch_members_match_the_oracle(uw, oracle, oracle_pm, cuda):
    """One FP64 run of the 1,048,576-column batch (30/35/51/30 levels, about 5/25/45/60 %
    convecting); 4,096 sampled columns of every member against the oracle: bit for bit against the
    build with the kernel's math routines, identical trigger, cloud-base and cloud-top decisions
    against the glibc build (pinned to the reference)."""
    import torch
    from util import FIELDS, decisions

    assert uw.init_default() == 0
    assert uw.set_precision(uw.PREC_FP64) == 0
    ss = [soundings.make_soundings(n, pver, seed=100 + j, rh_pbl=rh) for j, (n, pver, rh) in enumerate(MEMBERS_FULL)]
    cases = [uw.DeviceCase(s) for s in ss]
    plan = uw.BatchPlan(cases)
    stream = torch.cuda.Stream()
    try:
        assert plan.run(stream) == 0, uw.last_cuda_error()
        assert plan.status(stream) == 0
    finally:
        plan.close()
    rng = np.random.default_rng(0)
    for j, (s, case) in enumerate(zip(ss, cases)):
        idx = np.sort(rng.choice(s["ncol"], 4096, replace=False))
        it = torch.from_numpy(idx).to(case.out["cush"].device)
        out = {k: v.index_select(v.dim() - 1, it).cpu().numpy() for k, v in case.out.items()}
        sub = _columns(s, idx)
        pm = oracle_pm.compute(sub, diag=False)
        bad = [f for f in FIELDS if not np.array_equal(out[f], pm[f])]
        assert not bad, (j, bad)
        g = oracle.compute(sub, diag=False)
        for name, x, y in zip(("trigger", "cloud base", "cloud top"), decisions(out), decisions(g)):
            assert np.array_equal(x, y), (j, name)
    del cases
    torch.cuda.empty_cache()
