"""FP64 CUDA path against the CPU oracle, through the C ABI.

Bar (per output field): the norm-wise relative error of a column, max_k |gpu-oracle| / max_k
|oracle|, is at most 1e-11 on at least 99.99 % of the columns, and the trigger, cloud-base (cnb) and
cloud-top (cnt) decisions agree on at least 99.99 % of the columns.  The reference here is the
oracle build with the same exp/log/pow/erfc routines as the kernel (uw_math.h); both sides keep the
Fortran operation order without FMA contraction, so the expected result is bit for bit.  The
comparison with the glibc build (pinned to the reference) is test_gpu_vs_glibc_oracle.
"""
import numpy as np
import pytest

import soundings
from util import FIELDS, compare, conditioned_compare, decisions

pytestmark = pytest.mark.gpu

TOL = 1e-11
FRAC = 0.9999


def _check(out, ref, n, tol=TOL, frac=FRAC, fields=FIELDS):
    res, worst = compare(out, ref, tol=tol, fields=fields, ncol=n)
    bad = {f: v for f, v in res.items() if v[0] < frac}
    assert not bad, "fields below %.4f within %g: %s" % (frac, tol, bad)
    tg, cb, ct = decisions({k: out[k][..., :n] for k in ("cush", "cnb", "cnt")})
    tr, rb, rt = decisions({k: ref[k][..., :n] for k in ("cush", "cnb", "cnt")})
    for name, a, b in (("trigger", tg, tr), ("cloud base", cb, rb), ("cloud top", ct, rt)):
        agree = float(np.mean(a == b))
        assert agree >= frac, "%s decisions agree on %.5f of columns" % (name, agree)
    return worst


@pytest.mark.parametrize("ncol,pver,seed", [(4096, 30, 11), (2000, 35, 12), (1500, 51, 13)])
def test_host_entry_matches_oracle(uw, oracle_pm, cuda, ncol, pver, seed):
    s = soundings.make_soundings(ncol, pver, seed=seed)
    ref = oracle_pm.compute(s, nthreads=0, diag=False)
    rc, out = uw.compute_host(s)
    assert rc == ref["status"], (rc, ref["status"], uw.last_cuda_error())
    _check(out, ref, ncol)


def test_device_entry_and_diagnostics(uw, oracle_pm, cuda):
    s = soundings.make_soundings(3000, 30, seed=21)
    ref = oracle_pm.compute(s, diag=True)
    case = uw.DeviceCase(s, diag=True)
    assert case.launch() == 0
    assert case.status() == ref["status"]
    out = case.outputs_numpy()
    _check(out, ref, s["ncol"])
    # level indices of the scheme's decisions (kinv, klcl, klfc, krel, kbup, kpen) and exit flags
    agree = np.mean(np.all(out["diag_int"] == ref["diag_int"], axis=0))
    assert agree >= FRAC, agree


def test_inv_entries_match_oracle(uw, oracle_pm, cuda):
    s = soundings.make_soundings(2048, 30, seed=31)
    si = soundings.to_inv(s)
    ref = oracle_pm.compute(si, inv=True)
    for entry in ("compute_uwshcu_inv_", "bxcompute_uwshcu_inv_"):
        rc, out = uw.compute_host(si, entry=entry)
        assert rc == ref["status"], entry
        _check(out, ref, s["ncol"])


def test_leading_dimension_larger_than_iend(uw, oracle_pm, cuda):
    """mix = pcols > iend = ncol: the reference drop-in indexes k*iend+i and breaks here
    (bxcompute_uwshcu_inv.cpp:6505-6540); the ABI must honour mix."""
    s = soundings.make_soundings(1024, 30, seed=41)
    iend = 700
    ref = oracle_pm.compute({**_subset(s, iend)}, diag=False)
    rc, out = uw.compute_host(s, iend=iend)
    assert rc == ref["status"]
    _check({k: v[..., :iend] for k, v in out.items()}, ref, iend)
    # columns past iend are not touched
    assert np.all(out["umf"][:, iend:] == 0.0)


def _subset(s, n):
    out = dict(s)
    for k, v in s.items():
        if isinstance(v, np.ndarray) and v.shape[-1] == s["ncol"]:
            out[k] = np.ascontiguousarray(v[..., :n])
    out["ncol"] = n
    return out


def test_repeat_calls_are_deterministic(uw, cuda):
    s = soundings.make_soundings(1024, 30, seed=51)
    rc1, o1 = uw.compute_host(s)
    rc2, o2 = uw.compute_host(s)
    assert rc1 == rc2 == 0
    for f in FIELDS:
        assert np.array_equal(o1[f], o2[f]), f


def test_schedules_agree_bit_for_bit(uw, cuda):
    """The single-pass, the two-phase (trigger pass + worklist) and the sorted (worklist split at the
    iteration-2 CIN decision) schedules compute the same column code on the same inputs."""
    s = soundings.make_soundings(5000, 30, seed=61)
    outs = []
    try:
        for sched in (uw.SCHED_SINGLE_PASS, uw.SCHED_TWO_PHASE, uw.SCHED_SORTED):
            assert uw.set_schedule(sched) == 0
            rc, o = uw.compute_host(s)
            assert rc == 0
            outs.append(o)
    finally:
        uw.set_schedule(uw.SCHED_DEFAULT)
    for f in FIELDS:
        assert np.array_equal(outs[0][f], outs[1][f]), f


def test_gpu_vs_glibc_oracle(uw, oracle, cuda):
    """Against the build pinned to the reference: identical decisions and level indices, values
    within the conditioning bound of two ulp-accurate libms (see test_oracle_variants.py)."""
    s = soundings.make_soundings(6000, 30, seed=71)
    ref = oracle.compute(s, diag=True)
    case = uw.DeviceCase(s, diag=True)
    assert case.launch() == 0 and case.status() == ref["status"]
    out = case.outputs_numpy()
    assert np.mean(np.all(out["diag_int"][2:] == ref["diag_int"][2:], axis=0)) >= FRAC
    w = conditioned_compare(out, ref)
    assert np.mean(w <= 1e-6) >= 0.999


def test_math_routines_are_bit_identical_on_host_and_device(uw, oracle, cuda):
    rng = np.random.default_rng(5)
    cases = [(0, rng.uniform(-700, 700, 200000), None), (0, rng.uniform(-1, 1, 200000), None),
             (1, np.exp(rng.uniform(-700, 700, 200000)), None),
             (2, rng.uniform(0.01, 2.0, 200000), rng.uniform(-4, 4, 200000)),
             (3, rng.uniform(-3, 27, 200000), None)]
    for fn, x, y in cases:
        dev = uw.eval_math_device(fn, x, y)
        host = oracle.uwmath(fn, x, y)
        assert np.array_equal(dev.view(np.int64), host.view(np.int64)), fn


@pytest.mark.gpu
def test_pipelined_host_entries_match_one_chunk(uw, cuda):
    """Host-array calls split into column chunks over several streams give the same bits as one
    chunk, for both level orders and with mix > iend."""
    s = soundings.make_soundings(5000, 30, seed=61)
    try:
        for entry in ("compute_uwshcu_", "compute_uwshcu_inv_"):
            si = s if entry == "compute_uwshcu_" else soundings.to_inv(s)
            assert uw.set_pipeline(0, 1) == 0
            rc0, o0 = uw.compute_host(si, entry=entry, iend=4700)
            for chunk, streams in ((1024, 3), (777, 2), (4096, 4)):
                assert uw.set_pipeline(chunk, streams) == 0
                rc, o = uw.compute_host(si, entry=entry, iend=4700)
                assert rc == rc0
                bad = [k for k in o0 if not np.array_equal(o[k], o0[k])]
                assert not bad, (entry, chunk, streams, bad)
    finally:
        assert uw.set_pipeline(-1, 0) == 0


@pytest.mark.gpu
def test_auto_pipeline_with_ramped_chunks_matches_one_chunk(uw, cuda):
    """The default pipeline shape at 400,000 columns: chunks of 32,768, 32,768, 5 x 50,176, 18,048,
    32,768 and 32,768 columns over 2 streams; the same bits as one chunk."""
    s = soundings.make_soundings(400_000, 30, seed=62)
    try:
        assert uw.set_pipeline(0, 1) == 0
        rc0, o0 = uw.compute_host(s)
        assert uw.set_pipeline(-1, 0) == 0
        rc, o = uw.compute_host(s)
        assert rc == rc0 == 0
        bad = [k for k in o0 if not np.array_equal(o[k], o0[k])]
        assert not bad, bad
    finally:
        assert uw.set_pipeline(-1, 0) == 0


@pytest.mark.gpu
def test_tuning_parameters_match_oracle(uw, oracle_pm, cuda):
    """uwshcu_set_params (rpen, rle, rkm, criqc) against the oracle with the same values."""
    s = soundings.make_soundings(2048, 30, seed=81)
    try:
        assert uw.set_params(12.0, 0.12, 15.0, 0.6e-3) == 0
        assert oracle_pm.set_params(12.0, 0.12, 15.0, 0.6e-3) == 0
        ref = oracle_pm.compute(s, diag=False)
        rc, out = uw.compute_host(s)
        assert rc == ref["status"]
        _check(out, ref, 2048)
    finally:
        assert uw.init_default() == 0
        oracle_pm.init_default()


@pytest.mark.gpu
def test_page_locked_host_arrays_match_pageable(uw, cuda):
    """Page-locked caller arrays take the direct path (strided copies between them and the device,
    no staging): the same bits as pageable arrays, for both level orders, with mix > iend and with
    several chunks over several streams."""
    import torch

    keep = []

    def pinned(x):
        t = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
        keep.append(t)
        return t.numpy()

    s = soundings.make_soundings(5000, 30, seed=63)
    try:
        for entry in ("compute_uwshcu_", "compute_uwshcu_inv_"):
            si = s if entry == "compute_uwshcu_" else soundings.to_inv(s)
            sp = {k: pinned(v) if isinstance(v, np.ndarray) else v for k, v in si.items()}
            for chunk, streams in ((0, 1), (1024, 3)):
                assert uw.set_pipeline(chunk, streams) == 0
                rc0, o0 = uw.compute_host(si, entry=entry, iend=4700)
                outp = {k: pinned(v) for k, v in uw.alloc_outputs(30, 5, 5000, si["cush"]).items()}
                rc, o = uw.compute_host(sp, entry=entry, iend=4700, out=outp)
                assert rc == rc0 == 0
                bad = [k for k in o0 if not np.array_equal(o[k], o0[k])]
                assert not bad, (entry, chunk, streams, bad)
    finally:
        assert uw.set_pipeline(-1, 0) == 0
