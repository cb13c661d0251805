"""uwshcu_set_depth_order: the worklist passes order their columns by the updraft each column had in
the previous call.  Which columns share a warp does not change a column's result, so every call
gives the bits of the trigger-ordered path: on repeated inputs, on a state that evolves by the
computed tendencies from call to call, for both worklist schedules, and for the host-array entry
(chunked, the keys kept per device)."""
import numpy as np
import pytest

import soundings

pytestmark = pytest.mark.gpu


def _advance(case, dt=1800.0, cp=1004.64):
    """The state a time step later under the computed tendencies alone."""
    import torch
    with torch.no_grad():
        o, i = case.out, case.inp
        i["t0"] += dt * o["sten"] / cp
        i["s0"] += dt * o["sten"]
        for a, b in (("qv0", "qvten"), ("ql0", "qlten"), ("qi0", "qiten")):
            i[a] += dt * o[b]
            i[a].clamp_(min=0.0)
        i["u0"] += dt * o["uten"]
        i["v0"] += dt * o["vten"]
        case.cush0.copy_(o["cush"])


@pytest.mark.parametrize("sched", ["sorted", "two_phase"])
def test_depth_order_gives_the_same_bits(uw, cuda, sched):
    import torch
    assert uw.init_default() == 0
    s = soundings.make_soundings(20000, 30, seed=611, rh_pbl=(0.675, 0.93))
    a, b = uw.DeviceCase(s, diag=True), uw.DeviceCase(s, diag=True)
    try:
        assert uw.set_schedule(uw.SCHED_SORTED if sched == "sorted" else uw.SCHED_TWO_PHASE) == 0
        for step in range(4):
            for case, on in ((a, False), (b, True)):
                assert uw.set_depth_order(on) == 0
                case.out["cush"].copy_(case.cush0)
                assert case.launch() == 0, uw.last_cuda_error()
                if step == 0 and on:   # the same inputs again: the keys of the call just made
                    case.out["cush"].copy_(case.cush0)
                    assert case.launch() == 0
            torch.cuda.synchronize()
            oa, ob = a.outputs_numpy(), b.outputs_numpy()
            bad = [k for k in oa if not np.array_equal(oa[k], ob[k])]
            assert not bad, (step, bad)
            assert torch.equal(a.diag_int, b.diag_int)
            if step < 3:
                _advance(a)
                _advance(b)
    finally:
        assert uw.set_depth_order(False) == 0
        assert uw.set_schedule(uw.SCHED_DEFAULT) == 0


def test_depth_order_host_entry(uw, cuda):
    """Host arrays in ramped chunks (400,000 columns): two calls with the order on, the second ordered
    by the keys of the first, give the bits of a call without it."""
    assert uw.init_default() == 0
    s = soundings.make_soundings(400_000, 30, seed=612)
    rc0, o0 = uw.compute_host(s)
    try:
        assert uw.set_depth_order(True) == 0
        for _ in range(2):
            rc, o = uw.compute_host(s)
            assert rc == rc0 == 0
            bad = [k for k in o0 if not np.array_equal(o[k], o0[k])]
            assert not bad, bad
    finally:
        assert uw.set_depth_order(False) == 0
