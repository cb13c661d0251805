"""Device-array calls on different streams may overlap on the GPU: the library keeps a worklist, a
hand-off region and an endrun word per caller stream, and uwshcu_device_status(stream) reports the
calls of that stream only."""
import numpy as np
import pytest

import soundings
from util import FIELDS

pytestmark = pytest.mark.gpu

WARN_NONFINITE = 4


def test_overlapping_calls_on_two_streams(uw, cuda):
    torch = cuda
    sa = soundings.make_soundings(20000, 30, seed=91)
    sb = soundings.make_soundings(30000, 30, seed=92)
    sb["t0"][5, 17] = np.nan          # one bad column: status 4 on b's stream only
    a, b = uw.DeviceCase(sa), uw.DeviceCase(sb)
    for sched in (uw.SCHED_SORTED, uw.SCHED_TWO_PHASE):
        assert uw.set_schedule(sched) == 0
        try:
            a.reset_cush()
            assert a.launch() == 0 and a.status() == 0
            ra = {k: v.clone() for k, v in a.out.items()}
            b.reset_cush()
            assert b.launch() == 0 and b.status() == WARN_NONFINITE
            rb = {k: v.clone() for k, v in b.out.items()}
            s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
            torch.cuda.synchronize()
            for _ in range(3):
                for case, st in ((a, s1), (b, s2)):
                    with torch.cuda.stream(st):
                        case.reset_cush()
                        for t in case.out.values():
                            if t is not case.out["cush"]:
                                t.fill_(-1.0e30)
                        assert case.launch(stream=st) == 0
            assert a.status(stream=s1) == 0
            assert b.status(stream=s2) == WARN_NONFINITE
            assert b.status(stream=s2) == 0          # read and reset
            for f in FIELDS:
                assert torch.equal(a.out[f], ra[f]), (sched, "a", f)
                assert torch.equal(b.out[f], rb[f]), (sched, "b", f)
        finally:
            assert uw.set_schedule(uw.SCHED_DEFAULT) == 0
