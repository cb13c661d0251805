"""uwshcu_compute_device_noalloc: the device entry whose worklist is a fixed library array.

The GPU test calls the new entry point twice in a row through the C ABI and checks both results
against uwshcu_compute_device on the same inputs, with the parity tolerance of the other device
tests (column error <= 1e-11, identical cloud-top/base decisions), and that the second call leaves
the device's free memory unchanged.  The CPU test checks the size
limit, which is rejected before any CUDA call."""
import ctypes

import numpy as np
import pytest

import soundings
from util import conditioned_compare


def _noalloc_null_call(uw, iend):
    """Call the entry with every pointer NULL: only the argument checks run."""
    L = uw.lib()
    nulls = [None] * 47
    return L.uwshcu_compute_device_noalloc(ctypes.c_int(iend), ctypes.c_int(30), ctypes.c_int(iend),
                                           ctypes.c_int(5), ctypes.c_double(1800.0), ctypes.c_int(0),
                                           *nulls, None)


def test_noalloc_rejects_more_columns_than_its_array(uw):
    assert uw.init_default() == 0
    assert uw.set_precision(uw.PREC_FP64) == 0
    rc = _noalloc_null_call(uw, uw.NOALLOC_MAX_COLUMNS + 1)
    assert rc == uw.ERR_TOO_LARGE
    assert str(uw.NOALLOC_MAX_COLUMNS) in uw.last_cuda_error()
    # at the limit the size passes and the NULL pointers are what is rejected
    assert _noalloc_null_call(uw, uw.NOALLOC_MAX_COLUMNS) == uw.ERR_BAD_ARGS


@pytest.mark.gpu
def test_noalloc_matches_device_entry_on_two_calls(uw, cuda):
    import torch

    assert uw.init_default() == 0
    assert uw.set_precision(uw.PREC_FP64) == 0
    assert uw.set_schedule(uw.SCHED_TWO_PHASE) == 0
    assert uw.set_block(128) == 0
    s = soundings.make_soundings(4096, 30, seed=31)
    ref_case = uw.DeviceCase(s, diag=True)
    assert ref_case.launch() == 0, uw.last_cuda_error()
    assert ref_case.status() == 0
    ref = ref_case.outputs_numpy()

    case = uw.DeviceCase(s, diag=True, inputs=ref_case.inp)
    bits = torch.full((1,), 0x7FFF, dtype=torch.int32, device="cuda")
    for call in range(2):
        if call == 1:
            # the second call must overwrite every output of the first
            for t in case.out.values():
                t.fill_(-777.0)
            case.diag_int.fill_(-7)
            case.diag_real.fill_(-777.0)
            bits.fill_(0x7FFF)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        case.reset_cush()
        assert case.launch_noalloc(status_bits=bits) == 0, uw.last_cuda_error()
        torch.cuda.synchronize()
        if call == 1:
            # after the first call on the device, a call allocates no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        out = case.outputs_numpy()
        assert int(bits.item()) == 0, "endrun bits %#x on call %d" % (int(bits.item()), call)
        for f in ("cnt", "cnb"):
            assert np.array_equal(out[f], ref[f]), (call, f)
        assert np.array_equal(out["diag_int"], ref["diag_int"]), call
        err = conditioned_compare(out, ref, s["ncol"])
        assert float(np.max(err)) <= 1e-11, (call, float(np.max(err)))
        np.testing.assert_allclose(out["diag_real"], ref["diag_real"], rtol=1e-11, atol=0.0)
