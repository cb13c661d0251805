"""uwshcu_fp64_peak: the measured FP64 throughput that the benchmark divides by.  A B200 has 148
SMs of 64 FP64 lanes (2 flops per fused multiply-add) at up to 1.965 GHz, 37.2 TFLOP/s; the
measured figure lies within a few per cent below that at full clock."""
import pytest


@pytest.mark.gpu
def test_fp64_peak_is_measured(uw, cuda):
    rc, tf = uw.fp64_peak()
    assert rc == 0, uw.last_cuda_error()
    print("FP64 peak: %.2f TFLOP/s" % tf)
    assert 10.0 < tf < 45.0, tf
