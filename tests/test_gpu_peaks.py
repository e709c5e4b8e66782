"""efem_fma_peak, the compute roof of the element residual kernels: plausible
and consistent figures on the device, and the argument check."""
import ctypes

import pytest

from efem_b200 import api

pytestmark = pytest.mark.gpu


def test_fma_peak_plausible():
    """FP64 and FP32 CUDA-core FMA throughput: positive, repeatable to 10 %,
    FP32 at least the FP64 figure, and neither above 2 flops per CUDA core per
    cycle at 2.5 GHz (a measurement far above that would not be timing the
    work)."""
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    bound = sms * 128 * 2 * 2.5  # GFLOP/s: 128 FP32 lanes per SM, 2.5 GHz
    f64 = [api.fma_peak(fp32=False) for _ in range(2)]
    f32 = api.fma_peak(fp32=True)
    assert all(0.0 < g < bound for g in f64)
    assert 0.0 < f32 < bound
    assert abs(f64[0] - f64[1]) <= 0.1 * max(f64)
    assert f32 >= 0.9 * max(f64)


def test_fma_peak_null_output():
    assert api.lib().efem_fma_peak(0, ctypes.POINTER(ctypes.c_double)()) == api.ERR_ARG
