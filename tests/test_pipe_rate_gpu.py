"""Raw pipe-rate probes (GPU): the measured denominators of the bench's roofline fractions."""
from __future__ import annotations

import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_pipe_rates_are_measured(lib):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rate = C.c_double(0.0)
    assert lib.zynum_blas_gpu_measure_pipe_rate(0, C.byref(rate), stream) == 0, lib.zynum_blas_gpu_last_error()
    assert 15.0 < rate.value < 45.0, rate.value  # FP64 DMMA, TFLOP/s (nominal 37.2 at 1965 MHz)
    assert lib.zynum_blas_gpu_measure_pipe_rate(1, C.byref(rate), stream) == 0, lib.zynum_blas_gpu_last_error()
    assert 1000.0 < rate.value < 6000.0, rate.value  # INT8 tcgen05, TOP/s
    assert lib.zynum_blas_gpu_device_status(stream) == 0
    assert lib.zynum_blas_gpu_measure_pipe_rate(7, C.byref(rate), stream) == 1
