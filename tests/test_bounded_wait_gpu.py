"""Bounded waits of the tensor-core product kernels (GPU).

Every mbarrier wait in the Ozaki product kernels gives up after a time limit:
the waiting role raises the CTA's abort flag (and its pair's), records the
site, the copies and MMAs already issued are drained, TMEM is freed and the
kernels that follow leave C alone.  The tests make one wait run out without
any GPU fault: fault injection kind 3 makes the next product kernel's MMA
issuer wait, with a 1 ms limit, on a barrier that nothing arrives on.  The
reference's rule is "failure before write" (gemm.zig:48-53, :1364-1383): the
call reports the failure and C keeps its values; the next call is correct.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
U64 = 2.0 ** -53
HOLD = 3


def _dev_call(L, torch, m, n, k, A, B, Cm, alpha=1.0, beta=0.5):
    stream = torch.cuda.current_stream().cuda_stream
    return L.zynum_blas_gpu_dgemm_device(b"N", b"N", m, n, k, alpha, A.data_ptr(), m, B.data_ptr(), k, beta,
                                         Cm.data_ptr(), m, stream)


@pytest.mark.parametrize("m", [128, 512], ids=["one-cta", "cta-pair"])
def test_wait_runs_out_reports_and_leaves_c(lib, oracle, m):
    import torch
    L = lib
    n, k = 384, 640
    g = torch.Generator(device="cuda").manual_seed(m)
    A = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1  # column-major m x k
    B = torch.rand((n, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1  # column-major k x n
    C0 = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    stream = torch.cuda.current_stream().cuda_stream
    old_method = L.zynum_blas_gpu_set_dgemm_method(1)
    old_scheme = L.zynum_blas_gpu_set_ozaki_scheme(2)
    try:
        assert L.zynum_blas_gpu_device_status(stream) == 0  # nothing pending
        Cm = C0.clone()
        L.zynum_blas_gpu_inject_fault(HOLD, 1)
        assert _dev_call(L, torch, m, n, k, A, B, Cm) == 0  # enqueued
        st = L.zynum_blas_gpu_device_status(stream)
        assert st < 0, "the held product kernel did not report its abandoned wait"
        assert b"bounded wait" in L.zynum_blas_gpu_last_error()
        assert torch.equal(Cm, C0), "C was written by an abandoned product"
        assert L.zynum_blas_gpu_device_status(stream) == 0  # the report was cleared
        # the next call runs normally: TMEM was freed, the copies drained
        assert _dev_call(L, torch, m, n, k, A, B, Cm) == 0
        assert L.zynum_blas_gpu_device_status(stream) == 0
    finally:
        L.zynum_blas_gpu_set_ozaki_scheme(old_scheme)
        L.zynum_blas_gpu_set_dgemm_method(old_method)
    a = np.asfortranarray(A.cpu().numpy().T)
    b = np.asfortranarray(B.cpu().numpy().T)
    ref = np.asfortranarray(C0.cpu().numpy().T)
    c0 = ref.copy(order="F")
    oracle.gemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, ref, m)
    got = Cm.cpu().numpy().T
    bound = 4 * k * U64 * (np.abs(a) @ np.abs(b) + 0.5 * np.abs(c0))
    assert np.all(np.abs(got - ref) <= bound)


def test_host_entry_point_reports_and_leaves_c(blas, lib):
    """dgemm_ (host buffers) checks the report before copying C back."""
    L = lib
    rng = np.random.default_rng(5)
    m, n, k = 300, 200, 256
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    c0 = c.copy(order="F")
    blas.set_dgemm_method(blas.METHOD_OZAKI)
    old = blas.set_ozaki_scheme(blas.OZAKI_CRT)
    try:
        L.zynum_blas_gpu_inject_fault(HOLD, 1)
        blas.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 1.0, c, m)
        assert np.array_equal(c, c0), "dgemm_ copied back a product it had abandoned"
        assert b"bounded wait" in L.zynum_blas_gpu_last_error()
        blas.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 1.0, c, m)
    finally:
        blas.set_ozaki_scheme(old)
        blas.set_dgemm_method(blas.METHOD_NATIVE)
    np.testing.assert_allclose(c, c0 + a @ b, rtol=1e-12, atol=1e-12)
