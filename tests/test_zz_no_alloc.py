"""The allocation-free DGEMM entry point (GPU).

zynum_blas_gpu_dgemm_noalloc_device exists for callers that cannot let the
library call cudaMalloc (their device memory belongs to their own pool
allocator, or cudaMalloc's device synchronisation is not acceptable in their
loop).  It keeps its split-K partial sums in a fixed 32 MiB array inside the
library.  This file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
U64 = 2.0 ** -53


def _call_noalloc(L, torch, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, splits):
    stream = torch.cuda.current_stream().cuda_stream
    return L.zynum_blas_gpu_dgemm_noalloc_device(ta.encode(), tb.encode(), m, n, k, alpha, A.data_ptr(), lda,
                                                 B.data_ptr(), ldb, beta, Cm.data_ptr(), ldc, splits, stream)


def _call_existing(L, torch, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    stream = torch.cuda.current_stream().cuda_stream
    return L.zynum_blas_gpu_dgemm_device(ta.encode(), tb.encode(), m, n, k, alpha, A.data_ptr(), lda,
                                         B.data_ptr(), ldb, beta, Cm.data_ptr(), ldc, stream)


@pytest.mark.parametrize("ta,tb,splits", [("N", "N", 0), ("T", "N", 0), ("N", "T", 24)])
def test_noalloc_matches_existing_entry_point_twice(lib, ta, tb, splits):
    import torch
    L = lib
    L.zynum_blas_gpu_set_dgemm_method(0)  # compare against the native method of the existing entry point
    g = torch.Generator(device="cuda").manual_seed(17)
    m, n, k = 256, 192, 65536  # K-dominant: the planner splits K (scratch in use)
    # column-major storage: a torch (cols, ld) row-major tensor
    A = torch.rand((k if ta == "N" else m, m if ta == "N" else k), generator=g, device="cuda",
                   dtype=torch.float64) * 2 - 1
    B = torch.rand((n if tb == "N" else k, k if tb == "N" else n), generator=g, device="cuda",
                   dtype=torch.float64) * 2 - 1
    lda = m if ta == "N" else k
    ldb = k if tb == "N" else n
    C0 = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    ref = C0.clone()
    assert _call_existing(L, torch, ta, tb, m, n, k, 1.5, A, lda, B, ldb, -0.5, ref, m) == 0
    absAB = (A.abs().T if ta == "N" else A.abs()) @ (B.abs().T if tb == "N" else B.abs())  # (m, n)
    bound = 4 * k * U64 * (1.5 * absAB + 0.5 * C0.abs().T)
    for _ in range(2):  # two calls in a row: the shared array keeps the previous call's contents
        out = C0.clone()
        st = _call_noalloc(L, torch, ta, tb, m, n, k, 1.5, A, lda, B, ldb, -0.5, out, m, splits)
        assert st == 0, L.zynum_blas_gpu_last_error()
        torch.cuda.synchronize()
        err = (out - ref).abs().T
        assert bool((err <= bound).all()), float(err.max())


def test_noalloc_rejects_oversized_scratch(lib):
    import torch
    L = lib
    m = n = 1024
    k = 4096
    A = torch.zeros((k, m), device="cuda", dtype=torch.float64)
    B = torch.zeros((n, k), device="cuda", dtype=torch.float64)
    out = torch.full((n, m), 3.0, device="cuda", dtype=torch.float64)
    st = _call_noalloc(L, torch, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m, 8)  # 8 * 1024^2 > 4194304
    assert st < 0
    assert b"exceed the fixed scratch" in L.zynum_blas_gpu_last_error()
    torch.cuda.synchronize()
    assert bool((out == 3.0).all())


def test_noalloc_second_call_allocates_nothing(lib, oracle):
    """After one call per GPU (which loads the library's module there and with it the
    fixed array), a split-K call leaves the GPU's free memory unchanged, and its
    result meets the oracle's bound."""
    import torch
    L = lib
    g = torch.Generator(device="cuda").manual_seed(23)
    m, n, k = 192, 160, 65536  # split K: the planner uses the fixed array
    A = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    B = torch.rand((n, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    C0 = torch.rand((n, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    out = C0.clone()
    assert _call_noalloc(L, torch, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m, 0) == 0  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    out.copy_(C0)
    assert _call_noalloc(L, torch, "N", "N", m, n, k, 1.0, A, m, B, k, 0.5, out, m, 0) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    a = np.asfortranarray(A.cpu().numpy().T)
    b = np.asfortranarray(B.cpu().numpy().T)
    ref = np.asfortranarray(C0.cpu().numpy().T)
    c0 = ref.copy(order="F")
    oracle.gemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, ref, m)
    bound = 4 * k * U64 * (np.abs(a) @ np.abs(b) + 0.5 * np.abs(c0))
    assert np.all(np.abs(out.cpu().numpy().T - ref) <= bound)


def test_noalloc_forced_splits_only_count_where_used(lib):
    """The tall-skinny route keeps no partial sums, so a forced split count does not
    make a large call fail; huge forced counts are capped like the planner's."""
    import torch
    L = lib
    g = torch.Generator(device="cuda").manual_seed(29)
    m, n, k = 131072, 64, 64
    A = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    B = torch.rand((n, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    ref = torch.zeros((n, m), device="cuda", dtype=torch.float64)
    assert _call_existing(L, torch, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, ref, m) == 0
    out = torch.zeros_like(ref)
    st = _call_noalloc(L, torch, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m, 2)
    assert st == 0, L.zynum_blas_gpu_last_error()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    m2, n2, k2 = 64, 48, 1 << 20
    A2 = torch.rand((k2, m2), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    B2 = torch.rand((n2, k2), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    ref2 = torch.zeros((n2, m2), device="cuda", dtype=torch.float64)
    assert _call_existing(L, torch, "N", "N", m2, n2, k2, 1.0, A2, m2, B2, k2, 0.0, ref2, m2) == 0
    out2 = torch.zeros_like(ref2)
    st = _call_noalloc(L, torch, "N", "N", m2, n2, k2, 1.0, A2, m2, B2, k2, 0.0, out2, m2, 100000)
    assert st == 0, L.zynum_blas_gpu_last_error()
    torch.cuda.synchronize()
    absAB = A2.abs().T @ B2.abs().T
    assert bool(((out2 - ref2).abs().T <= 4 * k2 * U64 * absAB).all())
