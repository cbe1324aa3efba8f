"""Zynum BLAS GEMM backend for NVIDIA B200 (sm_100a).

The product is the C-ABI shared library ``zynum_b200/lib/libzynum_blas_gpu.so``
(Fortran ``dgemm_``/``sgemm_``/..., CBLAS ``cblas_?gemm``/..., and device-pointer
``zynum_blas_gpu_*_device`` entry points).  This package loads it with ctypes:

* :mod:`zynum_b200.blas`      Python mirror of the Fortran / CBLAS / device API
* :mod:`zynum_b200.autograd`  torch.autograd.Function adjoints (GEMM, TRSM, SYRK)
"""
from __future__ import annotations

import ctypes as _C


def ozaki_info(m: int, n: int, k: int) -> dict:
    """Slice count and slice-product count the Ozaki DGEMM uses for this shape."""
    from ._lib import load
    s, p = _C.c_int(0), _C.c_int(0)
    load().zynum_blas_gpu_ozaki_plan(m, n, k, _C.byref(s), _C.byref(p))
    return {"slices": s.value, "slice_products": p.value}
