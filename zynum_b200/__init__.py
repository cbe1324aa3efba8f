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
    """Scheme ("slices" or "crt"), digit count (slices or moduli) and INT8 product-GEMM
    count the Ozaki DGEMM uses for this shape under the current settings."""
    from ._lib import load
    sc, s, p = _C.c_int(0), _C.c_int(0), _C.c_int(0)
    load().zynum_blas_gpu_ozaki_plan_ex(m, n, k, _C.byref(sc), _C.byref(s), _C.byref(p))
    scheme = "crt" if sc.value == 2 else "slices"
    out = {"scheme": scheme, "products": p.value, "slice_products": p.value}
    out["moduli" if scheme == "crt" else "slices"] = s.value
    out["slices"] = s.value if scheme == "slices" else 0
    return out
