"""Python mirror of the Zynum BLAS GEMM-path interface over the C ABI.

Host functions (`dgemm`, `sgemm`, `cblas_dgemm`, ...) take numpy arrays in
column-major storage exactly like the Fortran routines take pointers: a matrix
with leading dimension `ld` is an array of shape (ld, cols), order='F'.  They
call the library's `dgemm_` / `cblas_dgemm` symbols, so they behave exactly
like a C or Fortran caller: xerbla_ on an illegal argument, C untouched.

Device functions (`dgemm_device`, ...) take CUDA torch tensors (column-major
views, i.e. tensors whose stride is (1, ld)) and run on the current torch
stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load

CblasRowMajor, CblasColMajor = 101, 102
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113
CblasUpper, CblasLower = 121, 122
CblasNonUnit, CblasUnit = 131, 132
CblasLeft, CblasRight = 141, 142

METHOD_NATIVE, METHOD_OZAKI, METHOD_AUTO = 0, 1, 2
SMETHOD_NATIVE, SMETHOD_BF16X3, SMETHOD_OZAKI = 0, 1, 2


def _i(v: int):
    return C.byref(C.c_int32(int(v)))


def _ptr(a) -> int:
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor


def _ch(c: str) -> bytes:
    return c.encode()[:1]


def dgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Fortran dgemm_ on host arrays (in-place on c)."""
    al, be = np.array([alpha], np.float64), np.array([beta], np.float64)
    load().dgemm_(_ch(transa), _ch(transb), _i(m), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
                  _i(ldb), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def sgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    al, be = np.array([alpha], np.float32), np.array([beta], np.float32)
    load().sgemm_(_ch(transa), _ch(transb), _i(m), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
                  _i(ldb), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def cblas_dgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    load().cblas_dgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta),
                       _ptr(c), ldc)
    return c


def cblas_sgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    load().cblas_sgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta),
                       _ptr(c), ldc)
    return c


def _cscalar(dtype, v):
    return np.array([complex(v)], dtype=dtype)


def zgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Fortran zgemm_ on complex128 host arrays (in-place on c)."""
    al, be = _cscalar(np.complex128, alpha), _cscalar(np.complex128, beta)
    load().zgemm_(_ch(transa), _ch(transb), _i(m), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
                  _i(ldb), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def cgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    al, be = _cscalar(np.complex64, alpha), _cscalar(np.complex64, beta)
    load().cgemm_(_ch(transa), _ch(transb), _i(m), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
                  _i(ldb), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def cblas_zgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    al, be = _cscalar(np.complex128, alpha), _cscalar(np.complex128, beta)
    load().cblas_zgemm(layout, transa, transb, m, n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data,
                       _ptr(c), ldc)
    return c


def cblas_cgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    al, be = _cscalar(np.complex64, alpha), _cscalar(np.complex64, beta)
    load().cblas_cgemm(layout, transa, transb, m, n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data,
                       _ptr(c), ldc)
    return c


def trsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """Fortran ?trsm_ on host arrays (d / s / z / c from b's dtype; in-place on b)."""
    L = load()
    if np.iscomplexobj(b):
        fn = L.ztrsm_ if b.dtype == np.complex128 else L.ctrsm_
        al = np.array([alpha], b.dtype)
        fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), _i(m), _i(n), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
           _i(ldb))
        return b
    fn, dt = (L.dtrsm_, np.float64) if b.dtype == np.float64 else (L.strsm_, np.float32)
    al = np.array([alpha], dt)
    fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), _i(m), _i(n), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
       _i(ldb))
    return b


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """Fortran ?syrk_ on host arrays (d / s / z / c from c's dtype; in-place on c's triangle)."""
    L = load()
    if np.iscomplexobj(c):
        fn = L.zsyrk_ if c.dtype == np.complex128 else L.csyrk_
        al, be = np.array([alpha], c.dtype), np.array([beta], c.dtype)
        fn(_ch(uplo), _ch(trans), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), be.ctypes.data, _ptr(c), _i(ldc))
        return c
    fn, dt = (L.dsyrk_, np.float64) if c.dtype == np.float64 else (L.ssyrk_, np.float32)
    al, be = np.array([alpha], dt), np.array([beta], dt)
    fn(_ch(uplo), _ch(trans), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """Fortran ?symm_ on host arrays (d / s / z / c from c's dtype; in-place on c); with herm
    (complex only) zhemm_ / chemm_."""
    L = load()
    if np.iscomplexobj(c):
        z = c.dtype == np.complex128
        fn = (L.zhemm_ if z else L.chemm_) if herm else (L.zsymm_ if z else L.csymm_)
        al, be = np.array([alpha], c.dtype), np.array([beta], c.dtype)
    else:
        fn, dt = (L.dsymm_, np.float64) if c.dtype == np.float64 else (L.ssymm_, np.float32)
        al, be = np.array([alpha], dt), np.array([beta], dt)
    fn(_ch(side), _ch(uplo), _i(m), _i(n), al.ctypes.data, _ptr(a), _i(lda), _ptr(b), _i(ldb), be.ctypes.data,
       _ptr(c), _i(ldc))
    return c


def hemm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """Fortran zhemm_ / chemm_ on host arrays (dtype from c; in-place on c)."""
    return symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=True)


def trmm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """Fortran ?trmm_ on host arrays (d / s / z / c from b's dtype; in-place on b)."""
    L = load()
    if np.iscomplexobj(b):
        fn = L.ztrmm_ if b.dtype == np.complex128 else L.ctrmm_
        al = np.array([alpha], b.dtype)
    else:
        fn, dt = (L.dtrmm_, np.float64) if b.dtype == np.float64 else (L.strmm_, np.float32)
        al = np.array([alpha], dt)
    fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), _i(m), _i(n), al.ctypes.data, _ptr(a), _i(lda), _ptr(b),
       _i(ldb))
    return b


def syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """Fortran ?syr2k_ on host arrays (d / s / z / c from c's dtype; in-place on c's triangle);
    with herm (complex only) zher2k_ / cher2k_, beta real."""
    L = load()
    if np.iscomplexobj(c):
        z = c.dtype == np.complex128
        al = np.array([alpha], c.dtype)
        if herm:
            fn, be = (L.zher2k_ if z else L.cher2k_), np.array([float(np.real(beta))], np.float64 if z else np.float32)
        else:
            fn, be = (L.zsyr2k_ if z else L.csyr2k_), np.array([beta], c.dtype)
    else:
        fn, dt = (L.dsyr2k_, np.float64) if c.dtype == np.float64 else (L.ssyr2k_, np.float32)
        al, be = np.array([alpha], dt), np.array([beta], dt)
    fn(_ch(uplo), _ch(trans), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), _ptr(b), _i(ldb), be.ctypes.data,
       _ptr(c), _i(ldc))
    return c


def her2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Fortran zher2k_ / cher2k_ on host arrays (beta real; in-place on c's triangle)."""
    return syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, herm=True)


def herk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """Fortran zherk_ / cherk_ on host arrays (alpha, beta real; in-place on c's triangle)."""
    L = load()
    z = c.dtype == np.complex128
    fn, rt = (L.zherk_, np.float64) if z else (L.cherk_, np.float32)
    al, be = np.array([float(alpha)], rt), np.array([float(beta)], rt)
    fn(_ch(uplo), _ch(trans), _i(n), _i(k), al.ctypes.data, _ptr(a), _i(lda), be.ctypes.data, _ptr(c), _i(ldc))
    return c


def cblas_symm(layout, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """cblas_dsymm / cblas_ssymm (dtype from c)."""
    L = load()
    fn, cast = (L.cblas_dsymm, float) if c.dtype == np.float64 else (L.cblas_ssymm, float)
    fn(layout, side, uplo, m, n, cast(alpha), _ptr(a), lda, _ptr(b), ldb, cast(beta), _ptr(c), ldc)
    return c


def cblas_trmm(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """cblas_dtrmm / cblas_strmm (dtype from b)."""
    L = load()
    fn = L.cblas_dtrmm if b.dtype == np.float64 else L.cblas_strmm
    fn(layout, side, uplo, transa, diag, m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb)
    return b


def cblas_syr2k(layout, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """cblas_dsyr2k / cblas_ssyr2k (dtype from c)."""
    L = load()
    fn = L.cblas_dsyr2k if c.dtype == np.float64 else L.cblas_ssyr2k
    fn(layout, uplo, trans, n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc)
    return c


def cblas_dtrsm(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    load().cblas_dtrsm(layout, side, uplo, transa, diag, m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb)
    return b


def cblas_dsyrk(layout, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    load().cblas_dsyrk(layout, uplo, trans, n, k, float(alpha), _ptr(a), lda, float(beta), _ptr(c), ldc)
    return c


def set_complex_method(method: int) -> int:
    return load().zynum_blas_gpu_set_complex_method(method)


COMPLEX_4M, COMPLEX_3M = 0, 1


def _stream(stream=None) -> int:
    if stream is not None:
        return int(stream)
    import torch
    return int(torch.cuda.current_stream().cuda_stream)


def dgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    """Device dgemm on torch CUDA tensors / raw device pointers; raises on a non-zero status."""
    st = load().zynum_blas_gpu_dgemm_device(_ch(transa), _ch(transb), m, n, k, float(alpha), _ptr(a), lda,
                                            _ptr(b), ldb, float(beta), _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_dgemm_device")
    return c


def sgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    st = load().zynum_blas_gpu_sgemm_device(_ch(transa), _ch(transb), m, n, k, float(alpha), _ptr(a), lda,
                                            _ptr(b), ldb, float(beta), _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_sgemm_device")
    return c


def zgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    """Device zgemm on complex128 torch CUDA tensors (alpha / beta are Python numbers)."""
    al, be = _cscalar(np.complex128, alpha), _cscalar(np.complex128, beta)
    st = load().zynum_blas_gpu_zgemm_device(_ch(transa), _ch(transb), m, n, k, al.ctypes.data, _ptr(a), lda,
                                            _ptr(b), ldb, be.ctypes.data, _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_zgemm_device")
    return c


def cgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    al, be = _cscalar(np.complex64, alpha), _cscalar(np.complex64, beta)
    st = load().zynum_blas_gpu_cgemm_device(_ch(transa), _ch(transb), m, n, k, al.ctypes.data, _ptr(a), lda,
                                            _ptr(b), ldb, be.ctypes.data, _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_cgemm_device")
    return c


def dtrsm_device(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream=None):
    st = load().zynum_blas_gpu_dtrsm_device(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, float(alpha),
                                            _ptr(a), lda, _ptr(b), ldb, _stream(stream))
    check(st, "zynum_blas_gpu_dtrsm_device")
    return b


def dtrsm_inverse_bytes(n):
    """Bytes of the diagonal-block inverses of an n x n triangular matrix."""
    return int(load().zynum_blas_gpu_dtrsm_inverse_bytes(n))


def dtrsm_inverse_device(uplo, diag, n, a, lda, inv, stream=None):
    """inv (a device buffer of dtrsm_inverse_bytes(n)) := the inverses of A's diagonal blocks."""
    st = load().zynum_blas_gpu_dtrsm_inverse_device(_ch(uplo), _ch(diag), n, _ptr(a), lda, _ptr(inv), _stream(stream))
    check(st, "zynum_blas_gpu_dtrsm_inverse_device")
    return inv


def dtrsm_with_inverse_device(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, inv, stream=None):
    """dtrsm_device with the inverses dtrsm_inverse_device formed for the same A, uplo and diag."""
    st = load().zynum_blas_gpu_dtrsm_with_inverse_device(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n,
                                                         float(alpha), _ptr(a), lda, _ptr(b), ldb, _ptr(inv),
                                                         _stream(stream))
    check(st, "zynum_blas_gpu_dtrsm_with_inverse_device")
    return b


def dsyrk_device(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream=None):
    st = load().zynum_blas_gpu_dsyrk_device(_ch(uplo), _ch(trans), n, k, float(alpha), _ptr(a), lda, float(beta),
                                            _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_dsyrk_device")
    return c


def trsm_device_c(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream=None):
    """Device ztrsm / ctrsm on complex128 / complex64 torch tensors (in place on b)."""
    import torch
    L = load()
    z = b.dtype == torch.complex128
    fn, dt = (L.zynum_blas_gpu_ztrsm_device, np.complex128) if z else (L.zynum_blas_gpu_ctrsm_device, np.complex64)
    al = _cscalar(dt, alpha)
    st = fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb,
            _stream(stream))
    check(st, "zynum_blas_gpu_ztrsm_device" if z else "zynum_blas_gpu_ctrsm_device")
    return b


def syrk_device_c(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream=None):
    """Device zsyrk / csyrk on complex128 / complex64 torch tensors (c's triangle)."""
    import torch
    L = load()
    z = c.dtype == torch.complex128
    fn, dt = (L.zynum_blas_gpu_zsyrk_device, np.complex128) if z else (L.zynum_blas_gpu_csyrk_device, np.complex64)
    al, be = _cscalar(dt, alpha), _cscalar(dt, beta)
    st = fn(_ch(uplo), _ch(trans), n, k, al.ctypes.data, _ptr(a), lda, be.ctypes.data, _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_zsyrk_device" if z else "zynum_blas_gpu_csyrk_device")
    return c


def symm_device_c(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=False, stream=None):
    """Device zsymm / csymm (zhemm / chemm with herm) on complex128 / complex64 torch tensors."""
    import torch
    L = load()
    z = c.dtype == torch.complex128
    p = "z" if z else "c"
    name = f"zynum_blas_gpu_{p}{'hemm' if herm else 'symm'}_device"
    dt = np.complex128 if z else np.complex64
    al, be = _cscalar(dt, alpha), _cscalar(dt, beta)
    st = getattr(L, name)(_ch(side), _ch(uplo), m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data,
                          _ptr(c), ldc, _stream(stream))
    check(st, name)
    return c


def trmm_device_c(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream=None):
    """Device ztrmm / ctrmm on complex128 / complex64 torch tensors (in place on b)."""
    import torch
    L = load()
    z = b.dtype == torch.complex128
    fn, dt = (L.zynum_blas_gpu_ztrmm_device, np.complex128) if z else (L.zynum_blas_gpu_ctrmm_device, np.complex64)
    al = _cscalar(dt, alpha)
    st = fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb,
            _stream(stream))
    check(st, "zynum_blas_gpu_ztrmm_device" if z else "zynum_blas_gpu_ctrmm_device")
    return b


def syr2k_device_c(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, herm=False, stream=None):
    """Device zsyr2k / csyr2k (zher2k / cher2k with herm: beta real) on complex torch tensors."""
    import torch
    L = load()
    z = c.dtype == torch.complex128
    p = "z" if z else "c"
    dt = np.complex128 if z else np.complex64
    al = _cscalar(dt, alpha)
    if herm:
        name = f"zynum_blas_gpu_{p}her2k_device"
        st = getattr(L, name)(_ch(uplo), _ch(trans), n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb,
                              float(np.real(beta)), _ptr(c), ldc, _stream(stream))
    else:
        name = f"zynum_blas_gpu_{p}syr2k_device"
        be = _cscalar(dt, beta)
        st = getattr(L, name)(_ch(uplo), _ch(trans), n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb,
                              be.ctypes.data, _ptr(c), ldc, _stream(stream))
    check(st, name)
    return c


def herk_device(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream=None):
    """Device zherk / cherk on complex torch tensors (alpha, beta real; c's triangle, real diagonal)."""
    import torch
    L = load()
    z = c.dtype == torch.complex128
    fn = L.zynum_blas_gpu_zherk_device if z else L.zynum_blas_gpu_cherk_device
    st = fn(_ch(uplo), _ch(trans), n, k, float(alpha), _ptr(a), lda, float(beta), _ptr(c), ldc, _stream(stream))
    check(st, "zynum_blas_gpu_zherk_device" if z else "zynum_blas_gpu_cherk_device")
    return c


def cblas_trsm_c(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """cblas_ztrsm / cblas_ctrsm (dtype from b)."""
    L = load()
    fn = L.cblas_ztrsm if b.dtype == np.complex128 else L.cblas_ctrsm
    al = np.array([alpha], b.dtype)
    fn(layout, side, uplo, transa, diag, m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb)
    return b


def cblas_symm_c(layout, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """cblas_zsymm / cblas_csymm, or cblas_zhemm / cblas_chemm with herm (dtype from c)."""
    L = load()
    z = c.dtype == np.complex128
    fn = (L.cblas_zhemm if z else L.cblas_chemm) if herm else (L.cblas_zsymm if z else L.cblas_csymm)
    al, be = np.array([alpha], c.dtype), np.array([beta], c.dtype)
    fn(layout, side, uplo, m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data, _ptr(c), ldc)
    return c


def cblas_trmm_c(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """cblas_ztrmm / cblas_ctrmm (dtype from b)."""
    L = load()
    fn = L.cblas_ztrmm if b.dtype == np.complex128 else L.cblas_ctrmm
    al = np.array([alpha], b.dtype)
    fn(layout, side, uplo, transa, diag, m, n, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb)
    return b


def cblas_syr2k_c(layout, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """cblas_zsyr2k / cblas_csyr2k, or cblas_zher2k / cblas_cher2k (beta real) with herm."""
    L = load()
    z = c.dtype == np.complex128
    al = np.array([alpha], c.dtype)
    if herm:
        fn = L.cblas_zher2k if z else L.cblas_cher2k
        fn(layout, uplo, trans, n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, float(np.real(beta)), _ptr(c), ldc)
    else:
        fn = L.cblas_zsyr2k if z else L.cblas_csyr2k
        be = np.array([beta], c.dtype)
        fn(layout, uplo, trans, n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data, _ptr(c), ldc)
    return c


def cblas_herk(layout, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """cblas_zherk / cblas_cherk (alpha, beta real)."""
    L = load()
    fn = L.cblas_zherk if c.dtype == np.complex128 else L.cblas_cherk
    fn(layout, uplo, trans, n, k, float(alpha), _ptr(a), lda, float(beta), _ptr(c), ldc)
    return c


def symm_device(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    """Device dsymm / ssymm on torch CUDA tensors (dtype from c)."""
    import torch
    L = load()
    fn, name = ((L.zynum_blas_gpu_dsymm_device, "dsymm") if c.dtype == torch.float64
                else (L.zynum_blas_gpu_ssymm_device, "ssymm"))
    st = fn(_ch(side), _ch(uplo), m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc,
            _stream(stream))
    check(st, f"zynum_blas_gpu_{name}_device")
    return c


def trmm_device(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream=None):
    """Device dtrmm / strmm on torch CUDA tensors (dtype from b; in-place on b)."""
    import torch
    L = load()
    fn, name = ((L.zynum_blas_gpu_dtrmm_device, "dtrmm") if b.dtype == torch.float64
                else (L.zynum_blas_gpu_strmm_device, "strmm"))
    st = fn(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb,
            _stream(stream))
    check(st, f"zynum_blas_gpu_{name}_device")
    return b


def syr2k_device(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    """Device dsyr2k / ssyr2k on torch CUDA tensors (dtype from c)."""
    import torch
    L = load()
    fn, name = ((L.zynum_blas_gpu_dsyr2k_device, "dsyr2k") if c.dtype == torch.float64
                else (L.zynum_blas_gpu_ssyr2k_device, "ssyr2k"))
    st = fn(_ch(uplo), _ch(trans), n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc,
            _stream(stream))
    check(st, f"zynum_blas_gpu_{name}_device")
    return c


def set_dgemm_method(method: int) -> int:
    return load().zynum_blas_gpu_set_dgemm_method(method)


def set_sgemm_method(method: int) -> int:
    return load().zynum_blas_gpu_set_sgemm_method(method)


def set_ozaki_slices(slices: int) -> int:
    return load().zynum_blas_gpu_set_ozaki_slices(slices)


OZAKI_AUTO, OZAKI_SLICES, OZAKI_CRT = 0, 1, 2


def set_ozaki_scheme(scheme: int) -> int:
    """0 = automatic, 1 = INT8 slices (scheme I), 2 = CRT residues (scheme II)."""
    return load().zynum_blas_gpu_set_ozaki_scheme(scheme)


def set_ozaki_moduli(moduli: int) -> int:
    """CRT moduli 2..16; 0 = default."""
    return load().zynum_blas_gpu_set_ozaki_moduli(moduli)


def inject_fault(kind: int, count: int) -> None:
    load().zynum_blas_gpu_inject_fault(kind, count)


def last_error() -> str:
    return load().zynum_blas_gpu_last_error().decode(errors="replace")


def shutdown() -> None:
    load().zynum_blas_shutdown()


# ------------------------------------------------------------------ batches
class _Batch:
    def __init__(self, handle):
        self.handle = handle

    def info(self):
        items, grid = C.c_int(0), C.c_int(0)
        cfg = (C.c_int * 3)()
        load().zynum_blas_gpu_batch_info(self.handle, C.byref(items), C.byref(grid), cfg)
        return {"items": items.value, "grid": grid.value, "tiles_per_cfg": {32: cfg[0], 64: cfg[1], 128: cfg[2]}}

    def close(self):
        if self.handle:
            load().zynum_blas_gpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _int_array(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


class GemmBatch(_Batch):
    """Variable-size batched GEMM plan (one persistent kernel per run).

    m, n, k: per-problem sizes (host sequences).  run() takes torch CUDA
    tensors (or raw device pointers) for the per-problem operands.
    """

    def __init__(self, m, n, k, dtype="f64", transa="N", transb="N", tune=False):
        self.dt = 0 if dtype in ("f64", np.float64) else 1
        m, n, k = _int_array(m), _int_array(n), _int_array(k)
        h = C.c_void_p()
        st = load().zynum_blas_gpu_gemm_batch_create(C.byref(h), self.dt, _ch(transa), _ch(transb), len(m),
                                                     m.ctypes.data, n.ctypes.data, k.ctypes.data, int(tune))
        check(st, "zynum_blas_gpu_gemm_batch_create")
        super().__init__(h)
        self.count = len(m)

    def run(self, alpha, a_ptrs, lda, b_ptrs, ldb, beta, c_ptrs, ldc, stream=None, use_graph=False):
        """a_ptrs / b_ptrs / c_ptrs: int64 CUDA tensors of device addresses; lda/ldb/ldc: int32 CUDA tensors."""
        fn = load().zynum_blas_gpu_dgemm_batch_run if self.dt == 0 else load().zynum_blas_gpu_sgemm_batch_run
        st = fn(self.handle, float(alpha), _ptr(a_ptrs), _ptr(lda), _ptr(b_ptrs), _ptr(ldb), float(beta),
                _ptr(c_ptrs), _ptr(ldc), _stream(stream), int(use_graph))
        check(st, "gemm_batch_run")


class TrsmBatch(_Batch):
    """Left-side variable-size batched TRSM plan: B_q (m_q x n_q, n_q <= 64) := alpha op(A_q)^-1 B_q."""

    def __init__(self, m, n, dtype="f64", uplo="L", transa="N", diag="N"):
        self.dt = 0 if dtype in ("f64", np.float64) else 1
        m, n = _int_array(m), _int_array(n)
        h = C.c_void_p()
        st = load().zynum_blas_gpu_trsm_batch_create(C.byref(h), self.dt, b"L", _ch(uplo), _ch(transa), _ch(diag),
                                                     len(m), m.ctypes.data, n.ctypes.data)
        check(st, "zynum_blas_gpu_trsm_batch_create")
        super().__init__(h)
        self.count = len(m)

    def run(self, alpha, a_ptrs, lda, b_ptrs, ldb, stream=None, use_graph=False):
        fn = load().zynum_blas_gpu_dtrsm_batch_run if self.dt == 0 else load().zynum_blas_gpu_strsm_batch_run
        st = fn(self.handle, float(alpha), _ptr(a_ptrs), _ptr(lda), _ptr(b_ptrs), _ptr(ldb), _stream(stream),
                int(use_graph))
        check(st, "trsm_batch_run")
