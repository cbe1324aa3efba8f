"""numpy front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker or the timed CPU reference.  The product
(zynum_b200) never imports it.

All matrices are numpy arrays in Fortran (column-major) order with an explicit
leading dimension: a matrix with ld rows of storage and `cols` columns is an
array of shape (ld, cols), order='F'.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = _HERE / "lib" / "liboracle.so"
        if not path.exists():
            from oracle import build as _b  # noqa: WPS433
            _b.build()
        _LIB = C.CDLL(str(path))
        _declare(_LIB)
    return _LIB


def _declare(L):
    i32, f64, f32, ch = C.c_int32, C.c_double, C.c_float, C.c_char
    vp = C.c_void_p
    L.oracle_dgemm.argtypes = [ch, ch, i32, i32, i32, f64, vp, i32, vp, i32, f64, vp, i32]
    L.oracle_sgemm.argtypes = [ch, ch, i32, i32, i32, f32, vp, i32, vp, i32, f32, vp, i32]
    L.oracle_zgemm.argtypes = [ch, ch, i32, i32, i32, vp, vp, i32, vp, i32, vp, vp, i32]
    L.oracle_cgemm.argtypes = [ch, ch, i32, i32, i32, vp, vp, i32, vp, i32, vp, vp, i32]
    L.oracle_ddgemm.argtypes = [ch, ch, i32, i32, i32, vp, i32, vp, i32, vp, vp, i32]
    L.oracle_ddgemm_sampled.argtypes = [ch, ch, i32, vp, i32, vp, i32, C.c_int64, vp, vp, vp, vp, vp]
    L.oracle_ddgemm_sampled_f32.argtypes = [ch, ch, i32, vp, i32, vp, i32, C.c_int64, vp, vp, vp, vp, vp]
    L.oracle_dtrsm.argtypes = [ch, ch, ch, ch, i32, i32, f64, vp, i32, vp, i32]
    L.oracle_strsm.argtypes = [ch, ch, ch, ch, i32, i32, f32, vp, i32, vp, i32]
    L.oracle_dsyrk.argtypes = [ch, ch, i32, i32, f64, vp, i32, f64, vp, i32]
    L.oracle_ssyrk.argtypes = [ch, ch, i32, i32, f32, vp, i32, f32, vp, i32]
    L.oracle_ztrsm.argtypes = [ch, ch, ch, ch, i32, i32, vp, vp, i32, vp, i32]
    L.oracle_ctrsm.argtypes = [ch, ch, ch, ch, i32, i32, vp, vp, i32, vp, i32]
    L.oracle_zsyrk.argtypes = [ch, ch, i32, i32, vp, vp, i32, vp, vp, i32]
    L.oracle_csyrk.argtypes = [ch, ch, i32, i32, vp, vp, i32, vp, vp, i32]
    L.oracle_dsymm.argtypes = [ch, ch, i32, i32, f64, vp, i32, vp, i32, f64, vp, i32]
    L.oracle_ssymm.argtypes = [ch, ch, i32, i32, f32, vp, i32, vp, i32, f32, vp, i32]
    L.oracle_dtrmm.argtypes = [ch, ch, ch, ch, i32, i32, f64, vp, i32, vp, i32]
    L.oracle_strmm.argtypes = [ch, ch, ch, ch, i32, i32, f32, vp, i32, vp, i32]
    L.oracle_dsyr2k.argtypes = [ch, ch, i32, i32, f64, vp, i32, vp, i32, f64, vp, i32]
    L.oracle_ssyr2k.argtypes = [ch, ch, i32, i32, f32, vp, i32, vp, i32, f32, vp, i32]
    for name in ("oracle_zsymm", "oracle_csymm"):
        getattr(L, name).argtypes = [ch, ch, i32, i32, vp, vp, i32, vp, i32, vp, vp, i32, C.c_int]
    for name in ("oracle_ztrmm", "oracle_ctrmm"):
        getattr(L, name).argtypes = [ch, ch, ch, ch, i32, i32, vp, vp, i32, vp, i32]
    L.oracle_zherk.argtypes = [ch, ch, i32, i32, f64, vp, i32, f64, vp, i32]
    L.oracle_cherk.argtypes = [ch, ch, i32, i32, f32, vp, i32, f32, vp, i32]
    for name in ("oracle_zsyr2k", "oracle_csyr2k"):
        getattr(L, name).argtypes = [ch, ch, i32, i32, vp, vp, i32, vp, i32, vp, vp, i32, C.c_int]


def _p(a: np.ndarray):
    assert a.flags.f_contiguous or a.ndim == 1
    return a.ctypes.data


def _b(c: str) -> bytes:
    return c.encode()[:1]


def gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """In-place C update, dtype picked from `c` (f64, f32, c128, c64)."""
    L = lib()
    if c.dtype == np.float64:
        L.oracle_dgemm(_b(ta), _b(tb), m, n, k, alpha, _p(a), lda, _p(b), ldb, beta, _p(c), ldc)
    elif c.dtype == np.float32:
        L.oracle_sgemm(_b(ta), _b(tb), m, n, k, alpha, _p(a), lda, _p(b), ldb, beta, _p(c), ldc)
    elif c.dtype == np.complex128:
        al = np.array([complex(alpha)], np.complex128)
        be = np.array([complex(beta)], np.complex128)
        L.oracle_zgemm(_b(ta), _b(tb), m, n, k, _p(al), _p(a), lda, _p(b), ldb, _p(be), _p(c), ldc)
    elif c.dtype == np.complex64:
        al = np.array([complex(alpha)], np.complex64)
        be = np.array([complex(beta)], np.complex64)
        L.oracle_cgemm(_b(ta), _b(tb), m, n, k, _p(al), _p(a), lda, _p(b), ldb, _p(be), _p(c), ldc)
    else:
        raise TypeError(c.dtype)
    return c


def ddgemm(ta, tb, m, n, k, a, lda, b, ldb):
    """Double-double op(A) op(B): returns (hi, lo) m x n arrays."""
    hi = np.zeros((m, n), np.float64, order="F")
    lo = np.zeros((m, n), np.float64, order="F")
    lib().oracle_ddgemm(_b(ta), _b(tb), m, n, k, _p(a), lda, _p(b), ldb, _p(hi), _p(lo), m)
    return hi, lo


def ddgemm_sampled(ta, tb, k, a, lda, b, ldb, rows, cols):
    """Double-double entries (hi, lo, sum|a||b|) of op(A) op(B) at (rows[q], cols[q])."""
    rows = np.ascontiguousarray(rows, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    n = rows.size
    hi, lo, ab = (np.zeros(n, np.float64) for _ in range(3))
    fn = lib().oracle_ddgemm_sampled if a.dtype == np.float64 else lib().oracle_ddgemm_sampled_f32
    fn(_b(ta), _b(tb), k, _p(a), lda, _p(b), ldb, n, rows.ctypes.data, cols.ctypes.data,
       hi.ctypes.data, lo.ctypes.data, ab.ctypes.data)
    return hi, lo, ab


def trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """In place on b; dtype from b (f64, f32, c128, c64)."""
    L = lib()
    if np.iscomplexobj(b):
        f = L.oracle_ztrsm if b.dtype == np.complex128 else L.oracle_ctrsm
        al = np.array([alpha], dtype=b.dtype)
        f(_b(side), _b(uplo), _b(trans), _b(diag), m, n, al.ctypes.data, _p(a), lda, _p(b), ldb)
        return b
    f = L.oracle_dtrsm if b.dtype == np.float64 else L.oracle_strsm
    f(_b(side), _b(uplo), _b(trans), _b(diag), m, n, alpha, _p(a), lda, _p(b), ldb)
    return b


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """In place on c's triangle; dtype from c (f64, f32, c128, c64)."""
    L = lib()
    if np.iscomplexobj(c):
        f = L.oracle_zsyrk if c.dtype == np.complex128 else L.oracle_csyrk
        al, be = np.array([alpha], dtype=c.dtype), np.array([beta], dtype=c.dtype)
        f(_b(uplo), _b(trans), n, k, al.ctypes.data, _p(a), lda, be.ctypes.data, _p(c), ldc)
        return c
    f = L.oracle_dsyrk if c.dtype == np.float64 else L.oracle_ssyrk
    f(_b(uplo), _b(trans), n, k, alpha, _p(a), lda, beta, _p(c), ldc)
    return c


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """In place on c; dtype from c.  herm (complex only): A Hermitian (zhemm / chemm)."""
    L = lib()
    if np.iscomplexobj(c):
        f = L.oracle_zsymm if c.dtype == np.complex128 else L.oracle_csymm
        al, be = np.array([alpha], dtype=c.dtype), np.array([beta], dtype=c.dtype)
        f(_b(side), _b(uplo), m, n, al.ctypes.data, _p(a), lda, _p(b), ldb, be.ctypes.data, _p(c), ldc, int(herm))
        return c
    f = L.oracle_dsymm if c.dtype == np.float64 else L.oracle_ssymm
    f(_b(side), _b(uplo), m, n, alpha, _p(a), lda, _p(b), ldb, beta, _p(c), ldc)
    return c


def trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    L = lib()
    if np.iscomplexobj(b):
        f = L.oracle_ztrmm if b.dtype == np.complex128 else L.oracle_ctrmm
        al = np.array([alpha], dtype=b.dtype)
        f(_b(side), _b(uplo), _b(trans), _b(diag), m, n, al.ctypes.data, _p(a), lda, _p(b), ldb)
        return b
    f = L.oracle_dtrmm if b.dtype == np.float64 else L.oracle_strmm
    f(_b(side), _b(uplo), _b(trans), _b(diag), m, n, alpha, _p(a), lda, _p(b), ldb)
    return b


def syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, herm=False):
    """In place on c's triangle.  herm (complex only): zher2k / cher2k (beta real)."""
    L = lib()
    if np.iscomplexobj(c):
        f = L.oracle_zsyr2k if c.dtype == np.complex128 else L.oracle_csyr2k
        al, be = np.array([alpha], dtype=c.dtype), np.array([beta], dtype=c.dtype)
        f(_b(uplo), _b(trans), n, k, al.ctypes.data, _p(a), lda, _p(b), ldb, be.ctypes.data, _p(c), ldc, int(herm))
        return c
    f = L.oracle_dsyr2k if c.dtype == np.float64 else L.oracle_ssyr2k
    f(_b(uplo), _b(trans), n, k, alpha, _p(a), lda, _p(b), ldb, beta, _p(c), ldc)
    return c


def herk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """zherk / cherk in place on c's triangle (alpha, beta real; diagonal made real)."""
    L = lib()
    f = L.oracle_zherk if c.dtype == np.complex128 else L.oracle_cherk
    f(_b(uplo), _b(trans), n, k, float(alpha), _p(a), lda, float(beta), _p(c), ldc)
    return c
