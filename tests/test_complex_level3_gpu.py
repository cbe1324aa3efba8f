"""Complex Level-3 beyond GEMM / TRSM / SYRK on the GPU against the C oracle:
ZSYMM / ZHEMM (and C), ZTRMM / CTRMM, ZHERK / CHERK, ZSYR2K / ZHER2K (and C),
through the Fortran and CBLAS exports.  Bounds are the usual forward-error
bounds c k u (|alpha| |op(A)| |op(B)| + |beta| |C|); untouched triangles and
padding must come back bit-identical; Hermitian diagonals exactly real.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cx(rng, shape, dtype):
    return np.asfortranarray((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype))


def _u(dtype):
    return 2.0 ** -53 if dtype == np.complex128 else 2.0 ** -24


def _op(x, trans):
    return x if trans == "N" else (x.T if trans == "T" else x.conj().T)


def _seed(*parts):
    return int.from_bytes("".join(map(str, parts)).encode(), "little") % 2**32


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("herm", [False, True], ids=["symm", "hemm"])
@pytest.mark.parametrize("side,uplo", list(itertools.product("LR", "UL")))
def test_symm_hemm(blas, oracle, dtype, herm, side, uplo):
    """The unstored triangle of A holds garbage and the diagonal a nonzero imaginary part:
    SYMM mirrors, HEMM mirrors conjugated and ignores the diagonal's imaginary part."""
    rng = np.random.default_rng(_seed(side, uplo, herm, dtype.__name__))
    m, n = 300, 70
    na = m if side == "L" else n
    lda, ldb, ldc = na + 1, m + 2, m + 3
    a = _cx(rng, (lda, na), dtype)
    b = _cx(rng, (ldb, n), dtype)
    for alpha, beta in ((0.5 - 0.75j, 0.25 + 0.5j), (1.0 - 0.5j, 0.0)):
        c = _cx(rng, (ldc, n), dtype)
        if beta == 0.0:
            c[:m] = np.nan
        c0 = c.copy(order="F")
        ref = c.copy(order="F")
        oracle.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, ref, ldc, herm=herm)
        blas.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, herm=herm)
        A = np.abs(a[:na, :na].astype(np.complex128))
        S = np.triu(A) + np.triu(A, 1).T if uplo == "U" else np.tril(A) + np.tril(A, -1).T
        B = np.abs(b[:m, :n].astype(np.complex128))
        prod = S @ B if side == "L" else B @ S
        bound = 8 * na * _u(dtype) * (abs(alpha) * prod + abs(beta) * np.nan_to_num(np.abs(c0[:m]))) + 1e-300
        err = np.abs(c[:m].astype(np.complex128) - ref[:m])
        assert np.all(np.isfinite(c[:m]))
        assert np.all(err <= bound), float((err / bound).max())
        assert np.array_equal(c[m:], c0[m:], equal_nan=True)


def _ctri(rng, na, ld, dtype):
    a = (rng.standard_normal((ld, na)) + 1j * rng.standard_normal((ld, na))) / np.sqrt(2 * na)
    for i in range(na):
        a[i, i] = 1.0 + 0.5 * rng.standard_normal() + 0.5j * rng.standard_normal()
    a[na:] = -999.0
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NTC", "NU")))
def test_ztrmm_all_cases(blas, oracle, side, uplo, trans, diag):
    """ZTRMM: every side / uplo / trans (C conjugates) / diag; orders of 600 cross three
    256-row diagonal blocks; complex alpha; padding rows of B untouched."""
    rng = np.random.default_rng(_seed(side, uplo, trans, diag))
    m, n = (600, 37) if side == "L" else (37, 600)
    na = m if side == "L" else n
    lda, ldb = na + 2, m + 3
    a = _ctri(rng, na, lda, np.complex128)
    b = _cx(rng, (ldb, n), np.complex128)
    b[m:] = -999.0
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    alpha = 0.75 - 0.5j
    oracle.trmm(side, uplo, trans, diag, m, n, alpha, a, lda, ref, ldb)
    blas.trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
    T = np.abs(a[:na, :na])
    T = np.triu(T) if uplo == "U" else np.tril(T)
    if diag == "U":
        np.fill_diagonal(T, 1.0)
    T = T if trans == "N" else T.T
    B = np.abs(b0[:m, :n])
    bound = 8 * na * _u(np.complex128) * abs(alpha) * (T @ B if side == "L" else B @ T) + 1e-300
    err = np.abs(b[:m] - ref[:m])
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(b[m:], b0[m:])


@pytest.mark.parametrize("side,uplo,trans", [("L", "L", "N"), ("R", "U", "C"), ("L", "U", "C"), ("R", "L", "T")])
def test_ctrmm(blas, oracle, side, uplo, trans):
    rng = np.random.default_rng(_seed(side, uplo, trans))
    m, n = (300, 20) if side == "L" else (20, 300)
    na = m if side == "L" else n
    a = _ctri(rng, na, na, np.complex64)
    b = _cx(rng, (m, n), np.complex64)
    ref = b.copy(order="F")
    oracle.trmm(side, uplo, trans, "N", m, n, 1.0 + 0.5j, a, na, ref, m)
    blas.trmm(side, uplo, trans, "N", m, n, 1.0 + 0.5j, a, na, b, m)
    assert np.all(np.abs(b - ref) <= 1e-4 * (1 + np.abs(ref)))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NTC")))
def test_herk(blas, oracle, dtype, uplo, trans):
    """ZHERK / CHERK: alpha, beta real; the triangle within c k u (|alpha| |A||A|^T + |beta| |C|),
    its diagonal exactly real, the other triangle and the padding bit-identical; beta = 0
    clears NaN."""
    rng = np.random.default_rng(_seed(uplo, trans, dtype.__name__))
    n, k = 150, 90
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = _cx(rng, (ra + 1, ca), dtype)
    for alpha, beta in ((0.75, -0.5), (1.0, 0.0)):
        c = _cx(rng, (n + 2, n), dtype)
        tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
        if beta == 0.0:
            c[:n][tri] = np.nan
        c0 = c.copy(order="F")
        ref = c.copy(order="F")
        oracle.herk(uplo, trans, n, k, alpha, a, ra + 1, beta, ref, n + 2)
        blas.herk(uplo, trans, n, k, alpha, a, ra + 1, beta, c, n + 2)
        A = np.abs(a[:ra, :ca].astype(np.complex128))
        A = A if trans == "N" else A.T
        bound = 8 * k * _u(dtype) * (abs(alpha) * (A @ A.T) + abs(beta) * np.nan_to_num(np.abs(c0[:n]))) + 1e-300
        got, want = c[:n].astype(np.complex128), ref[:n].astype(np.complex128)
        assert np.all(np.isfinite(got[tri]))
        assert np.all(np.abs(got - want)[tri] <= bound[tri]), float(np.abs(got - want)[tri].max())
        assert np.all(np.diag(c[:n]).imag == 0), "Hermitian diagonal not real"
        assert np.array_equal(c[:n][~tri], c0[:n][~tri], equal_nan=True), "the other triangle changed"
        assert np.array_equal(c[n:], c0[n:], equal_nan=True)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
def test_herk_k_zero_and_alpha_zero(blas, oracle, dtype):
    """k = 0 or alpha = 0: C := beta C on the triangle with the diagonal made real; A is not read."""
    rng = np.random.default_rng(31)
    n = 40
    for k, alpha in ((0, 1.0), (5, 0.0)):
        a = _cx(rng, (n, max(k, 1)), dtype)
        c = _cx(rng, (n, n), dtype)
        ref = c.copy(order="F")
        oracle.herk("L", "N", n, k, alpha, a, n, 0.5, ref, n)
        blas.herk("L", "N", n, k, alpha, a, n, 0.5, c, n)
        assert np.array_equal(c, ref)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("herm", [False, True], ids=["syr2k", "her2k"])
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NTC")))
def test_syr2k_her2k(blas, oracle, dtype, herm, uplo, trans):
    """ZSYR2K (op = C conjugates op(A), op(B)) and ZHER2K (alpha W + conj(alpha) W^H, beta
    real, diagonal exactly real); the other triangle bit-identical."""
    rng = np.random.default_rng(_seed(uplo, trans, herm, dtype.__name__))
    n, k = 130, 75
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = _cx(rng, (ra, ca), dtype)
    b = _cx(rng, (ra + 2, ca), dtype)
    alpha = 0.5 + 0.75j
    for beta in ((0.25 if herm else 0.25 - 0.5j), 0.0):
        c = _cx(rng, (n + 1, n), dtype)
        tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
        if beta == 0.0:
            c[:n][tri] = np.nan
        c0 = c.copy(order="F")
        ref = c.copy(order="F")
        oracle.syr2k(uplo, trans, n, k, alpha, a, ra, b, ra + 2, beta, ref, n + 1, herm=herm)
        blas.syr2k(uplo, trans, n, k, alpha, a, ra, b, ra + 2, beta, c, n + 1, herm=herm)
        A = np.abs(a.astype(np.complex128))
        B = np.abs(b[:ra].astype(np.complex128))
        A, B = (A, B) if trans == "N" else (A.T, B.T)
        prod = A @ B.T + B @ A.T
        bound = 8 * k * _u(dtype) * (abs(alpha) * prod + abs(beta) * np.nan_to_num(np.abs(c0[:n]))) + 1e-300
        got, want = c[:n].astype(np.complex128), ref[:n].astype(np.complex128)
        assert np.all(np.isfinite(got[tri]))
        assert np.all(np.abs(got - want)[tri] <= bound[tri]), float(np.abs(got - want)[tri].max())
        if herm:
            assert np.all(np.diag(c[:n]).imag == 0), "Hermitian diagonal not real"
        assert np.array_equal(c[:n][~tri], c0[:n][~tri], equal_nan=True)
        assert np.array_equal(c[n:], c0[n:], equal_nan=True)


def test_cblas_row_major_complex(blas, oracle):
    """Row-major CBLAS calls reach the Fortran routine with side / uplo flipped and trans
    mapped as the reference's cblas layer maps them: each result equals the oracle run on
    the mapped column-major arguments."""
    rng = np.random.default_rng(41)
    m, n, k = 90, 60, 50
    tol = 1e-12
    R = blas.CblasRowMajor
    # ZHEMM, side left, upper: row-major A (m x m) is column-major A^T with lower stored
    A = np.ascontiguousarray(rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m)))
    B = np.ascontiguousarray(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
    C = np.ascontiguousarray(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
    ref = np.asfortranarray(C.T.copy())
    oracle.symm("R", "L", n, m, 0.5 + 1j, np.asfortranarray(A.T), m, np.asfortranarray(B.T), n, 0.25, ref, n,
                herm=True)
    blas.cblas_symm_c(R, blas.CblasLeft, blas.CblasUpper, m, n, 0.5 + 1j, A, m, B, n, 0.25, C, n, herm=True)
    assert np.abs(C.T - ref).max() <= tol * (1 + np.abs(ref).max())
    # ZHERK, upper, no-trans: Fortran ('L', 'T') on the column-major view A^T (k x n)
    Ak = np.ascontiguousarray(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))
    C = np.ascontiguousarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ref = np.asfortranarray(C.T.copy())
    oracle.herk("L", "T", n, k, 1.5, np.asfortranarray(Ak.T), k, 0.5, ref, n)
    blas.cblas_herk(R, blas.CblasUpper, blas.CblasNoTrans, n, k, 1.5, Ak, k, 0.5, C, n)
    assert np.abs(C.T - ref).max() <= tol * (1 + np.abs(ref).max())
    # ZHER2K, lower, no-trans: Fortran ('U', 'T') on the column-major views (k x n)
    Ak = np.ascontiguousarray(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))
    Bk = np.ascontiguousarray(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))
    C = np.ascontiguousarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ref = np.asfortranarray(C.T.copy())
    oracle.syr2k("U", "T", n, k, 0.5 - 0.5j, np.asfortranarray(Ak.T), k, np.asfortranarray(Bk.T), k, 2.0, ref, n,
                 herm=True)
    blas.cblas_syr2k_c(R, blas.CblasLower, blas.CblasNoTrans, n, k, 0.5 - 0.5j, Ak, k, Bk, k, 2.0, C, n,
                       herm=True)
    assert np.abs(C.T - ref).max() <= tol * (1 + np.abs(ref).max())
    # ZTRMM right, lower, conj-trans, unit
    At = np.ascontiguousarray(_ctri(rng, n, n, np.complex128).T)
    X = np.ascontiguousarray(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
    ref = np.asfortranarray(X.T.copy())
    oracle.trmm("L", "U", "C", "U", n, m, 1.0 - 2.0j, np.asfortranarray(At.T), n, ref, n)
    blas.cblas_trmm_c(R, blas.CblasRight, blas.CblasLower, blas.CblasConjTrans, blas.CblasUnit, m, n, 1.0 - 2.0j,
                      At, n, X, n)
    assert np.abs(X.T - ref).max() <= tol * (1 + np.abs(ref).max())


def test_complex_argument_errors_leave_outputs(blas):
    """An invalid argument reports through xerbla and leaves C untouched (uplo 'X')."""
    c = _cx(np.random.default_rng(3), (8, 8), np.complex128)
    c0 = c.copy(order="F")
    a = _cx(np.random.default_rng(4), (8, 8), np.complex128)
    blas.herk("X", "N", 8, 8, 1.0, a, 8, 0.0, c, 8)
    blas.syr2k("U", "N", 8, 8, 1.0, a, 8, a, 8, 0.0, c, 4, herm=True)
    assert np.array_equal(c, c0)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
def test_complex_level3_device_entry_points(blas, oracle, dtype):
    """zynum_blas_gpu_{z,c}{symm,hemm,trmm,syr2k,her2k,herk}_device on torch tensors against the
    oracle on the same column-major data (device pointers, the caller's stream)."""
    import torch
    rng = np.random.default_rng(51 if dtype == np.complex128 else 52)
    tol = 1e-11 if dtype == np.complex128 else 2e-4
    tdt = torch.complex128 if dtype == np.complex128 else torch.complex64
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda", tdt)  # noqa: E731
    host = lambda t: np.asfortranarray(t.cpu().numpy().T)  # noqa: E731
    m, n, k = 140, 90, 70
    rel = lambda got, ref: np.abs(got - ref).max() / (1 + np.abs(ref).max())  # noqa: E731
    for herm in (False, True):  # SYMM / HEMM, side L, uplo U
        a, b, c = _cx(rng, (m, m), dtype), _cx(rng, (m, n), dtype), _cx(rng, (m, n), dtype)
        ref = c.copy(order="F")
        oracle.symm("L", "U", m, n, 0.5 + 0.25j, a, m, b, m, 1.5 - 0.5j, ref, m, herm=herm)
        C = dev(c)
        blas.symm_device_c("L", "U", m, n, 0.5 + 0.25j, dev(a), m, dev(b), m, 1.5 - 0.5j, C, m, herm=herm)
        torch.cuda.synchronize()
        assert rel(host(C), ref) <= tol, ("symm", herm)
    # TRMM, side R, lower, op = C
    a, b = _ctri(rng, n, n, dtype), _cx(rng, (m, n), dtype)
    ref = b.copy(order="F")
    oracle.trmm("R", "L", "C", "N", m, n, 2.0 - 1.0j, a, n, ref, m)
    B = dev(b)
    blas.trmm_device_c("R", "L", "C", "N", m, n, 2.0 - 1.0j, dev(a), n, B, m)
    torch.cuda.synchronize()
    assert rel(host(B), ref) <= tol, "trmm"
    up = np.triu(np.ones((n, n), bool))
    for herm in (False, True):  # SYR2K / HER2K, upper, op = C
        a, b, c = _cx(rng, (k, n), dtype), _cx(rng, (k, n), dtype), _cx(rng, (n, n), dtype)
        beta = 0.5 if herm else 0.5 + 0.5j
        ref = c.copy(order="F")
        oracle.syr2k("U", "C", n, k, 1.0 - 0.5j, a, k, b, k, beta, ref, n, herm=herm)
        C = dev(c)
        blas.syr2k_device_c("U", "C", n, k, 1.0 - 0.5j, dev(a), k, dev(b), k, beta, C, n, herm=herm)
        torch.cuda.synchronize()
        got = host(C)
        assert rel(got[up], ref[up]) <= tol, ("syr2k", herm)
        assert np.array_equal(got[~up], c[~up])
    # HERK, lower, op = N
    a, c = _cx(rng, (n, k), dtype), _cx(rng, (n, n), dtype)
    ref = c.copy(order="F")
    oracle.herk("L", "N", n, k, 1.25, a, n, -0.5, ref, n)
    C = dev(c)
    blas.herk_device("L", "N", n, k, 1.25, dev(a), n, -0.5, C, n)
    torch.cuda.synchronize()
    got = host(C)
    lo = np.tril(np.ones((n, n), bool))
    assert rel(got[lo], ref[lo]) <= tol, "herk"
    assert np.all(np.diag(got).imag == 0)
    assert np.array_equal(got[~lo], c[~lo])


@pytest.mark.parametrize("method", ["4M", "3M"])
@pytest.mark.parametrize("uplo,trans", [("U", "N"), ("L", "C"), ("L", "T")])
def test_herk_zsyrk_triangle_products_large(blas, oracle, method, uplo, trans):
    """ZHERK / ZSYRK compute only the stored triangle of the product (128 x 128 real tiles in
    triangle mode, K beyond 1024), through both complex forms; the other triangle stays untouched."""
    rng = np.random.default_rng(_seed(uplo, trans, method))
    n, k = 700, 1100
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = _cx(rng, (ra, ca), np.complex128)
    tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    A = np.abs(a)
    A = A if trans == "N" else A.T
    old = blas.set_complex_method(blas.COMPLEX_3M if method == "3M" else blas.COMPLEX_4M)
    try:
        for herm in (True, False):
            if not herm and trans == "C":
                continue  # zsyrk takes N / T
            c = _cx(rng, (n, n), np.complex128)
            c0 = c.copy(order="F")
            ref = c.copy(order="F")
            if herm:
                oracle.herk(uplo, trans, n, k, 0.75, a, ra, -0.5, ref, n)
                blas.herk(uplo, trans, n, k, 0.75, a, ra, -0.5, c, n)
            else:
                oracle.syrk(uplo, trans, n, k, 0.75 - 0.25j, a, ra, -0.5 + 0.5j, ref, n)
                blas.syrk(uplo, trans, n, k, 0.75 - 0.25j, a, ra, -0.5 + 0.5j, c, n)
            bound = 16 * k * _u(np.complex128) * ((A @ A.T) + np.abs(c0)) + 1e-300
            assert np.all(np.abs(c - ref)[tri] <= bound[tri]), float(np.abs(c - ref)[tri].max())
            assert np.array_equal(c[~tri], c0[~tri]), "the other triangle changed"
    finally:
        blas.set_complex_method(old)
