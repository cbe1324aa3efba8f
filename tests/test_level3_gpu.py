"""SYMM, TRMM and SYR2K on the GEMM tiles against the CPU oracle (GPU).

SYMM mirrors symmetric.zig:56-70 (runSymmColumns): only the stored triangle of
A may be read, so the other one holds NaN here.  TRMM mirrors
triangular.zig:202-231 for every side / uplo / trans / diag, with orders that
cross several 256-row diagonal blocks; the unstored triangle (and the diagonal
when diag = 'U') holds NaN.  SYR2K mirrors symmetric.zig:301-329: the other
triangle of C must stay bit-identical.  Padding rows of every output must stay
bit-identical.  Bounds are componentwise, c n u (|alpha| |op(A)| |op(B)| +
|beta| |C0|), the same form as the GEMM tests.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
U = {np.float64: 2.0 ** -53, np.float32: 2.0 ** -24}
IDS = {np.float64: "d", np.float32: "s"}


def _mat(rng, rows, cols, ld, dtype, sentinel=-999.0):
    a = np.full((ld, max(cols, 1)), sentinel)
    a[:rows, :cols] = rng.uniform(-1.0, 1.0, (rows, cols))
    return np.asfortranarray(a.astype(dtype))


def _poison_unstored(a, n, uplo, diag_too=False):
    """NaN in the triangle the routine must not read (and on the diagonal for diag = 'U')."""
    mask = np.tril(np.ones((n, n), bool), -1) if uplo == "U" else np.triu(np.ones((n, n), bool), 1)
    if diag_too:
        mask |= np.eye(n, dtype=bool)
    a[:n, :n][mask] = np.nan


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=IDS.get)
@pytest.mark.parametrize("side,uplo", list(itertools.product("LR", "UL")))
@pytest.mark.parametrize("m,n,alpha,beta", [(300, 70, 0.75, -0.5), (70, 300, -1.25, 0.0), (5, 3, 1.0, 1.0)],
                         ids=["300x70", "70x300", "5x3"])
def test_symm(blas, oracle, dtype, side, uplo, m, n, alpha, beta):
    rng = np.random.default_rng(int.from_bytes((side + uplo).encode(), "little") + m)
    na = m if side == "L" else n
    lda, ldb, ldc = na + 3, m + 2, m + 1
    a = _mat(rng, na, na, lda, dtype)
    full = np.triu(a[:na, :na]) + np.triu(a[:na, :na], 1).T if uplo == "U" else \
        np.tril(a[:na, :na]) + np.tril(a[:na, :na], -1).T
    _poison_unstored(a, na, uplo)
    b = _mat(rng, m, n, ldb, dtype)
    c = _mat(rng, m, n, ldc, dtype, -777.0)
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, ref, ldc)
    blas.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)
    S = np.abs(full.astype(np.float64))
    B = np.abs(b[:m, :n].astype(np.float64))
    prod = S @ B if side == "L" else B @ S
    bound = 4 * na * U[dtype] * (abs(alpha) * prod + abs(beta) * np.abs(c0[:m, :n].astype(np.float64))) + 1e-300
    err = np.abs(c[:m, :n].astype(np.float64) - ref[:m, :n].astype(np.float64))
    assert np.all(err <= bound), float(err.max())
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"


def _tri_dense(a, n, uplo, trans, diag):
    t = np.triu(a[:n, :n]) if uplo == "U" else np.tril(a[:n, :n])
    if diag == "U":
        t = t - np.diag(np.diag(t)) + np.eye(n)
    return t if trans == "N" else t.T


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NT", "NU")))
def test_dtrmm_all_cases(blas, oracle, side, uplo, trans, diag):
    rng = np.random.default_rng(int.from_bytes((side + uplo + trans + diag).encode(), "little"))
    m, n = (600, 37) if side == "L" else (37, 600)
    na = m if side == "L" else n
    lda, ldb = na + 3, m + 2
    a = _mat(rng, na, na, lda, np.float64)
    T = _tri_dense(a.astype(np.float64), na, uplo, trans, diag)
    _poison_unstored(a, na, uplo, diag_too=(diag == "U"))
    b = _mat(rng, m, n, ldb, np.float64)
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    alpha = 0.75
    oracle.trmm(side, uplo, trans, diag, m, n, alpha, a, lda, ref, ldb)
    blas.trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
    B = np.abs(b0[:m, :n])
    prod = np.abs(T) @ B if side == "L" else B @ np.abs(T)
    bound = 4 * na * U[np.float64] * abs(alpha) * prod + 1e-300
    err = np.abs(b[:m, :n] - ref[:m, :n])
    assert np.all(err <= bound), float(err.max())
    assert np.array_equal(b[m:], b0[m:]), "padding rows of B were written"


@pytest.mark.parametrize("side,uplo,trans", [("L", "L", "N"), ("R", "U", "T"), ("L", "U", "T"), ("R", "L", "N")])
@pytest.mark.parametrize("m,n", [(3, 2), (257, 9), (9, 513)])
def test_strmm(blas, oracle, side, uplo, trans, m, n):
    rng = np.random.default_rng(m * 7 + n)
    na = m if side == "L" else n
    a = _mat(rng, na, na, na, np.float32)
    T = _tri_dense(a.astype(np.float64), na, uplo, trans, "N")
    _poison_unstored(a, na, uplo)
    b = _mat(rng, m, n, m, np.float32)
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    oracle.trmm(side, uplo, trans, "N", m, n, -1.5, a, na, ref, m)
    blas.trmm(side, uplo, trans, "N", m, n, -1.5, a, na, b, m)
    B = np.abs(b0.astype(np.float64))
    prod = np.abs(T) @ B if side == "L" else B @ np.abs(T)
    bound = 4 * na * U[np.float32] * 1.5 * prod + 1e-30
    assert np.all(np.abs(b.astype(np.float64) - ref.astype(np.float64)) <= bound)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=IDS.get)
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NT")))
@pytest.mark.parametrize("n,k,alpha,beta", [(300, 70, 0.75, -0.5), (129, 1000, 1.0, 0.0), (4, 3, -2.0, 1.0)],
                         ids=["300x70", "129x1000", "4x3"])
def test_syr2k(blas, oracle, dtype, uplo, trans, n, k, alpha, beta):
    rng = np.random.default_rng(n + k + ord(uplo) + ord(trans))
    ra, ca = (n, k) if trans == "N" else (k, n)
    lda, ldb, ldc = ra + 2, ra + 5, n + 3
    a = _mat(rng, ra, ca, lda, dtype)
    b = _mat(rng, ra, ca, ldb, dtype)
    c = _mat(rng, n, n, ldc, dtype, -777.0)
    if beta == 0.0:  # beta = 0 must clear NaN in the triangle
        tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
        c[:n, :n][tri] = np.nan
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, ref, ldc)
    blas.syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    A = np.abs(a[:ra, :ca].astype(np.float64))
    B = np.abs(b[:ra, :ca].astype(np.float64))
    if trans != "N":
        A, B = A.T, B.T
    c0n = np.nan_to_num(np.abs(c0[:n, :n].astype(np.float64)))
    bound = 8 * k * U[dtype] * (abs(alpha) * (A @ B.T + B @ A.T) + abs(beta) * c0n) + 1e-300
    tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    got, want = c[:n, :n].astype(np.float64), ref[:n, :n].astype(np.float64)
    assert np.all(np.isfinite(got[tri]))
    assert np.all(np.abs(got - want)[tri] <= bound[tri]), float(np.abs(got - want)[tri].max())
    assert np.array_equal(c[:n, :n][~tri], c0[:n, :n][~tri]), "the other triangle changed"
    assert np.array_equal(c[n:], c0[n:], equal_nan=True), "padding rows of C were written"


def test_argument_errors_leave_outputs(blas):
    """Fortran argument checks (fortran.zig:239-250, :105-117, :264-275): outputs untouched."""
    a = np.ones((4, 4), order="F")
    b = np.ones((4, 4), order="F")
    c = np.full((4, 4), 3.0, order="F")
    c0 = c.copy()
    blas.symm("X", "U", 4, 4, 1.0, a, 4, b, 4, 0.0, c, 4)       # side
    blas.symm("L", "U", 4, 4, 1.0, a, 3, b, 4, 0.0, c, 4)       # lda < m
    blas.syr2k("U", "N", 4, 4, 1.0, a, 4, b, 3, 0.0, c, 4)      # ldb < n
    blas.trmm("L", "U", "N", "Q", 4, 4, 1.0, a, 4, c, 4)        # diag
    assert np.array_equal(c, c0)


def test_cblas_row_major(blas):
    rng = np.random.default_rng(5)
    m, n, k = 40, 30, 20
    S = rng.uniform(-1, 1, (m, m))
    S = np.ascontiguousarray(np.triu(S) + np.triu(S, 1).T)
    B = np.ascontiguousarray(rng.uniform(-1, 1, (m, n)))
    C = np.zeros((m, n))
    blas.cblas_symm(blas.CblasRowMajor, blas.CblasLeft, blas.CblasUpper, m, n, 2.0, S, m, B, n, 0.0, C, n)
    assert np.abs(C - 2.0 * S @ B).max() <= 1e-12
    T = np.ascontiguousarray(np.tril(rng.uniform(-1, 1, (m, m))))
    X = B.copy()
    blas.cblas_trmm(blas.CblasRowMajor, blas.CblasLeft, blas.CblasLower, blas.CblasNoTrans, blas.CblasNonUnit,
                    m, n, 0.5, T, m, X, n)
    assert np.abs(X - 0.5 * T @ B).max() <= 1e-12
    Ak = np.ascontiguousarray(rng.uniform(-1, 1, (m, k)))
    Bk = np.ascontiguousarray(rng.uniform(-1, 1, (m, k)))
    Cs = np.zeros((m, m))
    blas.cblas_syr2k(blas.CblasRowMajor, blas.CblasLower, blas.CblasNoTrans, m, k, 1.0, Ak, k, Bk, k, 0.0, Cs, m)
    want = Ak @ Bk.T + Bk @ Ak.T
    lower = np.tril(np.ones((m, m), bool))
    assert np.abs(Cs - want)[lower].max() <= 1e-12
    assert np.all(Cs[~lower] == 0.0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=IDS.get)
def test_device_entry_points(blas, oracle, dtype):
    """zynum_blas_gpu_{d,s}{symm,trmm,syr2k}_device on torch tensors against the oracle."""
    import torch
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    tol = 1e-12 if dtype == np.float64 else 2e-4
    rng = np.random.default_rng(9)
    m, n = 520, 33
    a = np.asfortranarray(rng.uniform(-1, 1, (m, m)).astype(dtype))
    b = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(dtype))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(dtype))
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")  # noqa: E731  column-major storage
    host = lambda t: np.asfortranarray(t.cpu().numpy().T)  # noqa: E731

    ref = c.copy(order="F")
    oracle.symm("L", "L", m, n, 0.5, a, m, b, m, 2.0, ref, m)
    C = dev(c)
    blas.symm_device("L", "L", m, n, 0.5, dev(a), m, dev(b), m, 2.0, C, m)
    torch.cuda.synchronize()
    assert np.abs(host(C) - ref).max() <= tol * max(1.0, np.abs(ref).max())

    ref = b.copy(order="F")
    oracle.trmm("L", "U", "T", "N", m, n, 1.0, a, m, ref, m)
    B = dev(b)
    blas.trmm_device("L", "U", "T", "N", m, n, 1.0, dev(a), m, B, m)
    torch.cuda.synchronize()
    assert np.abs(host(B) - ref).max() <= tol * max(1.0, np.abs(ref).max())

    k = n
    ref = np.asfortranarray(np.zeros((m, m), dtype))
    oracle.syr2k("U", "N", m, k, 1.0, b, m, c, m, 0.0, ref, m)
    Cs = torch.zeros((m, m), device="cuda", dtype=tdt)
    blas.syr2k_device("U", "N", m, k, 1.0, dev(b), m, dev(c), m, 0.0, Cs, m)
    torch.cuda.synchronize()
    up = np.triu(np.ones((m, m), bool))
    got = host(Cs)
    assert np.abs(got - ref)[up].max() <= tol * max(1.0, np.abs(ref).max())
    assert np.all(got[~up] == 0.0)


@pytest.mark.parametrize("routine", ["syrk", "syr2k"])
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NT")))
def test_rank_k_ozaki_route(blas, oracle, routine, uplo, trans):
    """DSYRK / DSYR2K under the Ozaki method: one full emulated product W into scratch, then
    alpha (W [+ W^T]) + beta C on the triangle; the other triangle and padding stay bit-identical,
    beta = 0 clears NaN."""
    rng = np.random.default_rng(ord(uplo) * 3 + ord(trans) + len(routine))
    n, k = 301, 190
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = _mat(rng, ra, ca, ra + 1, np.float64)
    b = _mat(rng, ra, ca, ra + 2, np.float64)
    old = blas.set_dgemm_method(blas.METHOD_OZAKI)
    try:
        for alpha, beta in ((0.75, -0.5), (1.0, 0.0)):
            c = _mat(rng, n, n, n + 3, np.float64, -777.0)
            tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
            if beta == 0.0:
                c[:n, :n][tri] = np.nan
            c0 = c.copy(order="F")
            ref = c.copy(order="F")
            if routine == "syrk":
                oracle.syrk(uplo, trans, n, k, alpha, a, ra + 1, beta, ref, n + 3)
                blas.syrk(uplo, trans, n, k, alpha, a, ra + 1, beta, c, n + 3)
                A = np.abs(a[:ra, :ca]) if trans == "N" else np.abs(a[:ra, :ca]).T
                prod = A @ A.T
            else:
                oracle.syr2k(uplo, trans, n, k, alpha, a, ra + 1, b, ra + 2, beta, ref, n + 3)
                blas.syr2k(uplo, trans, n, k, alpha, a, ra + 1, b, ra + 2, beta, c, n + 3)
                A = np.abs(a[:ra, :ca]) if trans == "N" else np.abs(a[:ra, :ca]).T
                B = np.abs(b[:ra, :ca]) if trans == "N" else np.abs(b[:ra, :ca]).T
                prod = A @ B.T + B @ A.T
            bound = 8 * k * U[np.float64] * (abs(alpha) * prod + abs(beta) * np.nan_to_num(np.abs(c0[:n, :n])))
            err = np.abs(c[:n, :n] - ref[:n, :n])
            assert np.all(np.isfinite(c[:n, :n][tri]))
            assert np.all(err[tri] <= bound[tri] + 1e-300), float(err[tri].max())
            assert np.array_equal(c[:n, :n][~tri], c0[:n, :n][~tri]), "the other triangle changed"
            assert np.array_equal(c[n:], c0[n:]), "padding rows of C were written"
    finally:
        blas.set_dgemm_method(old)


@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NT")))
def test_syrk_ozaki_triangle_tiles(blas, oracle, uplo, trans):
    """DSYRK under the Ozaki method on several 256 x 256 tiles per side: the modular products
    run only on the tiles meeting the stored triangle and op(A) is split once (op(B)^T is
    op(A)); the stored triangle meets the oracle's bound, the other triangle is untouched."""
    rng = np.random.default_rng(ord(uplo) * 5 + ord(trans))
    n, k = 1100, 700
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = _mat(rng, ra, ca, ra + 2, np.float64)
    c = _mat(rng, n, n, n + 1, np.float64, -777.0)
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    alpha, beta = -0.5, 1.25
    old = blas.set_dgemm_method(blas.METHOD_OZAKI)
    try:
        oracle.syrk(uplo, trans, n, k, alpha, a, ra + 2, beta, ref, n + 1)
        blas.syrk(uplo, trans, n, k, alpha, a, ra + 2, beta, c, n + 1)
    finally:
        blas.set_dgemm_method(old)
    tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    A = np.abs(a[:ra, :ca]) if trans == "N" else np.abs(a[:ra, :ca]).T
    bound = 8 * k * U[np.float64] * (abs(alpha) * (A @ A.T) + abs(beta) * np.abs(c0[:n, :n]))
    err = np.abs(c[:n, :n] - ref[:n, :n])
    assert np.all(err[tri] <= bound[tri] + 1e-300), float(err[tri].max())
    assert np.array_equal(c[:n, :n][~tri], c0[:n, :n][~tri]), "the other triangle changed"
    assert np.array_equal(c[n:], c0[n:]), "padding rows of C were written"
