"""TRSM and SYRK on the GEMM tiles against the CPU oracle (GPU).

TRSM mirrors src/blas/triangular_parallel_test.zig (every side / uplo / trans /
diag) with sizes that cross several 64-row diagonal blocks, padded leading
dimensions and alpha != 1; the bound is |X - X_ref| <= 1e-11 (1 + |X_ref|)
for the well-conditioned triangles used (diagonal 2 + |N(0,1)|).
SYRK mirrors symmetric.zig:180-199: only the chosen triangle changes (the
other one must stay bit-identical), bound 4 k u (|alpha| |A||A^T| + |beta| |C|).
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tri_matrix(rng, n, ld, dtype):
    a = rng.standard_normal((ld, n)) * 0.3
    for i in range(n):
        a[i, i] = 2.0 + abs(a[i, i])
    a[n:] = -999.0
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NT", "NU")))
def test_dtrsm_all_cases(blas, oracle, side, uplo, trans, diag):
    rng = np.random.default_rng(abs(hash((side, uplo, trans, diag))) % 2**32)
    m, n = (150, 37) if side == "L" else (37, 150)
    na = m if side == "L" else n
    lda, ldb = na + 3, m + 2
    a = _tri_matrix(rng, na, lda, np.float64)
    b = np.asfortranarray(rng.standard_normal((ldb, n)))
    b[m:] = -999.0
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, trans, diag, m, n, 0.75, a, lda, ref, ldb)
    blas.trsm(side, uplo, trans, diag, m, n, 0.75, a, lda, b, ldb)
    err = np.abs(b[:m] - ref[:m])
    assert np.all(err <= 1e-11 * (1 + np.abs(ref[:m]))), float(err.max())
    assert np.array_equal(b[m:], b0[m:])


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NT", "NU")))
def test_dtrsm_multi_leaf(blas, oracle, side, uplo, trans, diag):
    """Orders of 700 cross three 256-row leaves (the last one partial, with a partial 64-block);
    45 right-hand sides leave the last 16-column group of each leaf launch partial."""
    rng = np.random.default_rng(int.from_bytes((side + uplo + trans + diag).encode(), "little") % 2**32)
    m, n = (700, 45) if side == "L" else (45, 700)
    na = m if side == "L" else n
    lda, ldb = na + 1, m + 3
    # off-diagonals N(0, 1/na): well conditioned also with a unit diagonal at this order
    a = rng.standard_normal((lda, na)) / np.sqrt(na)
    for i in range(na):
        a[i, i] = 2.0 + abs(a[i, i])
    a[na:] = -999.0
    a = np.asfortranarray(a)
    b = np.asfortranarray(rng.standard_normal((ldb, n)))
    b[m:] = -999.0
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, trans, diag, m, n, -1.5, a, lda, ref, ldb)
    blas.trsm(side, uplo, trans, diag, m, n, -1.5, a, lda, b, ldb)
    err = np.abs(b[:m] - ref[:m])
    assert np.all(err <= 1e-11 * (1 + np.abs(ref[:m]))), float(err.max())
    assert np.array_equal(b[m:], b0[m:])


@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("L", "U", "T", "U"), ("R", "U", "N", "N"),
                                                   ("R", "L", "T", "U")])
def test_dtrsm_wide_right_hand_sides(blas, oracle, side, uplo, trans, diag):
    """More than 1024 right-hand sides: each leaf inverse is applied as a GEMM from a copy of the
    leaf's rows (columns for side R)."""
    rng = np.random.default_rng(int.from_bytes((side + uplo + trans + diag).encode(), "little") % 2**32)
    m, n = (600, 1100) if side == "L" else (1100, 600)
    na = m if side == "L" else n
    a = rng.standard_normal((na, na)) / np.sqrt(na)
    for i in range(na):
        a[i, i] = 2.0 + abs(a[i, i])
    a = np.asfortranarray(a)
    b = np.asfortranarray(rng.standard_normal((m + 1, n)))
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, trans, diag, m, n, 0.5, a, na, ref, m + 1)
    blas.trsm(side, uplo, trans, diag, m, n, 0.5, a, na, b, m + 1)
    err = np.abs(b[:m] - ref[:m])
    assert np.all(err <= 1e-11 * (1 + np.abs(ref[:m]))), float(err.max())
    assert np.array_equal(b[m:], b0[m:])


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NT", "NU")))
@pytest.mark.parametrize("wide", [False, True], ids=["clusters", "wide"])
def test_dtrsm_with_inverse(blas, oracle, side, uplo, trans, diag, wide):
    """Diagonal-block inverses formed once (dtrsm_inverse_device) and used by several solves
    (dtrsm_with_inverse_device): every side / transpose from one set of inverses of A, with
    three leaves (the last partial) and 45 or 1100 right-hand sides (leaf applies by the cluster
    kernel or as GEMMs), against the oracle, with B's padding rows untouched."""
    import torch
    rng = np.random.default_rng(int.from_bytes((side + uplo + trans + diag + str(wide)).encode(), "little") % 2**32)
    na, nrhs = 700, (1100 if wide else 45)
    m, n = (na, nrhs) if side == "L" else (nrhs, na)
    lda, ldb = na + 2, m + 3  # even lda: the inverses need a 16-byte aligned A
    a = rng.standard_normal((lda, na)) / np.sqrt(na)
    for i in range(na):
        a[i, i] = 2.0 + abs(a[i, i])
    a[na:] = -999.0
    a = np.asfortranarray(a)
    b = np.asfortranarray(rng.standard_normal((ldb, n)))
    b[m:] = -999.0
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, trans, diag, m, n, -1.5, a, lda, ref, ldb)
    ta = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    inv = torch.empty(blas.dtrsm_inverse_bytes(na) // 8, dtype=torch.float64, device="cuda")
    blas.dtrsm_inverse_device(uplo, diag, na, ta, lda, inv)
    for _ in range(2):  # the same inverses serve repeated solves
        tb = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
        blas.dtrsm_with_inverse_device(side, uplo, trans, diag, m, n, -1.5, ta, lda, tb, ldb, inv)
        got = np.asfortranarray(tb.cpu().numpy().T)
        err = np.abs(got[:m] - ref[:m])
        assert np.all(err <= 1e-11 * (1 + np.abs(ref[:m]))), float(err.max())
        assert np.array_equal(got[m:], b[m:])


def test_dtrsm_inverse_argument_errors(blas):
    """Bad arguments are numbered; an unaligned A is refused with a message."""
    import torch
    L = blas.load()
    a = torch.eye(64, dtype=torch.float64, device="cuda")
    inv = torch.empty(blas.dtrsm_inverse_bytes(64) // 8, dtype=torch.float64, device="cuda")
    assert L.zynum_blas_gpu_dtrsm_inverse_device(b"X", b"N", 64, a.data_ptr(), 64, inv.data_ptr(), None) == 1
    assert L.zynum_blas_gpu_dtrsm_inverse_device(b"L", b"X", 64, a.data_ptr(), 64, inv.data_ptr(), None) == 2
    assert L.zynum_blas_gpu_dtrsm_inverse_device(b"L", b"N", -1, a.data_ptr(), 64, inv.data_ptr(), None) == 3
    assert L.zynum_blas_gpu_dtrsm_inverse_device(b"L", b"N", 64, a.data_ptr(), 32, inv.data_ptr(), None) == 5
    assert L.zynum_blas_gpu_dtrsm_inverse_device(b"L", b"N", 64, a.data_ptr(), 64, None, None) == 6
    st = L.zynum_blas_gpu_dtrsm_inverse_device(b"L", b"N", 63, a.data_ptr() + 8, 63, inv.data_ptr(), None)
    assert st < 0 and b"16-byte aligned" in L.zynum_blas_gpu_last_error()
    b = torch.zeros((8, 64), dtype=torch.float64, device="cuda")
    assert L.zynum_blas_gpu_dtrsm_with_inverse_device(b"L", b"L", b"N", b"N", 64, 8, 1.0, a.data_ptr(), 64,
                                                      b.data_ptr(), 64, None, None) == 12
    assert blas.dtrsm_inverse_bytes(0) == 0


@pytest.mark.parametrize("side,uplo", [("L", "L"), ("R", "U"), ("L", "U"), ("R", "L")])
def test_strsm_multi_leaf(blas, oracle, side, uplo):
    rng = np.random.default_rng(4)
    m, n = (530, 20) if side == "L" else (20, 530)
    na = m if side == "L" else n
    a = _tri_matrix(rng, na, na, np.float32)
    b = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, "T", "N", m, n, 1.0, a, na, ref, m)
    blas.trsm(side, uplo, "T", "N", m, n, 1.0, a, na, b, m)
    assert np.all(np.abs(b - ref) <= 2e-4 * (1 + np.abs(ref)))


@pytest.mark.parametrize("side,uplo", [("L", "L"), ("R", "U")])
def test_strsm(blas, oracle, side, uplo):
    rng = np.random.default_rng(2)
    m, n = (130, 20) if side == "L" else (20, 130)
    na = m if side == "L" else n
    a = _tri_matrix(rng, na, na, np.float32)
    b = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, "N", "N", m, n, 1.0, a, na, ref, m)
    blas.trsm(side, uplo, "N", "N", m, n, 1.0, a, na, b, m)
    assert np.all(np.abs(b - ref) <= 2e-4 * (1 + np.abs(ref)))


def test_dtrsm_differentiation_shape(blas, oracle):
    """L lower with off-diagonals N(0, 1/n), diagonal 1 + |N(0,1)| (the chain's TRSM), n = 512, 64 RHS."""
    rng = np.random.default_rng(11)
    n, r = 512, 64
    L = np.tril(rng.standard_normal((n, n)) / np.sqrt(n), -1) + np.diag(1 + np.abs(rng.standard_normal(n)))
    L = np.asfortranarray(L)
    B = np.asfortranarray(rng.standard_normal((n, r)))
    ref = B.copy(order="F")
    oracle.trsm("L", "L", "N", "N", n, r, 1.0, L, n, ref, n)
    blas.trsm("L", "L", "N", "N", n, r, 1.0, L, n, B, n)
    assert np.abs(B - ref).max() <= 1e-11 * (1 + np.abs(ref).max())


def test_cblas_dtrsm_row_major(blas):
    rng = np.random.default_rng(3)
    m, n = 70, 90
    A = np.tril(rng.standard_normal((m, m)) * 0.3) + np.diag(2 + np.abs(rng.standard_normal(m)))
    B = rng.standard_normal((m, n))
    want = np.linalg.solve(A, 0.5 * B)
    a = np.ascontiguousarray(A)
    b = np.ascontiguousarray(B)
    blas.cblas_dtrsm(blas.CblasRowMajor, blas.CblasLeft, blas.CblasLower, blas.CblasNoTrans, blas.CblasNonUnit,
                     m, n, 0.5, a, m, b, n)
    assert np.abs(b - want).max() <= 1e-11 * (1 + np.abs(want).max())


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NT")))
def test_syrk(blas, oracle, dtype, uplo, trans):
    rng = np.random.default_rng(5)
    n, k = 150, 77
    lda = (n if trans == "N" else k) + 2
    ldc = n + 3
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, k if trans == "N" else n)).astype(dtype))
    c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(dtype))
    c[n:] = -777.0
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.syrk(uplo, trans, n, k, 1.5, a, lda, 0.5, ref, ldc)
    blas.syrk(uplo, trans, n, k, 1.5, a, lda, 0.5, c, ldc)
    opA = (a[:n, :k] if trans == "N" else a[:k, :n].T).astype(np.float64)
    u = 2.0 ** -53 if dtype == np.float64 else 2.0 ** -24
    bound = 4 * k * u * (1.5 * np.abs(opA) @ np.abs(opA).T + 0.5 * np.abs(c0[:n, :n]))
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    err = np.abs(c[:n, :n].astype(np.float64) - ref[:n, :n])
    assert np.all(err[mask] <= bound[mask])
    assert np.array_equal(c[:n, :n][~mask], c0[:n, :n][~mask]), "the other triangle changed"
    assert np.array_equal(c[n:], c0[n:])


def test_syrk_k_zero_and_split(blas, oracle):
    rng = np.random.default_rng(6)
    n = 40
    c = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    ref = c.copy(order="F")
    a = np.zeros((n, 1), order="F")
    oracle.syrk("L", "N", n, 0, 1.0, a, n, 2.0, ref, n)
    blas.syrk("L", "N", n, 0, 1.0, a, n, 2.0, c, n)
    assert np.array_equal(c, ref)
    # long K, few tiles: split-K with the triangle mask in the reduction
    n, k = 96, 30000
    a = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.syrk("U", "T", n, k, 1.0, a, k, -1.0, ref, n)
    blas.syrk("U", "T", n, k, 1.0, a, k, -1.0, c, n)
    mask = np.triu(np.ones((n, n), bool))
    assert np.abs(c - ref)[mask].max() <= 4 * k * 2.0 ** -53 * (np.abs(a).T @ np.abs(a) + 1)[mask].max()
    assert np.array_equal(c[~mask], c0[~mask])


def _ctri(rng, na, ld, dtype):
    """Complex triangle source: off-diagonals N(0, 1/na) (re and im), diagonal 2 + |N| + i N(0, 0.3)."""
    a = (rng.standard_normal((ld, na)) + 1j * rng.standard_normal((ld, na))) / np.sqrt(2 * na)
    for i in range(na):
        a[i, i] = 2.0 + abs(rng.standard_normal()) + 0.3j * rng.standard_normal()
    a[na:] = -999.0
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product("LR", "UL", "NTC", "NU")))
def test_ztrsm_all_cases(blas, oracle, side, uplo, trans, diag):
    """ZTRSM: every side / uplo / trans (C conjugates) / diag; orders of 600 cross three 256-row
    leaves; 37 right-hand sides; complex alpha; padding rows of B untouched."""
    rng = np.random.default_rng(int.from_bytes((side + uplo + trans + diag).encode(), "little") % 2**32)
    m, n = (600, 37) if side == "L" else (37, 600)
    na = m if side == "L" else n
    lda, ldb = na + 2, m + 3
    a = _ctri(rng, na, lda, np.complex128)
    b = np.asfortranarray((rng.standard_normal((ldb, n)) + 1j * rng.standard_normal((ldb, n))))
    b[m:] = -999.0
    b0 = b.copy(order="F")
    ref = b.copy(order="F")
    alpha = 0.75 - 0.5j
    oracle.trsm(side, uplo, trans, diag, m, n, alpha, a, lda, ref, ldb)
    blas.trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
    err = np.abs(b[:m] - ref[:m])
    assert np.all(err <= 1e-11 * (1 + np.abs(ref[:m]))), float(err.max())
    assert np.array_equal(b[m:], b0[m:])


@pytest.mark.parametrize("side,uplo,trans", [("L", "L", "N"), ("R", "U", "C"), ("L", "U", "C"), ("R", "L", "T")])
def test_ctrsm(blas, oracle, side, uplo, trans):
    rng = np.random.default_rng(7)
    m, n = (300, 20) if side == "L" else (20, 300)
    na = m if side == "L" else n
    a = _ctri(rng, na, na, np.complex64)
    b = np.asfortranarray((rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64))
    ref = b.copy(order="F")
    oracle.trsm(side, uplo, trans, "N", m, n, 1.0 + 0.5j, a, na, ref, m)
    blas.trsm(side, uplo, trans, "N", m, n, 1.0 + 0.5j, a, na, b, m)
    assert np.all(np.abs(b - ref) <= 1e-3 * (1 + np.abs(ref)))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("uplo,trans", list(itertools.product("UL", "NTC")))
def test_complex_syrk(blas, oracle, dtype, uplo, trans):
    """ZSYRK / CSYRK (symmetric, no conjugation of the product; op = C conjugates op(A)):
    the triangle within c k u (|alpha| |A||A|^T + |beta| |C|), the other triangle and the
    padding bit-identical, beta = 0 clears NaN."""
    rng = np.random.default_rng(ord(uplo) + 3 * ord(trans))
    n, k = 150, 90
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = np.asfortranarray((rng.standard_normal((ra + 1, ca)) + 1j * rng.standard_normal((ra + 1, ca))).astype(dtype))
    u = 2.0 ** -53 if dtype == np.complex128 else 2.0 ** -24
    for alpha, beta in ((0.5 - 1.0j, 0.25 + 0.5j), (1.0 + 0.0j, 0.0)):
        c = np.asfortranarray((rng.standard_normal((n + 2, n)) + 1j * rng.standard_normal((n + 2, n))).astype(dtype))
        tri = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
        if beta == 0.0:
            c[:n][tri] = np.nan
        c0 = c.copy(order="F")
        ref = c.copy(order="F")
        oracle.syrk(uplo, trans, n, k, alpha, a, ra + 1, beta, ref, n + 2)
        blas.syrk(uplo, trans, n, k, alpha, a, ra + 1, beta, c, n + 2)
        A = np.abs(a[:ra, :ca].astype(np.complex128))
        A = A if trans == "N" else A.T
        bound = 8 * k * u * (abs(alpha) * (A @ A.T) + abs(beta) * np.nan_to_num(np.abs(c0[:n]))) + 1e-300
        got, want = c[:n].astype(np.complex128), ref[:n].astype(np.complex128)
        assert np.all(np.isfinite(got[tri]))
        assert np.all(np.abs(got - want)[tri] <= bound[tri]), float(np.abs(got - want)[tri].max())
        assert np.array_equal(c[:n][~tri], c0[:n][~tri], equal_nan=True), "the other triangle changed"
        assert np.array_equal(c[n:], c0[n:], equal_nan=True)


def test_complex_device_entry_points(blas, oracle):
    """zynum_blas_gpu_ztrsm_device / zsyrk_device on torch tensors, and cblas_ztrsm row-major."""
    import torch
    rng = np.random.default_rng(13)
    m, n = 300, 24
    a = _ctri(rng, m, m, np.complex128)
    b = np.asfortranarray(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")  # noqa: E731
    host = lambda t: np.asfortranarray(t.cpu().numpy().T)  # noqa: E731
    ref = b.copy(order="F")
    oracle.trsm("L", "L", "C", "N", m, n, 2.0 - 1.0j, a, m, ref, m)
    B = dev(b)
    blas.trsm_device_c("L", "L", "C", "N", m, n, 2.0 - 1.0j, dev(a), m, B, m)
    torch.cuda.synchronize()
    assert np.abs(host(B) - ref).max() <= 1e-11 * (1 + np.abs(ref).max())
    ref = np.zeros((n, n), complex, order="F")
    oracle.syrk("U", "T", n, m, 1.0, b, m, 0.0, ref, n)
    C = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    blas.syrk_device_c("U", "T", n, m, 1.0, dev(b), m, 0.0, C, n)
    torch.cuda.synchronize()
    got = host(C)
    up = np.triu(np.ones((n, n), bool))
    assert np.abs(got - ref)[up].max() <= 1e-12 * (1 + np.abs(ref).max())
    # row-major CBLAS: A (m x m, row-major) solves A X = 0.5 B
    A = np.tril(rng.standard_normal((m, m)) / np.sqrt(m) + 1j * rng.standard_normal((m, m)) / np.sqrt(m))
    A += np.diag(2.0 + np.abs(rng.standard_normal(m)))
    Bm = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    X = np.ascontiguousarray(Bm.copy())
    blas.cblas_trsm_c(blas.CblasRowMajor, blas.CblasLeft, blas.CblasLower, blas.CblasNoTrans, blas.CblasNonUnit,
                      m, n, 0.5, np.ascontiguousarray(A), m, X, n)
    assert np.abs(A @ X - 0.5 * Bm).max() <= 1e-10
