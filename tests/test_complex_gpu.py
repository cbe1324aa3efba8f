"""ZGEMM / CGEMM (expanded-real 4M and 3M forms) against the CPU oracle (GPU).

Follows the reference's complex tests (test/abi/fortran_compat_test.zig:783-970,
:1048-1074; cblas_compat_test.zig:423-460): every N/T/C combination, padded
leading dimensions, complex alpha / beta, NaN isolation, quick returns,
padding rows untouched.  Bound: |C - C_ref| <= c k u (|alpha| |A||B| + |beta| |C0|)
with |x| = |re| + |im| elementwise (c = 8 for 4M, 16 for 3M).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())
TRANS = ["N", "T", "C"]


def _op(x, t, r, c):
    if t == "N":
        return x[:r, :c]
    y = x[:c, :r].T
    return np.conj(y) if t == "C" else y


def _mag(x):
    return np.abs(x.real) + np.abs(x.imag)


def _case(blas, oracle, dtype, method, ta, tb, m, n, k, alpha, beta, rng, dmethod=0):
    u = 2.0 ** -53 if dtype == np.complex128 else 2.0 ** -24
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = ar + 3, br + 2, m + 1

    def mat(rows, cols, ld):
        x = (rng.uniform(-1, 1, (ld, max(cols, 1))) + 1j * rng.uniform(-1, 1, (ld, max(cols, 1)))).astype(dtype)
        x[rows:] = -999.0 - 999.0j
        return np.asfortranarray(x)

    a, b, c = mat(ar, ac, lda), mat(br, bc, ldb), mat(m, n, ldc)
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ref, ldc)
    old = blas.set_complex_method(method)
    oldd = blas.set_dgemm_method(dmethod)
    try:
        fn = blas.zgemm if dtype == np.complex128 else blas.cgemm
        fn(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    finally:
        blas.set_complex_method(old)
        blas.set_dgemm_method(oldd)
    A = _mag(_op(a, ta, m, k).astype(np.complex128))
    B = _mag(_op(b, tb, k, n).astype(np.complex128))
    cf = 8.0 if method == blas.COMPLEX_4M else 16.0
    bound = cf * max(k, 1) * u * (abs(alpha) * (A @ B) + abs(beta) * _mag(c0[:m, :n].astype(np.complex128))) + 1e-300
    err = np.abs(c[:m, :n].astype(np.complex128) - ref[:m, :n].astype(np.complex128))
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"


@pytest.mark.parametrize("method", [0, 1], ids=["4M", "3M"])
@pytest.mark.parametrize("ta", TRANS)
@pytest.mark.parametrize("tb", TRANS)
def test_zgemm_all_transposes(blas, oracle, method, ta, tb):
    rng = np.random.default_rng(hash((method, ta, tb)) % 2**32)
    _case(blas, oracle, np.complex128, method, ta, tb, 37, 29, 53, 0.75 - 0.25j, -0.5 + 0.125j, rng)


@pytest.mark.parametrize("method", [0, 1], ids=["4M", "3M"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "T"), ("T", "C")])
def test_cgemm(blas, oracle, method, ta, tb):
    rng = np.random.default_rng(4)
    _case(blas, oracle, np.complex64, method, ta, tb, 130, 70, 150, 0.75 - 0.25j, -0.5 + 0.25j, rng)


def test_zgemm_larger_and_ozaki(blas, oracle):
    rng = np.random.default_rng(5)
    _case(blas, oracle, np.complex128, 0, "N", "C", 300, 260, 200, 1.0, 0.0, rng)
    # the real GEMM of the expanded form can run on the Ozaki INT8 method
    _case(blas, oracle, np.complex128, 0, "C", "N", 200, 300, 256, 1.5 + 0.5j, 0.25, rng, dmethod=1)


def test_zgemm_quick_returns_and_nan_isolation(blas, oracle):
    g = GOLDEN["zgemm_nan_isolation"]
    a = np.array([[complex(*g["a"])]], np.complex128, order="F")
    b = np.array([[complex(*g["b"])]], np.complex128, order="F")
    c = np.array([[complex(np.nan, np.nan)]], np.complex128, order="F")
    blas.zgemm("N", "N", 1, 1, 1, 1.0, a, 1, b, 1, 0.0, c, 1)
    assert c[0, 0] == complex(*g["c_beta0"])
    a[:] = complex(np.nan, np.nan)
    b[:] = complex(np.nan, np.nan)
    c = np.array([[complex(4, 3)]], np.complex128, order="F")
    blas.zgemm("N", "N", 1, 1, 1, 0.0, a, 1, b, 1, complex(2, -1), c, 1)
    assert c[0, 0] == complex(*g["c_alpha0"])
    rng = np.random.default_rng(6)
    _case(blas, oracle, np.complex128, 0, "N", "N", 5, 7, 0, 1.0, 2.0 - 1.0j, rng)  # k == 0


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "C"), ("T", "N"), ("C", "C")])
def test_cblas_zgemm_row_major(blas, oracle, ta, tb):
    """Row-major CBLAS: C (m x n, row-major) = op(A) op(B) computed as the column-major transpose."""
    rng = np.random.default_rng(8)
    m, n, k = 17, 19, 41
    cmap = {"N": blas.CblasNoTrans, "T": blas.CblasTrans, "C": blas.CblasConjTrans}
    A = (rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)) + 1j * rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)))
    B = (rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)) + 1j * rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
    C = rng.uniform(-1, 1, (m, n)) + 1j * rng.uniform(-1, 1, (m, n))
    opA = A if ta == "N" else (A.T if ta == "T" else A.conj().T)
    opB = B if tb == "N" else (B.T if tb == "T" else B.conj().T)
    alpha, beta = 0.75 - 0.25j, -0.5 + 0.125j
    want = alpha * (opA @ opB) + beta * C
    a = np.ascontiguousarray(A)
    b = np.ascontiguousarray(B)
    c = np.ascontiguousarray(C)
    blas.cblas_zgemm(blas.CblasRowMajor, cmap[ta], cmap[tb], m, n, k, alpha, a, a.shape[1], b, b.shape[1], beta, c, n)
    assert np.abs(c - want).max() <= 1e-12 * k
