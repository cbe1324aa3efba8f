"""Ozaki-emulated DGEMM and 3xBF16 SGEMM against the double-double oracle (GPU).

Ozaki bound (from the splitting, see zynum_b200/csrc/ozaki.cu): with s 7-bit
digits per operand and row / column exponents e_i, f_j (2^e_i <= 2 max_p |a_ip|),
  |C - C_exact| <= |alpha| (s + 2) k 2^{-7 s} 2^{e_i + f_j} + 8 u (|alpha| |A||B| + |beta| |C0|).
3xBF16 bound: |C - C_exact| <= |alpha| (2^-15 + 2 k 2^-24) |A||B| + 2^-22 |beta| |C0|.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
U64 = 2.0 ** -53


def _op(x, t, r, c):
    return x[:r, :c] if t == "N" else x[:c, :r].T


def _exact(oracle, ta, tb, m, n, k, a, lda, b, ldb):
    hi, lo = oracle.ddgemm(ta, tb, m, n, k, a, lda, b, ldb)
    return hi, lo


def _ozaki_case(blas, oracle, ta, tb, m, n, k, lda, ldb, ldc, alpha, beta, slices, rng, phi=0.0):
    def mat(rows, cols, ld):
        x = rng.uniform(-1, 1, (ld, cols))
        if phi:
            x *= 10.0 ** rng.uniform(-phi, phi, (ld, cols))
        x[rows:] = -999.0
        return np.asfortranarray(x)

    a = mat(m if ta == "N" else k, k if ta == "N" else m, lda)
    b = mat(k if tb == "N" else n, n if tb == "N" else k, ldb)
    c = mat(m, n, ldc)
    c0 = c.copy(order="F")
    blas.set_dgemm_method(blas.METHOD_OZAKI)
    old = blas.set_ozaki_slices(slices)
    try:
        blas.dgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    finally:
        blas.set_ozaki_slices(old)
        blas.set_dgemm_method(blas.METHOD_NATIVE)
    hi, lo = _exact(oracle, ta, tb, m, n, k, a, lda, b, ldb)
    exact = alpha * (hi + lo) + beta * c0[:m, :n]
    A, B = _op(a, ta, m, k), _op(b, tb, k, n)
    ea = np.frexp(np.abs(A).max(axis=1))[1].astype(float)
    fb = np.frexp(np.abs(B).max(axis=0))[1].astype(float)
    scale = np.exp2(ea[:, None] + fb[None, :])
    bound = abs(alpha) * (slices + 2) * k * 2.0 ** (-7 * slices) * scale \
        + 8 * U64 * (abs(alpha) * (np.abs(A) @ np.abs(B)) + abs(beta) * np.abs(c0[:m, :n]))
    err = np.abs(c[:m, :n] - exact)
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"
    return err, exact


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_ozaki_small_all_transposes(blas, oracle, ta, tb):
    rng = np.random.default_rng(100)
    _ozaki_case(blas, oracle, ta, tb, 200, 300, 150, 211, 309, 203, 1.5, 0.5, 7, rng)


@pytest.mark.parametrize("slices", [3, 5, 7, 9])
def test_ozaki_slice_counts(blas, oracle, slices):
    rng = np.random.default_rng(slices)
    _ozaki_case(blas, oracle, "N", "N", 130, 257, 300, 130, 300, 131, -0.75, 0.0, slices, rng)


def test_ozaki_tails_and_edges(blas, oracle):
    rng = np.random.default_rng(7)
    for (m, n, k) in [(1, 1, 1), (1, 257, 131), (257, 1, 131), (129, 255, 129), (5, 7, 3)]:
        _ozaki_case(blas, oracle, "N", "T", m, n, k, m + 2, n + 3, m + 1, 1.0, -0.25, 7, rng)


def test_ozaki_k_segments(blas, oracle):
    """K beyond one INT32-safe segment (7 slices: 148 chunks of 128) accumulates per segment."""
    rng = np.random.default_rng(9)
    _ozaki_case(blas, oracle, "N", "N", 64, 96, 20000, 64, 20000, 64, 1.0, 1.0, 7, rng)


@pytest.mark.parametrize("phi", [4.0, 8.0])
def test_ozaki_wide_dynamic_range(blas, oracle, phi):
    rng = np.random.default_rng(int(phi))
    _ozaki_case(blas, oracle, "T", "N", 96, 80, 512, 512, 512, 96, 1.0, 0.0, 8, rng, phi=phi)


def test_ozaki_config1_matches_native_error(blas, oracle):
    """1024^3, ld 1031, alpha 1.5, beta 0.5: Ozaki's max error is no worse than native FP64's."""
    rng = np.random.default_rng(20260101)
    m = n = k = 1024
    ld = 1031
    a = np.asfortranarray(rng.uniform(-1, 1, (ld, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (ld, n)))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (ld, n)))
    hi, lo = oracle.ddgemm("N", "N", m, n, k, a, ld, b, ld)
    exact = 1.5 * (hi + lo) + 0.5 * c0[:m]
    errs = {}
    for method in (blas.METHOD_NATIVE, blas.METHOD_OZAKI):
        c = c0.copy(order="F")
        blas.set_dgemm_method(method)
        blas.dgemm("N", "N", m, n, k, 1.5, a, ld, b, ld, 0.5, c, ld)
        errs[method] = np.abs(c[:m] - exact).max()
    blas.set_dgemm_method(blas.METHOD_NATIVE)
    assert errs[blas.METHOD_OZAKI] <= errs[blas.METHOD_NATIVE], errs


@pytest.mark.parametrize("phi", [0.0, 2.0, 4.0, 8.0])
def test_ozaki_auto_slices_match_native_error(blas, oracle, phi):
    """Automatic slice count on u * 10^e data (u ~ U[-1,1], e ~ U[-phi,phi]), 2048^2 x 2048:
    the max relative error on 4096 sampled entries of C (double-double oracle) is no worse
    than native FP64's on the same entries."""
    rng = np.random.default_rng(int(phi) + 77)
    n = 2048
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-phi, phi, (n, n)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-phi, phi, (n, n)))
    rows = rng.integers(0, n, 4096)
    cols = rng.integers(0, n, 4096)
    hi, lo, _ = oracle.ddgemm_sampled("N", "N", n, a, n, b, n, rows, cols)
    exact = hi + lo
    errs = {}
    for method in (blas.METHOD_NATIVE, blas.METHOD_OZAKI):
        c = np.zeros((n, n), order="F")
        blas.set_dgemm_method(method)
        old = blas.set_ozaki_slices(0)
        try:
            blas.dgemm("N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c, n)
        finally:
            blas.set_ozaki_slices(old)
            blas.set_dgemm_method(blas.METHOD_NATIVE)
        errs[method] = float((np.abs(c[rows, cols] - exact) / np.abs(exact)).max())
    assert errs[blas.METHOD_OZAKI] <= errs[blas.METHOD_NATIVE], errs


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T"), ("N", "T")])
def test_sgemm_bf16x3(blas, oracle, ta, tb):
    rng = np.random.default_rng(3)
    m, n, k = 257, 300, 333
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 1
    ldc = m + 2
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, k if ta == "N" else m)).astype(np.float32))
    b = np.asfortranarray(rng.uniform(-1, 1, (ldb, n if tb == "N" else k)).astype(np.float32))
    c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(np.float32))
    c0 = c.copy(order="F")
    blas.set_sgemm_method(blas.SMETHOD_BF16X3)
    try:
        blas.sgemm(ta, tb, m, n, k, 1.25, a, lda, b, ldb, -0.5, c, ldc)
    finally:
        blas.set_sgemm_method(blas.SMETHOD_NATIVE)
    A = _op(a.astype(np.float64), ta, m, k)
    B = _op(b.astype(np.float64), tb, k, n)
    exact = 1.25 * (A @ B) - 0.5 * c0[:m, :n].astype(np.float64)
    bound = 1.25 * (2.0 ** -15 + 2 * k * 2.0 ** -24) * (np.abs(A) @ np.abs(B)) + 2.0 ** -22 * np.abs(c0[:m, :n])
    err = np.abs(c[:m, :n] - exact)
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(c[m:], c0[m:])
