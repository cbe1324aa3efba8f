"""SGEMM through INT8 CRT residues (method 3) against FP64 products of the FP32 data (GPU).

Every FP32 entry widens exactly to FP64.  Each row of op(A) and column of op(B)
is scaled by a power of two so that its 2-norm stays below 2^P, with P >= 25 +
log2(sqrt(k)) chosen through the modulus count, so entries near the top of a
row keep their whole significand; the modular products are exact INT32 sums,
the reconstruction is exact, and alpha x + beta C is formed in FP64 and rounded
once to FP32.  The tests hold the result to the componentwise bound native
FP32 GEMM is held to, 4 k u32 (|alpha| |A||B| + |beta| |C0|), and to an error
no larger than the native FFMA kernel's on the same data.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24


def _op(x, t, r, c):
    return x[:r, :c] if t == "N" else x[:c, :r].T


def _run(blas, method, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    old = blas.set_sgemm_method(method)
    try:
        blas.sgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    finally:
        blas.set_sgemm_method(old)


def _case(blas, ta, tb, m, n, k, pad, alpha, beta, rng, lo=-1.0, row_scale=0.0, compare_native=True):
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = ar + pad, br + pad + 1, m + 2
    a = rng.uniform(lo, 1, (lda, ac))
    b = rng.uniform(lo, 1, (ldb, bc))
    if row_scale:
        # whole rows of op(A) / columns of op(B) scaled over 2^(+-row_scale)
        sa = np.exp2(np.round(rng.uniform(-row_scale, row_scale, m)))
        sb = np.exp2(np.round(rng.uniform(-row_scale, row_scale, n)))
        if ta == "N":
            a[:m] *= sa[:, None]
        else:
            a[:, :m] *= sa[None, :]
        if tb == "N":
            b[:, :n] *= sb[None, :]
        else:
            b[:n] *= sb[:, None]
    a = np.asfortranarray(a.astype(np.float32))
    b = np.asfortranarray(b.astype(np.float32))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(np.float32))
    c0[m:] = -999.0
    A = _op(a.astype(np.float64), ta, m, k)
    B = _op(b.astype(np.float64), tb, k, n)
    exact = alpha * (A @ B) + beta * c0[:m, :n].astype(np.float64)
    ab = np.abs(A) @ np.abs(B)
    bound = 4 * k * U32 * (abs(alpha) * ab + abs(beta) * np.abs(c0[:m, :n])) + 1e-300
    out = c0.copy(order="F")
    _run(blas, blas.SMETHOD_OZAKI, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, out, ldc)
    err = np.abs(out[:m, :n] - exact)
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(out[m:], c0[m:]), "padding rows of C were written"
    if compare_native:
        nat = c0.copy(order="F")
        _run(blas, blas.SMETHOD_NATIVE, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, nat, ldc)
        scale = abs(alpha) * ab + abs(beta) * np.abs(c0[:m, :n]) + 1e-300
        e_oz = float((err / scale).max())
        e_nat = float((np.abs(nat[:m, :n] - exact) / scale).max())
        assert e_oz <= e_nat, (e_oz, e_nat)
    return err


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_sgemm_ozaki_fp32_accurate(blas, ta, tb):
    _case(blas, ta, tb, 300, 257, 1500, 3, 1.25, -0.5, np.random.default_rng(4))


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 300, 7), (300, 1, 129), (255, 257, 128), (256, 256, 256),
                                   (700, 520, 4097), (1030, 300, 65)], ids=lambda s: "x".join(map(str, s)))
def test_sgemm_ozaki_shapes(blas, shape):
    """One-CTA and CTA-pair product kernels, ragged tails, K past 4096 (one more modulus)."""
    m, n, k = shape
    _case(blas, "N", "T", m, n, k, 1, -0.75, 0.5, np.random.default_rng(m + n + k), compare_native=False)


def test_sgemm_ozaki_positive_data_long_k(blas):
    """U[0, 1) data at k = 8192: |C| = |A||B|, so the error is one FP32 rounding of the result."""
    rng = np.random.default_rng(8)
    err = _case(blas, "N", "N", 256, 256, 8192, 0, 1.0, 0.0, rng, lo=0.0)
    assert err.max() > 0.0


@pytest.mark.parametrize("scale", [20.0, 60.0])
def test_sgemm_ozaki_row_and_column_scales(blas, scale):
    """Rows of op(A) and columns of op(B) spread over 2^(+-scale): each gets its own power of two."""
    _case(blas, "T", "N", 384, 320, 640, 2, 1.0, 1.0, np.random.default_rng(int(scale)), row_scale=scale,
          compare_native=False)


def test_sgemm_ozaki_long_k_panels(blas):
    """K beyond one modular product's INT32 bound (130816): two K panels, the second added to C."""
    _case(blas, "N", "N", 64, 48, 140000, 0, 1.0, -1.0, np.random.default_rng(12), compare_native=False)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_sgemm_ozaki_nonfinite_entries_match_reference_loop(blas, oracle, ta, tb):
    """Inf / NaN in single entries of op(A), op(B) and C: the same entries are NaN, +Inf and
    -Inf as in the reference's FP32 loop (gemm.zig:1422-1429, the oracle); finite entries
    meet the componentwise bound."""
    rng = np.random.default_rng(43)
    m, n, k, ld = 600, 520, 384, 611
    a = np.asfortranarray(rng.uniform(-1, 1, (ld, k if ta == "N" else m)).astype(np.float32))
    b = np.asfortranarray(rng.uniform(-1, 1, (ld, n if tb == "N" else k)).astype(np.float32))
    c = np.asfortranarray(rng.uniform(-1, 1, (ld, n)).astype(np.float32))

    def put_a(i, p, v):
        a[(i, p) if ta == "N" else (p, i)] = v

    def put_b(p, j, v):
        b[(p, j) if tb == "N" else (j, p)] = v

    put_a(5, 17, np.inf)
    put_b(17, 40, 0.0)
    put_a(9, 100, -np.inf)
    put_b(100, 41, np.nan)
    put_a(500, 3, np.nan)
    put_b(64, 300, np.inf)
    put_a(9, 64, np.inf)
    c[11, 12] = -np.inf
    c[5, 13] = np.nan
    c0 = c.copy(order="F")
    alpha, beta = 1.5, 0.5
    _run(blas, blas.SMETHOD_OZAKI, ta, tb, m, n, k, alpha, a, ld, b, ld, beta, c, ld)
    ref = c0.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, alpha, a, ld, b, ld, beta, ref, ld)
    got, want = c[:m, :n], ref[:m, :n]
    assert np.array_equal(np.isnan(got), np.isnan(want)), "NaN entries differ"
    assert np.array_equal(np.isposinf(got), np.isposinf(want)), "+Inf entries differ"
    assert np.array_equal(np.isneginf(got), np.isneginf(want)), "-Inf entries differ"
    assert np.isnan(want).sum() > n and np.isinf(want).sum() > n
    fin = np.isfinite(want)
    A = _op(a.astype(np.float64), ta, m, k)
    B = _op(b.astype(np.float64), tb, k, n)
    with np.errstate(invalid="ignore"):
        exact = alpha * (np.nan_to_num(A, nan=0.0, posinf=0.0, neginf=0.0) @ np.nan_to_num(B, nan=0.0, posinf=0.0,
                                                                                         neginf=0.0))
    exact += beta * np.nan_to_num(c0[:m, :n].astype(np.float64), nan=0.0, posinf=0.0, neginf=0.0)
    ab = np.abs(np.nan_to_num(A, nan=0.0, posinf=0.0, neginf=0.0)) @ np.abs(np.nan_to_num(B, nan=0.0, posinf=0.0,
                                                                                         neginf=0.0))
    bound = 4 * k * U32 * (alpha * ab + beta * np.abs(np.nan_to_num(c0[:m, :n].astype(np.float64))))
    err = np.abs(got[fin] - exact[fin])
    assert np.all(err <= bound[fin]), float((err / bound[fin]).max())
    assert np.array_equal(c[m:], c0[m:])


@pytest.mark.parametrize("method", [0, 1], ids=["4M", "3M"])
def test_cgemm_on_int8_real_products(blas, method):
    """CGEMM whose real products run through the INT8 route (its scratch sizing included)."""
    rng = np.random.default_rng(21 + method)
    m, n, k = 200, 150, 700
    a = np.asfortranarray((rng.uniform(-1, 1, (m, k)) + 1j * rng.uniform(-1, 1, (m, k))).astype(np.complex64))
    b = np.asfortranarray((rng.uniform(-1, 1, (k, n)) + 1j * rng.uniform(-1, 1, (k, n))).astype(np.complex64))
    c = np.asfortranarray(np.zeros((m, n), np.complex64))
    old_c = blas.set_complex_method(method)
    old_s = blas.set_sgemm_method(blas.SMETHOD_OZAKI)
    try:
        blas.cgemm("N", "N", m, n, k, 1.0 + 0.5j, a, m, b, k, 0.0, c, m)
    finally:
        blas.set_sgemm_method(old_s)
        blas.set_complex_method(old_c)
    A, B = a.astype(np.complex128), b.astype(np.complex128)
    exact = (1.0 + 0.5j) * (A @ B)
    bound = 8 * k * U32 * 1.2 * (np.abs(A) @ np.abs(B))
    assert np.all(np.abs(c - exact) <= bound)
