"""Pins the CPU oracle against the reference's own known-answer tests and
against exact rational arithmetic (CPU only, no GPU)."""
from __future__ import annotations

import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from conftest import padded

GOLDEN = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())


def _col_major(vals, rows, cols):
    return np.asfortranarray(np.array(vals, dtype=np.float64).reshape(cols, rows).T)


def test_dgemm_known_answer_column_major(oracle):
    g = GOLDEN["dgemm_column_major_nn"]
    a = _col_major(g["a"], 2, 3)
    b = _col_major(g["b"], 3, 2)
    c = np.zeros((2, 2), order="F")
    oracle.gemm("N", "N", 2, 2, 3, 1.0, a, 2, b, 3, 0.0, c, 2)
    assert list(c.T.ravel()) == g["c"]


def test_dgemm_nan_isolation(oracle):
    g = GOLDEN["gemm_nan_isolation"]
    a = _col_major(g["a"], 2, 2)
    b = _col_major(g["b"], 2, 2)
    c = np.full((2, 2), np.nan, order="F")
    oracle.gemm("N", "N", 2, 2, 2, 1.0, a, 2, b, 2, 0.0, c, 2)
    assert list(c.T.ravel()) == g["c_beta0"]
    a[:] = np.nan
    b[:] = np.nan
    c = _col_major([1, 2, 3, 4], 2, 2)
    oracle.gemm("N", "N", 2, 2, 2, 0.0, a, 2, b, 2, 2.0, c, 2)
    assert list(c.T.ravel()) == g["c_alpha0"]


def test_zgemm_known_answers(oracle):
    g = GOLDEN["zgemm_nan_isolation"]
    a = np.array([[complex(*g["a"])]], np.complex128, order="F")
    b = np.array([[complex(*g["b"])]], np.complex128, order="F")
    c = np.array([[complex(np.nan, np.nan)]], np.complex128, order="F")
    oracle.gemm("N", "N", 1, 1, 1, 1.0, a, 1, b, 1, 0.0, c, 1)
    assert c[0, 0] == complex(*g["c_beta0"])
    a[:] = complex(np.nan, np.nan)
    b[:] = complex(np.nan, np.nan)
    c = np.array([[complex(4, 3)]], np.complex128, order="F")
    oracle.gemm("N", "N", 1, 1, 1, 0.0, a, 1, b, 1, complex(2, -1), c, 1)
    assert c[0, 0] == complex(*g["c_alpha0"])


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_dgemm_exact_rationals(oracle, ta, tb):
    """sampleValue fills are k/9 rationals: compare against exact Fraction arithmetic."""
    m, n, k = 7, 5, 11
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 2
    ldc = m + 4
    a = padded(m if ta == "N" else k, k if ta == "N" else m, lda, 1, np.float64, -999.0)
    b = padded(k if tb == "N" else n, n if tb == "N" else k, ldb, 5, np.float64, -999.0)
    c = padded(m, n, ldc, 9, np.float64, -999.0)
    c0 = c.copy(order="F")
    alpha, beta = -0.5, 2.0
    oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    for j in range(n):
        for i in range(m):
            s = Fraction(0)
            for p in range(k):
                av = a[i, p] if ta == "N" else a[p, i]
                bv = b[p, j] if tb == "N" else b[j, p]
                s += Fraction(av) * Fraction(bv)
            exact = Fraction(alpha) * s + Fraction(beta) * Fraction(c0[i, j])
            assert abs(c[i, j] - float(exact)) <= 1e-13 * (1 + abs(float(exact)))
    # padding rows untouched
    assert np.array_equal(c[m:, :], c0[m:, :])


def test_ddgemm_is_exact_on_cancellation(oracle):
    """Double-double recovers a sum that cancels catastrophically in FP64."""
    a = np.asfortranarray(np.array([[1e16, 1.0, -1e16]]))
    b = np.asfortranarray(np.array([[1.0], [1.0], [1.0]]))
    hi, lo = oracle.ddgemm("N", "N", 1, 1, 3, a, 1, b, 3)
    assert hi[0, 0] + lo[0, 0] == 1.0
    c = np.zeros((1, 1), order="F")
    oracle.gemm("N", "N", 1, 1, 3, 1.0, a, 1, b, 3, 0.0, c, 1)
    assert c[0, 0] == 0.0  # plain FP64 loses it, as the reference's portable loop would


def test_ddgemm_sampled_matches_full(oracle):
    rng = np.random.default_rng(3)
    m, n, k = 9, 7, 33
    a = np.asfortranarray(rng.standard_normal((m, k)))
    b = np.asfortranarray(rng.standard_normal((k, n)))
    hi, lo = oracle.ddgemm("N", "N", m, n, k, a, m, b, k)
    rows = np.array([0, 3, 8, 5]); cols = np.array([0, 6, 2, 4])
    shi, slo, _ = oracle.ddgemm_sampled("N", "N", k, a, m, b, k, rows, cols)
    assert np.array_equal(shi, hi[rows, cols]) and np.array_equal(slo, lo[rows, cols])


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_trsm_solves(oracle, side, uplo, trans, diag):
    rng = np.random.default_rng(11)
    m, n = 6, 5
    na = m if side == "L" else n
    lda, ldb = na + 2, m + 3
    a = np.asfortranarray(rng.standard_normal((lda, na)))
    for i in range(na):
        a[i, i] = 2.0 + abs(a[i, i])
    b = np.asfortranarray(rng.standard_normal((ldb, n)))
    b0 = b.copy(order="F")
    alpha = 0.75
    oracle.trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
    T = np.triu(a[:na, :na]) if uplo == "U" else np.tril(a[:na, :na])
    if diag == "U":
        np.fill_diagonal(T, 1.0)
    opT = T if trans == "N" else T.T
    X = b[:m, :n]
    lhs = opT @ X if side == "L" else X @ opT
    np.testing.assert_allclose(lhs, alpha * b0[:m, :n], rtol=1e-12, atol=1e-12)
    assert np.array_equal(b[m:, :], b0[m:, :])


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_syrk_triangle(oracle, uplo, trans):
    rng = np.random.default_rng(5)
    n, k = 7, 9
    lda = (n if trans == "N" else k) + 1
    a = np.asfortranarray(rng.standard_normal((lda, k if trans == "N" else n)))
    ldc = n + 2
    c = np.asfortranarray(rng.standard_normal((ldc, n)))
    c0 = c.copy(order="F")
    oracle.syrk(uplo, trans, n, k, 1.5, a, lda, 0.5, c, ldc)
    opA = a[:n, :k] if trans == "N" else a[:k, :n].T
    full = 1.5 * opA @ opA.T + 0.5 * c0[:n, :n]
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    np.testing.assert_allclose(c[:n, :n][mask], full[mask], rtol=1e-12, atol=1e-12)
    assert np.array_equal(c[:n, :n][~mask], c0[:n, :n][~mask])


def _cx(rng, shape, dtype=np.complex128):
    return np.asfortranarray((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype))


def _op(x, trans):
    return x if trans == "N" else (x.T if trans == "T" else x.conj().T)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("herm", [False, True])
def test_complex_symm_hemm(oracle, side, uplo, herm):
    """zsymm / zhemm: the stored triangle mirrored (conjugated, diagonal real for HEMM)."""
    rng = np.random.default_rng(21)
    m, n = 6, 5
    na = m if side == "L" else n
    a, b = _cx(rng, (na + 1, na)), _cx(rng, (m + 2, n))
    c = _cx(rng, (m + 1, n))
    c0 = c.copy(order="F")
    al, be = 0.5 - 0.25j, 1.5 + 0.5j
    oracle.symm(side, uplo, m, n, al, a, na + 1, b, m + 2, be, c, m + 1, herm=herm)
    T = np.triu(a[:na, :na]) if uplo == "U" else np.tril(a[:na, :na])
    strict = T - np.diag(np.diag(T))
    S = T + (strict.conj().T if herm else strict.T)
    if herm:
        np.fill_diagonal(S, np.diag(S).real)
    B = b[:m, :n]
    ref = al * (S @ B if side == "L" else B @ S) + be * c0[:m, :n]
    np.testing.assert_allclose(c[:m, :n], ref, rtol=1e-12, atol=1e-12)
    assert np.array_equal(c[m:, :], c0[m:, :])


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_complex_trmm(oracle, side, uplo, trans, diag):
    rng = np.random.default_rng(22)
    m, n = 6, 4
    na = m if side == "L" else n
    a, b = _cx(rng, (na + 1, na)), _cx(rng, (m + 1, n))
    b0 = b.copy(order="F")
    al = 0.75 + 0.5j
    oracle.trmm(side, uplo, trans, diag, m, n, al, a, na + 1, b, m + 1)
    T = np.triu(a[:na, :na]) if uplo == "U" else np.tril(a[:na, :na])
    if diag == "U":
        np.fill_diagonal(T, 1.0)
    X = b0[:m, :n]
    ref = al * (_op(T, trans) @ X if side == "L" else X @ _op(T, trans))
    np.testing.assert_allclose(b[:m, :n], ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
def test_complex_herk(oracle, uplo, trans):
    """zherk: op(A) op(A)^H on the triangle, diagonal imaginary part zeroed (op = T gives
    A^T conj(A))."""
    rng = np.random.default_rng(23)
    n, k = 6, 7
    rows, cols = (n, k) if trans == "N" else (k, n)
    a, c = _cx(rng, (rows + 1, cols)), _cx(rng, (n + 2, n))
    c0 = c.copy(order="F")
    oracle.herk(uplo, trans, n, k, 1.25, a, rows + 1, 0.5, c, n + 2)
    opA = _op(a[:rows, :cols], trans)
    full = 1.25 * opA @ opA.conj().T + 0.5 * c0[:n, :n]
    np.fill_diagonal(full, np.diag(full).real)
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    np.testing.assert_allclose(c[:n, :n][mask], full[mask], rtol=1e-12, atol=1e-12)
    assert np.array_equal(c[:n, :n][~mask], c0[:n, :n][~mask])


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("herm", [False, True])
def test_complex_syr2k_her2k(oracle, uplo, trans, herm):
    rng = np.random.default_rng(24)
    n, k = 5, 6
    rows, cols = (n, k) if trans == "N" else (k, n)
    a, b, c = _cx(rng, (rows, cols)), _cx(rng, (rows, cols)), _cx(rng, (n + 1, n))
    c0 = c.copy(order="F")
    al = 0.5 + 0.75j
    be = 0.25 if herm else 0.25 - 0.5j
    oracle.syr2k(uplo, trans, n, k, al, a, rows, b, rows, be, c, n + 1, herm=herm)
    oa, ob = _op(a, trans), _op(b, trans)
    if herm:
        full = al * oa @ ob.conj().T + np.conj(al) * ob @ oa.conj().T + be * c0[:n, :n]
        np.fill_diagonal(full, np.diag(full).real)
    else:
        full = al * (oa @ ob.T + ob @ oa.T) + be * c0[:n, :n]
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    np.testing.assert_allclose(c[:n, :n][mask], full[mask], rtol=1e-12, atol=1e-12)
    assert np.array_equal(c[:n, :n][~mask], c0[:n, :n][~mask])


def _lv(vals, dtype=np.float64):
    """2 x 2 column-major array from the reference's flat lists ([re, im] pairs for complex)."""
    if isinstance(vals[0], list):
        vals = [complex(re, im) for re, im in vals]
        dtype = np.complex128
    return np.asfortranarray(np.array(vals, dtype=dtype).reshape(2, 2).T)


def test_level3_known_answers(oracle):
    """The oracle's SYMM / HEMM / SYRK / HERK / SYR2K / HER2K / TRMM / TRSM restatements reproduce
    the reference's own 2 x 2 known answers (side L, uplo U, trans N, alpha 1, beta 0)."""
    g = GOLDEN["level3_known_answers"]
    c = np.zeros((2, 2), order="F")
    oracle.symm("L", "U", 2, 2, 1.0, _lv(g["dsymm"]["a"]), 2, _lv(g["dsymm"]["b"]), 2, 0.0, c, 2)
    assert np.array_equal(c, _lv(g["dsymm"]["c"]))
    c = np.zeros((2, 2), np.complex128, order="F")
    oracle.symm("L", "U", 2, 2, 1.0, _lv(g["zhemm"]["a"]), 2, _lv(g["zhemm"]["b"]), 2, 0.0, c, 2, herm=True)
    assert np.array_equal(c, _lv(g["zhemm"]["c"]))
    c = _lv(g["dsyrk"]["c0"])
    oracle.syrk("U", "N", 2, 2, 1.0, _lv(g["dsyrk"]["a"]), 2, 0.0, c, 2)
    assert np.array_equal(c, _lv(g["dsyrk"]["c"]))
    c = _lv(g["zherk"]["c0"])
    oracle.herk("U", "N", 2, 2, 1.0, _lv(g["zherk"]["a"]), 2, 0.0, c, 2)
    assert np.array_equal(c, _lv(g["zherk"]["c"]))
    c = _lv(g["dsyr2k"]["c0"])
    oracle.syr2k("U", "N", 2, 2, 1.0, _lv(g["dsyr2k"]["a"]), 2, _lv(g["dsyr2k"]["b"]), 2, 0.0, c, 2)
    assert np.array_equal(c, _lv(g["dsyr2k"]["c"]))
    c = _lv(g["zher2k"]["c0"])
    oracle.syr2k("U", "N", 2, 2, 1.0, _lv(g["zher2k"]["a"]), 2, _lv(g["zher2k"]["b"]), 2, 0.0, c, 2, herm=True)
    assert np.array_equal(c, _lv(g["zher2k"]["c"]))
    b = _lv(g["dtrmm"]["b"])
    oracle.trmm("L", "U", "N", "N", 2, 2, 1.0, _lv(g["dtrmm"]["a"]), 2, b, 2)
    assert np.array_equal(b, _lv(g["dtrmm"]["b_out"]))
    b = _lv(g["dtrsm"]["b"])
    oracle.trsm("L", "U", "N", "N", 2, 2, 1.0, _lv(g["dtrsm"]["a"]), 2, b, 2)
    assert np.array_equal(b, _lv(g["dtrsm"]["b_out"]))


def test_golden_file_is_current():
    """tests/golden/known_answers.json is what tests/golden/make_golden.py writes."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", Path(__file__).parent / "golden" / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert json.loads(json.dumps(mod.KNOWN)) == GOLDEN, "rerun tests/golden/make_golden.py"
