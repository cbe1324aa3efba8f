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


# ----------------------------------------------------------- CRT scheme
CRT_MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191]


def _crt_bits(nmod):
    lm = sum(np.log2(CRT_MODULI[:nmod]))
    return min(62, int(np.floor((lm - 2.0) / 2.0)))


def _crt_case(blas, oracle, ta, tb, m, n, k, lda, ldb, ldc, alpha, beta, rng, nmod=0, phi=0.0, mat=None):
    """CRT-scheme DGEMM against the double-double oracle.  Bound: with row scale
    2^{a_i} <= 2^P / H_i (H_i = sqrt(max_p |a_ip| sum_p |a_ip|), likewise for columns of op(B)),
    |C - C_exact| <= |alpha| (2^-P H_i sum_p |b_pj| + 2^-P H_j sum_p |a_ip| + k 2^-2P 4 H_i H_j)
                     + 4 u (|alpha| |A||B| + |beta| |C0|)."""
    if mat is None:
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
    old_s = blas.set_ozaki_scheme(blas.OZAKI_CRT)
    old_m = blas.set_ozaki_moduli(nmod)
    try:
        from zynum_b200 import ozaki_info
        info = ozaki_info(m, n, k)
        assert info["scheme"] == "crt" and info["moduli"] == (nmod or 16), info
        blas.dgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    finally:
        blas.set_ozaki_moduli(old_m)
        blas.set_ozaki_scheme(old_s)
        blas.set_dgemm_method(blas.METHOD_NATIVE)
    hi, lo = oracle.ddgemm(ta, tb, m, n, k, a, lda, b, ldb)
    exact = alpha * (hi + lo) + beta * c0[:m, :n]
    A, B = _op(a, ta, m, k), _op(b, tb, k, n)
    P = _crt_bits(nmod or 16)
    ha = np.sqrt(np.abs(A).max(axis=1) * np.abs(A).sum(axis=1))
    hb = np.sqrt(np.abs(B).max(axis=0) * np.abs(B).sum(axis=0))
    sa, sb = np.abs(A).sum(axis=1), np.abs(B).sum(axis=0)
    bound = abs(alpha) * 2.0 ** -P * (ha[:, None] * sb[None, :] + sa[:, None] * hb[None, :]
                                      + k * 4 * 2.0 ** -P * ha[:, None] * hb[None, :]) \
        + 4 * U64 * (abs(alpha) * (np.abs(A) @ np.abs(B)) + abs(beta) * np.abs(c0[:m, :n]))
    err = np.abs(c[:m, :n] - exact)
    assert np.all(err <= bound), float((err / bound).max())
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"
    return err, exact


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_crt_small_all_transposes(blas, oracle, ta, tb):
    rng = np.random.default_rng(300)
    _crt_case(blas, oracle, ta, tb, 200, 300, 150, 211, 309, 203, 1.5, 0.5, rng)


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 300, 7), (300, 1, 129), (255, 257, 128), (256, 256, 256),
                                   (513, 130, 1000), (64, 700, 33)], ids=lambda s: "x".join(map(str, s)))
def test_crt_shapes_one_and_two_cta(blas, oracle, shape):
    """m < 256 runs the one-CTA kernel, m >= 256 the CTA-pair kernel; ragged m / n / k."""
    m, n, k = shape
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    _crt_case(blas, oracle, "N", "N", m, n, k, m + 1, k + 2, m + 3, -0.75, 0.25, rng)


@pytest.mark.parametrize("nmod", [4, 8, 12, 15])
def test_crt_moduli_counts(blas, oracle, nmod):
    """Fewer moduli: fewer scaling bits P, larger (bounded) error."""
    rng = np.random.default_rng(nmod)
    _crt_case(blas, oracle, "T", "N", 130, 257, 300, 300, 300, 131, 1.0, 0.0, rng, nmod=nmod)


@pytest.mark.parametrize("phi", [4.0, 8.0, 16.0])
def test_crt_wide_dynamic_range(blas, oracle, phi):
    rng = np.random.default_rng(int(phi) + 1)
    _crt_case(blas, oracle, "N", "T", 96, 80, 512, 96, 80, 96, 1.0, -1.0, rng, phi=phi)


def _nonfinite_case(blas, oracle, scheme, ta, tb, m, n, k, ld, rng):
    """Inf / NaN in single entries of op(A), op(B) and C, compared entry by entry
    with the reference's loop (gemm.zig:1422-1429, the oracle): the same entries are
    NaN, +Inf and -Inf, and every finite entry meets the scheme's bound."""
    def store(rows, cols):
        return np.asfortranarray(rng.uniform(-1, 1, (ld, cols)))
    a = store(m if ta == "N" else k, k if ta == "N" else m)
    b = store(k if tb == "N" else n, n if tb == "N" else k)
    c = store(m, n)

    def put_a(i, p, v):  # op(A)[i, p]
        if ta == "N":
            a[i, p] = v
        else:
            a[p, i] = v

    def put_b(p, j, v):  # op(B)[p, j]
        if tb == "N":
            b[p, j] = v
        else:
            b[j, p] = v

    put_a(5, 17, np.inf)        # row 5: +-Inf times B's column entries
    put_b(17, 40, 0.0)          # ... Inf * 0 = NaN at C[5, 40]
    put_a(9, 100, -np.inf)      # row 9
    put_b(100, 41, np.nan)      # column 41 holds NaN: NaN down the column
    put_a(700 % m, 3, np.nan)   # row 700: NaN across the row
    put_b(64, 300 % n, np.inf)  # column 300: +-Inf down the column
    put_a(9, 64, np.inf)        # C[9, 300] meets +Inf * +Inf and -Inf * B: NaN or Inf by sign
    c[11, 12] = -np.inf         # beta * C: -Inf in an otherwise finite entry
    c[5, 13] = np.nan           # beta * C: NaN in an already non-finite row
    c0 = c.copy(order="F")
    alpha, beta = 1.5, 0.5
    blas.set_dgemm_method(blas.METHOD_OZAKI)
    old_s = blas.set_ozaki_scheme(blas.OZAKI_CRT if scheme == "crt" else blas.OZAKI_SLICES)
    old_n = blas.set_ozaki_slices(8 if scheme == "slices" else 0)
    try:
        blas.dgemm(ta, tb, m, n, k, alpha, a, ld, b, ld, beta, c, ld)
    finally:
        blas.set_ozaki_slices(old_n)
        blas.set_ozaki_scheme(old_s)
        blas.set_dgemm_method(blas.METHOD_NATIVE)
    ref = c0.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, alpha, a, ld, b, ld, beta, ref, ld)
    got, want = c[:m, :n], ref[:m, :n]
    assert np.array_equal(np.isnan(got), np.isnan(want)), "NaN entries differ"
    assert np.array_equal(np.isposinf(got), np.isposinf(want)), "+Inf entries differ"
    assert np.array_equal(np.isneginf(got), np.isneginf(want)), "-Inf entries differ"
    assert np.isnan(want).sum() > n and np.isinf(want).sum() > n  # the case really spreads non-finite values
    fin = np.isfinite(want)
    A = np.nan_to_num(np.abs(_op(a, ta, m, k)), nan=0.0, posinf=0.0)
    B = np.nan_to_num(np.abs(_op(b, tb, k, n)), nan=0.0, posinf=0.0)
    ab = A @ B
    # finite entries lie in rows / columns free of Inf / NaN; the slice scheme (8 digits) and
    # the CRT scheme both stay within 64 k u |A||B| + 4 u |beta C0| on U[-1, 1] data
    bound = 64 * k * U64 * (abs(alpha) * ab) + 4 * U64 * abs(beta) * np.abs(np.nan_to_num(c0[:m, :n]))
    err = np.abs(got[fin] - want[fin])
    assert np.all(err <= bound[fin]), float((err / bound[fin]).max())
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_crt_nonfinite_entries_match_reference_loop(blas, oracle, ta, tb):
    """1024^3 with ld 1031 (CTA-pair kernel), Inf / NaN in single entries of A, B and C."""
    _nonfinite_case(blas, oracle, "crt", ta, tb, 1024, 1024, 1024, 1031, np.random.default_rng(41))


@pytest.mark.parametrize("shape", [(200, 320, 150), (1024, 333, 257)], ids=lambda s: "x".join(map(str, s)))
def test_crt_nonfinite_one_and_two_cta(blas, oracle, shape):
    m, n, k = shape
    _nonfinite_case(blas, oracle, "crt", "N", "T", m, n, k, max(m, n, k) + 3, np.random.default_rng(m + n))


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_slices_nonfinite_entries_match_reference_loop(blas, oracle, ta, tb):
    _nonfinite_case(blas, oracle, "slices", ta, tb, 1024, 512, 384, 1031, np.random.default_rng(43))


def test_crt_zero_rows_give_exact_zeros(blas, oracle):
    """A zero row of op(A) gives exact zeros in its row of C (beta = 0)."""
    rng = np.random.default_rng(9)
    m, n, k = 70, 40, 90
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    a[3, :] = 0.0
    c = np.full((m, n), np.nan, order="F")
    blas.set_dgemm_method(blas.METHOD_OZAKI)
    old = blas.set_ozaki_scheme(blas.OZAKI_CRT)
    try:
        blas.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    finally:
        blas.set_ozaki_scheme(old)
        blas.set_dgemm_method(blas.METHOD_NATIVE)
    assert np.all(c[3, :] == 0.0)
    np.testing.assert_allclose(c, a @ b, rtol=1e-12, atol=1e-13)


def test_crt_long_k_falls_back_to_slices(blas):
    """K beyond the INT32 bound of one modular product runs the slice scheme."""
    from zynum_b200 import ozaki_info
    blas.set_dgemm_method(blas.METHOD_OZAKI)
    old = blas.set_ozaki_scheme(blas.OZAKI_CRT)
    try:
        assert ozaki_info(64, 64, 130816)["scheme"] == "crt"
        assert ozaki_info(64, 64, 130817)["scheme"] == "slices"
    finally:
        blas.set_ozaki_scheme(old)
        blas.set_dgemm_method(blas.METHOD_NATIVE)


def test_crt_matches_native_error_at_2048(blas, oracle):
    """Default CRT scheme (16 moduli) vs native FP64 on 2048^3, u * 10^U[-4,4] entries:
    max relative error on 4096 sampled entries no worse than native."""
    rng = np.random.default_rng(41)
    n = 2048
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-4, 4, (n, n)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-4, 4, (n, n)))
    rows, cols = rng.integers(0, n, 4096), rng.integers(0, n, 4096)
    hi, lo, _ = oracle.ddgemm_sampled("N", "N", n, a, n, b, n, rows, cols)
    exact = hi + lo
    errs = {}
    for name, method, scheme in (("native", blas.METHOD_NATIVE, 0), ("crt", blas.METHOD_OZAKI, blas.OZAKI_CRT)):
        c = np.zeros((n, n), order="F")
        blas.set_dgemm_method(method)
        old = blas.set_ozaki_scheme(scheme)
        try:
            blas.dgemm("N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c, n)
        finally:
            blas.set_ozaki_scheme(old)
            blas.set_dgemm_method(blas.METHOD_NATIVE)
        errs[name] = float((np.abs(c[rows, cols] - exact) / np.abs(exact)).max())
    assert errs["crt"] <= errs["native"], errs


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


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_host_panels_reuse_a_residues_bit_identical(blas, ta, tb):
    """dgemm_ with host buffers large enough for column panels (here 8, the last one ragged)
    computes op(A)'s CRT residues once and reuses them for every panel: the result is
    bit-identical to the unpanelled device-pointer call on the same data."""
    import torch
    m, n, k = 600, 4100, 3400
    rng = np.random.default_rng(17 + ord(ta))
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)) * 10.0 ** rng.uniform(-2, 2, (ar, ac)))
    b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    old = blas.set_dgemm_method(blas.METHOD_OZAKI)
    try:
        dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")  # noqa: E731
        C = dev(c)
        blas.dgemm_device(ta, tb, m, n, k, 1.25, dev(a), ar, dev(b), br, -0.5, C, m)
        torch.cuda.synchronize()
        want = np.asfortranarray(C.cpu().numpy().T)
        got = c.copy(order="F")
        blas.dgemm(ta, tb, m, n, k, 1.25, a, ar, b, br, -0.5, got, m)
    finally:
        blas.set_dgemm_method(old)
    assert np.array_equal(got, want)
