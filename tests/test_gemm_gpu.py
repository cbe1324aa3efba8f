"""Parity of the native GPU DGEMM / SGEMM against the CPU oracle (GPU tests).

Mirrors the reference's ABI tests (test/abi/fortran_compat_test.zig):
sentinel-padded operands (padding rows of C must stay bit-exact), odd tails,
padded leading dimensions, every NN/NT/TN/TT combination, alpha/beta sets,
quick returns and NaN isolation.  Results must satisfy the componentwise
bound |C - C_oracle| <= 4 k u (|alpha| |op(A)| |op(B)| + |beta| |C0|).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from conftest import gemm_bound, padded

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())
U64, U32 = 2.0 ** -53, 2.0 ** -24


def _op_shape(t, rows, cols):
    return (rows, cols) if t == "N" else (cols, rows)


def _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, ldc, alpha, beta, salt=0):
    sentinel = -999.0 if dtype == np.float64 else -777.0
    ar, ac = _op_shape(ta, m, k)
    br, bc = _op_shape(tb, k, n)
    a = padded(ar, ac, lda, 1 + salt, dtype, sentinel)
    b = padded(br, bc, ldb, 5 + salt, dtype, sentinel)
    c = padded(m, n, ldc, 9 + salt, dtype, sentinel)
    ref = c.copy(order="F")
    c0 = c.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ref, ldc)
    fn = blas.dgemm if dtype == np.float64 else blas.sgemm
    fn(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    u = U64 if dtype == np.float64 else U32
    bound = gemm_bound(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c0, u)
    err = np.abs(c[:m, :n].astype(np.float64) - ref[:m, :n].astype(np.float64))
    assert np.all(err <= bound), (float(err.max()), float(bound[err > bound].min()))
    assert np.array_equal(c[m:, :], c0[m:, :]), "padding rows of C were written"
    assert np.array_equal(c[:, n:], c0[:, n:])


def test_dgemm_known_answer(blas):
    g = GOLDEN["dgemm_column_major_nn"]
    a = np.asfortranarray(np.array(g["a"], float).reshape(3, 2).T)
    b = np.asfortranarray(np.array(g["b"], float).reshape(2, 3).T)
    c = np.zeros((2, 2), order="F")
    blas.dgemm("N", "N", 2, 2, 3, 1.0, a, 2, b, 3, 0.0, c, 2)
    assert list(c.T.ravel()) == g["c"]


def test_cblas_row_major_known_answer(blas):
    g = GOLDEN["cblas_dgemm_row_major"]
    a = np.array(g["a_row_major"], float)
    b = np.array(g["b_row_major"], float)
    c = np.zeros(4)
    blas.cblas_dgemm(blas.CblasRowMajor, blas.CblasNoTrans, blas.CblasNoTrans, 2, 2, 3, 1.0, a, 3, b, 2, 0.0, c, 2)
    assert list(c) == g["c_row_major"]


def test_nan_isolation(blas):
    g = GOLDEN["gemm_nan_isolation"]
    a = np.asfortranarray(np.array(g["a"], float).reshape(2, 2).T)
    b = np.asfortranarray(np.array(g["b"], float).reshape(2, 2).T)
    c = np.full((2, 2), np.nan, order="F")
    blas.dgemm("N", "N", 2, 2, 2, 1.0, a, 2, b, 2, 0.0, c, 2)
    assert list(c.T.ravel()) == g["c_beta0"]
    a[:] = np.nan
    b[:] = np.nan
    c = np.asfortranarray(np.array([1.0, 2, 3, 4]).reshape(2, 2).T)
    blas.dgemm("N", "N", 2, 2, 2, 0.0, a, 2, b, 2, 2.0, c, 2)
    assert list(c.T.ravel()) == g["c_alpha0"]


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_dgemm_config1_padded_1024(blas, oracle, ta, tb):
    """M=N=K=1024, lda=ldb=ldc=1031, alpha=1.5, beta=0.5, U[-1,1] (the plain-DGEMM parity config)."""
    rng = np.random.default_rng(20260101)
    m = n = k = 1024
    ld = 1031
    a = np.asfortranarray(rng.uniform(-1, 1, (ld, 1024)))
    b = np.asfortranarray(rng.uniform(-1, 1, (ld, 1024)))
    c = np.asfortranarray(rng.uniform(-1, 1, (ld, 1024)))
    a[1024:] = -999.0
    b[1024:] = -999.0
    c[1024:] = -999.0
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, 1.5, a, ld, b, ld, 0.5, ref, ld)
    blas.dgemm(ta, tb, m, n, k, 1.5, a, ld, b, ld, 0.5, c, ld)
    bound = gemm_bound(ta, tb, m, n, k, 1.5, a, ld, b, ld, 0.5, c0, U64)
    err = np.abs(c[:m] - ref[:m])
    assert np.all(err <= bound)
    assert np.array_equal(c[m:], c0[m:])
    # the reference bench's sampled check |delta| <= 1e-9 k (gemm_sweep.zig:247-258)
    assert err.max() <= 1e-9 * k


SHAPES = [
    # (m, n, k, extra lda, extra ldb, extra ldc, alpha, beta) from fortran_compat_test.zig:638-730, :973-1010
    (5, 5, 3, 2, 2, 3, -0.5, 2.0),
    (7, 5, 3, 2, 2, 3, -0.5, 2.0),
    (35, 37, 67, 4, 4, 6, -0.5, 2.0),
    (37, 35, 71, 4, 4, 6, 1.0, 0.0),
    (128, 128, 128, 3, 9, 11, 1.0, 0.0),
    (17, 19, 2049, 6, 10, 14, 0.75, -0.25),
    (1, 257, 131, 2, 6, 4, -0.5, 2.0),
    (257, 1, 131, 6, 2, 12, -0.5, 2.0),
    (193, 65, 577, 4, 4, 6, 0.75, -0.25),
    (127, 129, 65, 4, 4, 8, 1.0, 0.0),
    (130, 161, 67, 3, 4, 5, 1.0, 0.0),
    (64, 129, 128, 3, 4, 5, 0.001, 0.0),
    (5, 7, 11, 2, 2, 6, 0.0, -0.25),   # alpha == 0 quick return
    (5, 7, 0, 3, 3, 6, 1.0, 2.0),      # k == 0 quick return
]


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s[:3])))
def test_gemm_shape_matrix(blas, oracle, dtype, ta, tb, shape):
    m, n, k, ea, eb, ec, alpha, beta = shape
    lda = max(1, (m if ta == "N" else k)) + ea
    ldb = max(1, (k if tb == "N" else n)) + eb
    ldc = m + ec
    _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, ldc, alpha, beta)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
def test_split_k_path(blas, oracle, dtype):
    """Few output tiles and long K go through the split-K workspace + ordered reduction."""
    _run_case(blas, oracle, dtype, "N", "N", 96, 80, 40000, 96, 40000, 97, 1.25, -0.5)
    _run_case(blas, oracle, dtype, "T", "T", 96, 80, 40000, 40000, 80, 96, 1.0, 0.0)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("T", "T"), ("C", "N")])
def test_sgemm_operand_relayout_path(blas, oracle, ta, tb):
    """m, n >= 1024: a K-contiguous operand (A with op T/C, B with op N) is first copied out
    MN-contiguous into the workspace; odd leading dimensions and a split-K case included."""
    _run_case(blas, oracle, np.float32, ta, tb, 1030, 1027, 301, (1030 if ta == "N" else 301) + 3,
              (301 if tb == "N" else 1027) + 1, 1033, 0.75, -1.25)
    _run_case(blas, oracle, np.float32, ta, tb, 1024, 1100, 4100, (1024 if ta == "N" else 4100) + 1,
              (4100 if tb == "N" else 1100) + 2, 1025, 1.0, 0.0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(5000, 64, 64), (2049, 1, 1), (3001, 37, 50), (2300, 64, 9)],
                         ids=lambda s: "x".join(map(str, s)))
def test_skinny_route(blas, oracle, dtype, ta, tb, shape):
    """n <= 64, k <= 64, m >= 2048: op(B) staged once per CTA, op(A) streamed in 128-row blocks;
    ragged m / n / k, padded leading dimensions, alpha and beta."""
    m, n, k = shape
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 1
    _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, m + 2, -1.25, 0.5)


def test_skinny_tile_path(blas, oracle):
    """Tall-skinny N <= 64 runs the 128 x 64 tile."""
    _run_case(blas, oracle, np.float64, "N", "N", 4096, 64, 64, 4096, 64, 4096, 1.0, 1.0)
    _run_case(blas, oracle, np.float64, "N", "T", 3001, 37, 50, 3003, 40, 3001, -1.0, 0.5)


def test_device_entry_torch(blas, oracle):
    import torch
    rng = np.random.default_rng(7)
    m, n, k = 300, 200, 150
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    ref = c.copy(order="F")
    oracle.gemm("N", "N", m, n, k, 2.0, a, m, b, k, -1.0, ref, m)
    ta = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # row-major (k, m) storage == column-major (m, k)
    tb = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    tc = torch.from_numpy(np.ascontiguousarray(c.T)).cuda()
    blas.dgemm_device("N", "N", m, n, k, 2.0, ta, m, tb, k, -1.0, tc, m)
    torch.cuda.synchronize()
    got = tc.cpu().numpy().T
    assert np.abs(got - ref).max() <= 4 * k * U64 * (2 * (np.abs(a) @ np.abs(b)) + np.abs(c)).max()


def test_injected_reservation_failure_leaves_c_unchanged(blas):
    """Failure before write: a denied device reservation returns with C untouched."""
    rng = np.random.default_rng(1)
    a = np.asfortranarray(rng.uniform(-1, 1, (64, 64)))
    c = np.asfortranarray(rng.uniform(-1, 1, (64, 64)))
    c0 = c.copy(order="F")
    blas.shutdown()  # drop cached buffers so the next call must reserve
    blas.inject_fault(1, 1)
    blas.dgemm("N", "N", 64, 64, 64, 1.0, a, 64, a, 64, 0.5, c, 64)
    assert np.array_equal(c, c0)
    assert "reservation" in blas.last_error()
    blas.dgemm("N", "N", 64, 64, 64, 1.0, a, 64, a, 64, 0.5, c, 64)  # works again
    assert not np.array_equal(c, c0)


def test_injected_sync_error_leaves_c_unchanged(blas):
    rng = np.random.default_rng(2)
    a = np.asfortranarray(rng.uniform(-1, 1, (32, 32)))
    c = np.asfortranarray(rng.uniform(-1, 1, (32, 32)))
    c0 = c.copy(order="F")
    blas.inject_fault(2, 700)  # report cudaErrorIllegalAddress from the host-side sync (no GPU fault)
    blas.dgemm("N", "N", 32, 32, 32, 1.0, a, 32, a, 32, 0.5, c, 32)
    assert np.array_equal(c, c0)


GEMV_SHAPES = [
    # (m, n, k): n == 1 and m == 1 with ragged output counts; long K takes the
    # K-split partials + ordered reduction, short K a single pass
    (5000, 1, 3000),
    (1, 4099, 2500),
    (70001, 1, 37),
    (1, 33333, 19),
    (300, 1, 100000),
    (1, 1, 5000),
    (129, 1, 1),
    (3001, 1, 64),
    (1, 2999, 9),
]


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", GEMV_SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("pad", [0, 1], ids=["vec", "odd_ld"])
def test_gemv_route(blas, oracle, dtype, ta, tb, shape, pad):
    """n == 1 / m == 1 run the matrix-vector kernels (gemm.zig:189-224, :228-240 route these
    to GEMV): every transpose pair, so both the outputs-contiguous and the dot-product kernel
    run with unit and strided vectors; pad = 0 keeps leading dimensions 16-byte multiples
    (vector loads), pad = 1 makes them odd (scalar loads)."""
    m, n, k = shape
    lda = (m if ta == "N" else k)
    ldb = (k if tb == "N" else n)
    lda = (lda + 3) // 4 * 4 + pad
    ldb = (ldb + 3) // 4 * 4 + pad
    _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, m + 2, -1.25, 0.5)
    _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, m, 0.75, 0.0, salt=3)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
def test_gemv_beta_zero_clears_nan(blas, dtype):
    """beta == 0 overwrites C without reading it (NaN in C does not propagate), on both
    matrix-vector kernels and through the K-split reduction."""
    rng = np.random.default_rng(11)
    for m, n, k in [(4000, 1, 5000), (1, 4000, 5000), (4000, 1, 64)]:
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k)).astype(dtype))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n)).astype(dtype))
        c = np.full((m, n), np.nan, dtype=dtype, order="F")
        fn = blas.dgemm if dtype == np.float64 else blas.sgemm
        fn("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m)
        ref = a.astype(np.float64) @ b.astype(np.float64)
        assert np.all(np.isfinite(c))
        tol = 1e-12 if dtype == np.float64 else 2e-4
        assert np.max(np.abs(c - ref)) <= tol * max(1.0, float(np.max(np.abs(ref))))


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(3000, 7, 5000), (5000, 16, 3000), (7, 3001, 4000), (16, 4100, 1030),
                                   (513, 2, 2000), (2, 777, 300), (4099, 13, 700), (3, 1200, 33)],
                         ids=lambda s: "x".join(map(str, s)))
def test_gemm_narrow_route(blas, oracle, dtype, ta, tb, shape):
    """n <= 16 (m <= 16) against a wide other side: FP64 128 x 16 (16 x 128) DMMA tiles, FP32
    the narrow FFMA kernel (2, 4, 8 or 16 vector slots); split K over long reductions, ragged
    tiles, odd leading dimensions (element copies) and 16-byte-multiple ones (vector copies)."""
    m, n, k = shape
    for pad, alpha, beta in ((1, -1.25, 0.5), (0, 1.0, 0.0)):
        lda = (m if ta == "N" else k) + pad
        ldb = (k if tb == "N" else n) + pad
        if pad == 0:
            lda, ldb = (lda + 3) // 4 * 4, (ldb + 3) // 4 * 4
        _run_case(blas, oracle, dtype, ta, tb, m, n, k, lda, ldb, m + 1, alpha, beta)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_host_column_panel_pipeline(blas, dtype, ta, tb):
    """Host calls with n >= 2048 and 2mnk >= 8e9 run as column panels of C (uploads, products
    and downloads overlapped on three streams); ragged last panel, padded leading dimensions,
    beta != 0, and the padding rows of C untouched."""
    m, n, k = 601, 2100, 3400
    rng = np.random.default_rng(5 + ord(ta) + 2 * ord(tb))
    ar, ac = _op_shape(ta, m, k)
    br, bc = _op_shape(tb, k, n)
    lda, ldb, ldc = ar + 3, br + 1, m + 2
    a = np.asfortranarray(np.full((lda, ac), -999.0)); a[:ar] = rng.uniform(-1, 1, (ar, ac))
    b = np.asfortranarray(np.full((ldb, bc), -999.0)); b[:br] = rng.uniform(-1, 1, (br, bc))
    c = np.asfortranarray(np.full((ldc, n), -777.0)); c[:m] = rng.uniform(-1, 1, (m, n))
    a, b, c = (np.asfortranarray(x.astype(dtype)) for x in (a, b, c))
    c0 = c.copy(order="F")
    A = a[:ar, :ac].astype(np.float64); A = A if ta == "N" else A.T
    B = b[:br, :bc].astype(np.float64); B = B if tb == "N" else B.T
    ref = 0.75 * (A @ B) - 0.5 * c0[:m].astype(np.float64)
    fn = blas.dgemm if dtype == np.float64 else blas.sgemm
    fn(ta, tb, m, n, k, 0.75, a, lda, b, ldb, -0.5, c, ldc)
    u = U64 if dtype == np.float64 else U32
    bound = 4 * k * u * (0.75 * (np.abs(A) @ np.abs(B)) + 0.5 * np.abs(c0[:m].astype(np.float64)))
    assert np.all(np.abs(c[:m].astype(np.float64) - ref) <= bound)
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"


def test_host_column_panel_injected_sync_error_leaves_c_unchanged(blas):
    """An error reported before the first panel's download leaves all of C untouched."""
    rng = np.random.default_rng(3)
    m, n, k = 512, 2048, 4096
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    c0 = c.copy(order="F")
    blas.inject_fault(2, 700)
    blas.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, c, m)
    assert np.array_equal(c, c0)
    blas.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, c, m)  # works again
    assert np.abs(c - (a @ b + 0.5 * c0)).max() <= 1e-11 * k
