"""Native DGEMM on 128 x 128 tiles and the tall-skinny routes against the CPU oracle (GPU).

Shapes large enough for the 128 x 128 route (many output tiles, or K beyond
1024), with even leading dimensions so that the TMA-fed kernel takes them,
and odd ones so that the cp.async kernel does: ragged M / N / K tails, K
tails of every residue class of the 32-deep slice, split K, every transpose
pair, and the triangle mode of SYRK.  Bound: |C - C_oracle| <= 4 k u
(|alpha| |op(A)| |op(B)| + |beta| |C0|); padding rows of C stay bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gemm_bound

pytestmark = pytest.mark.gpu
U64, U32 = 2.0 ** -53, 2.0 ** -24


def _case(blas, oracle, ta, tb, m, n, k, pad_a, pad_b, pad_c, alpha, beta, device, seed, dtype=np.float64):
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = ar + pad_a, br + pad_b, m + pad_c
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, ac)).astype(dtype))
    b = np.asfortranarray(rng.uniform(-1, 1, (ldb, bc)).astype(dtype))
    c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(dtype))
    a[ar:] = -999.0
    b[br:] = -999.0
    c[m:] = -999.0
    c0 = c.copy(order="F")
    ref = c.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ref, ldc)
    if device:
        import torch
        ta_ = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
        tb_ = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
        tc_ = torch.from_numpy(np.ascontiguousarray(c.T)).cuda()
        dev_fn = blas.dgemm_device if dtype == np.float64 else blas.sgemm_device
        dev_fn(ta, tb, m, n, k, alpha, ta_, lda, tb_, ldb, beta, tc_, ldc)
        torch.cuda.synchronize()
        c = np.asfortranarray(tc_.cpu().numpy().T)
    else:
        (blas.dgemm if dtype == np.float64 else blas.sgemm)(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    bound = gemm_bound(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c0, U64 if dtype == np.float64 else U32)
    err = np.abs(c[:m, :n].astype(np.float64) - ref[:m, :n].astype(np.float64))
    assert np.all(err <= bound), (float(err.max()), float((err / bound).max()))
    assert np.array_equal(c[m:], c0[m:]), "padding rows of C were written"


TRANS = [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")]


@pytest.mark.parametrize("ta,tb", TRANS)
@pytest.mark.parametrize("shape", [
    (1300, 1100, 1090),  # 99 tiles, no split, ragged tails
    (1000, 904, 1500),   # 64 tiles: split K in two
    (640, 512, 1057),    # K tail of 1 past a slice
    (520, 260, 1160),    # K tail of 8
    (384, 400, 1040),    # K tail of 16
    (130, 1030, 1105),   # K tail of 17
    (2048, 130, 1087),   # K tail of 31
], ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
def test_dgemm_128_tiles(blas, oracle, ta, tb, shape, device):
    m, n, k = shape
    # even leading dimensions (TMA-describable) on the device path; the host path stages compactly
    _case(blas, oracle, ta, tb, m, n, k, 2, 4, 3, 1.25, -0.5, device, m + n + k)


@pytest.mark.parametrize("ta,tb", TRANS)
def test_dgemm_128_tiles_odd_ld(blas, oracle, ta, tb):
    """Odd leading dimensions: the cp.async kernel."""
    _case(blas, oracle, ta, tb, 1030, 1020, 1500, 1, 3, 5, -0.75, 0.5, True, 7)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_dgemm_long_k_split(blas, oracle, ta, tb):
    """Few tiles, long K: split K over 32-deep-slice-aligned ranges plus the ordered reduction."""
    _case(blas, oracle, ta, tb, 256, 256, 40000, 2, 2, 1, 1.0, 0.0, True, 11)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_dsyrk_triangle_tiles(blas, oracle, uplo, trans):
    """SYRK's triangle mode on 128 x 128 tiles: only the stored triangle is written."""
    rng = np.random.default_rng(5)
    n, k = 1200, 1300
    ar, ac = (n, k) if trans == "N" else (k, n)
    a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)))
    c = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    c0 = c.copy(order="F")
    blas.syrk(uplo, trans, n, k, 0.5, a, ar, 1.5, c, n)
    opa = a if trans == "N" else a.T
    full = 0.5 * (opa @ opa.T) + 1.5 * c0
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    bound = 4 * k * U64 * (0.5 * (np.abs(opa) @ np.abs(opa).T) + 1.5 * np.abs(c0)) + 1e-300
    assert np.all(np.abs(c - full)[mask] <= bound[mask])
    assert np.array_equal(c[~mask], c0[~mask]), "the other triangle was written"


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("ta,tb", TRANS)
@pytest.mark.parametrize("shape,pad,beta", [
    ((131072, 64, 64), 0, 0.0),   # the sweep shape, TMA-fed when op(A) is aligned
    ((131072, 64, 64), 0, 1.0),
    ((5000, 37, 50), 4, 0.5),     # ragged n / k, padded leading dimension (TMA-describable)
    ((4097, 64, 33), 3, -1.0),    # ragged m tail and k, TMA-describable leading dimension
    ((3001, 64, 64), 1, 0.25),    # odd leading dimension: the cp.async kernel
], ids=["sweep-b0", "sweep-b1", "ragged", "mtail", "odd-ld"])
def test_skinny_device(blas, oracle, dtype, ta, tb, shape, pad, beta):
    m, n, k = shape
    _case(blas, oracle, ta, tb, m, n, k, pad, pad + 1, 3, -1.25, beta, True, m + 7 * n + k, dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_skinny_route_graph_capture(blas, dtype, beta):
    """The tall-skinny route needs no workspace, so a first call on a stream under CUDA-graph
    capture (a stream the library has not seen) records cleanly, and the replay writes the
    same C as a direct call (bit-identical: the same kernel on the same data)."""
    import torch
    torch.cuda.synchronize()
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    fn = blas.dgemm_device if dtype == np.float64 else blas.sgemm_device
    m, n, k = 131072, 64, 64
    g = torch.Generator(device="cuda").manual_seed(41)
    A = torch.rand((k, m), generator=g, device="cuda", dtype=tdt) * 2 - 1
    B = torch.rand((n, k), generator=g, device="cuda", dtype=tdt) * 2 - 1
    C0 = torch.rand((n, m), generator=g, device="cuda", dtype=tdt) * 2 - 1
    ref = C0.clone()
    fn("N", "N", m, n, k, 1.5, A, m, B, k, beta, ref, m)
    out = C0.clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        fn("N", "N", m, n, k, 1.5, A, m, B, k, beta, out, m)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


@pytest.mark.filterwarnings("ignore:The CUDA Graph is empty")  # the refused capture records nothing
def test_workspace_growth_refused_under_capture(blas):
    """A call whose per-stream workspace would have to grow (cudaMalloc) on a stream under
    CUDA-graph capture returns an error naming the remedy instead of invalidating the
    capture; after one uncaptured call on that stream the same call captures and replays
    to the direct result."""
    import torch
    from zynum_b200._lib import ZynumGpuError
    torch.cuda.synchronize()
    old = blas.set_dgemm_method(blas.METHOD_OZAKI)  # the CRT route keeps its planes in the workspace
    try:
        m, n, k = 1024, 768, 512
        g = torch.Generator(device="cuda").manual_seed(43)
        A = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        B = torch.rand((n, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        ref = torch.zeros((n, m), device="cuda", dtype=torch.float64)
        blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, ref, m)
        s = torch.cuda.Stream()
        out = torch.zeros_like(ref)
        graph = torch.cuda.CUDAGraph()
        with pytest.raises(ZynumGpuError, match="graph capture"):
            with torch.cuda.graph(graph, stream=s):
                blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):  # sizes the workspace of stream s
            blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m)
        s.synchronize()
        out.zero_()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, out, m)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    finally:
        blas.set_dgemm_method(old)


@pytest.mark.parametrize("ta,tb", TRANS)
@pytest.mark.parametrize("shape", [
    (256, 512, 256),   # blocked TRSM coupling: 32 tiles of 64 x 64, K split four ways
    (200, 130, 1000),  # ragged tiles, K split into 64-deep-aligned ranges
    (1030, 1020, 1500),  # 128 x 128 cp.async tiles (odd leading dimensions), K split in two
], ids=lambda s: "x".join(map(str, s)))
def test_splitk_fixup_repeats(blas, oracle, ta, tb, shape):
    """Split K through the workspace and the ordered reduction: right on every
    call and bit-identical across calls, with other split shapes run in
    between on the same stream."""
    import torch
    m, n, k = shape
    rng = np.random.default_rng(m + 3 * n + k)
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = ar + 1, br + 3, m + 1  # odd: the cp.async kernels
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, ac)))
    b = np.asfortranarray(rng.uniform(-1, 1, (ldb, bc)))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)))
    ref = c0.copy(order="F")
    oracle.gemm(ta, tb, m, n, k, 0.75, a, lda, b, ldb, -1.5, ref, ldc)
    ta_ = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    tb_ = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    other_a = torch.rand((300, 200), device="cuda", dtype=torch.float64)  # 200 x 300 x 300 split product
    other_c = torch.zeros((200, 200), device="cuda", dtype=torch.float64)
    outs = []
    for _ in range(3):
        tc_ = torch.from_numpy(np.ascontiguousarray(c0.T)).cuda()
        blas.dgemm_device(ta, tb, m, n, k, 0.75, ta_, lda, tb_, ldb, -1.5, tc_, ldc)
        blas.dgemm_device("N", "T", 200, 200, 300, 1.0, other_a, 200, other_a, 200, 0.0, other_c, 200)
        torch.cuda.synchronize()
        outs.append(np.asfortranarray(tc_.cpu().numpy().T))
    bound = gemm_bound(ta, tb, m, n, k, 0.75, a, lda, b, ldb, -1.5, c0, U64)
    err = np.abs(outs[0][:m, :n] - ref[:m, :n])
    assert np.all(err <= bound), (float(err.max()), float((err / bound).max()))
    assert np.array_equal(outs[0][m:], c0[m:]), "padding rows of C were written"
    for o in outs[1:]:
        assert np.array_equal(o, outs[0]), "split-K result changed between calls"


@pytest.mark.parametrize("uplo", ["U", "L"])
def test_splitk_fixup_triangle(blas, oracle, uplo):
    """SYRK on 64 x 64 tiles with split K: the reduction writes only the stored triangle."""
    rng = np.random.default_rng(9)
    n, k = 300, 900
    a = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    c0 = c.copy(order="F")
    blas.syrk(uplo, "T", n, k, -0.5, a, k, 2.0, c, n)
    full = -0.5 * (a.T @ a) + 2.0 * c0
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    bound = 4 * k * U64 * (0.5 * (np.abs(a.T) @ np.abs(a)) + 2.0 * np.abs(c0)) + 1e-300
    assert np.all(np.abs(c - full)[mask] <= bound[mask])
    assert np.array_equal(c[~mask], c0[~mask]), "the other triangle was written"
