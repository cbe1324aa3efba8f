"""Variable-size batched GEMM / TRSM (one persistent launch, CUDA-graph replay,
autotuned tile configs) against per-problem references (GPU)."""
from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _loguniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.int32)


def _pack(torch, mats, dtype):
    """Column-major device copies of host matrices; returns tensors, pointer array, ld array."""
    ts = [torch.from_numpy(np.ascontiguousarray(x.T)).to(device="cuda", dtype=dtype) for x in mats]
    ptrs = torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device="cuda")
    lds = torch.tensor([x.shape[0] for x in mats], dtype=torch.int32, device="cuda")
    return ts, ptrs, lds


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_gemm_batch(blas, dtype, ta, tb):
    import torch
    rng = np.random.default_rng(hash((dtype, ta, tb)) % 2**32)
    cnt = 300
    m, n, k = (_loguniform(rng, 8, 512, cnt) for _ in range(3))
    m[0], n[0], k[0] = 0, 5, 7     # empty problem
    m[1], n[1], k[1] = 9, 11, 0    # k == 0: C = beta C
    npdt = np.float64 if dtype == "f64" else np.float32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    A = [rng.uniform(-1, 1, (m[q], k[q]) if ta == "N" else (k[q], m[q])).astype(npdt) for q in range(cnt)]
    B = [rng.uniform(-1, 1, (k[q], n[q]) if tb == "N" else (n[q], k[q])).astype(npdt) for q in range(cnt)]
    Cm = [rng.uniform(-1, 1, (m[q], n[q])).astype(npdt) for q in range(cnt)]
    # leading dimensions >= 1 for empty extents
    A = [x if x.shape[0] > 0 else np.zeros((1, x.shape[1]), npdt) for x in A]
    B = [x if x.shape[0] > 0 else np.zeros((1, x.shape[1]), npdt) for x in B]
    Cm = [x if x.shape[0] > 0 else np.zeros((1, x.shape[1]), npdt) for x in Cm]
    ta_, pa, la = _pack(torch, A, tdt)
    tb_, pb, lb = _pack(torch, B, tdt)
    tc_, pc, lc = _pack(torch, Cm, tdt)
    batch = blas.GemmBatch(m, n, k, dtype=dtype, transa=ta, transb=tb, tune=True)
    info = batch.info()
    assert info["grid"] > 0 and sum(info["tiles_per_cfg"].values()) > 0
    for use_graph in (False, True, True):  # graph capture, then replay
        for q in range(cnt):
            tc_[q].copy_(torch.from_numpy(np.ascontiguousarray(Cm[q].T)))
        batch.run(1.25, pa, la, pb, lb, -0.5, pc, lc, use_graph=use_graph)
        torch.cuda.synchronize()
        u = 2.0 ** -53 if dtype == "f64" else 2.0 ** -24
        for q in range(cnt):
            if m[q] == 0 or n[q] == 0:
                continue
            opA = (A[q] if ta == "N" else A[q].T).astype(np.float64)[: m[q], : k[q]]
            opB = (B[q] if tb == "N" else B[q].T).astype(np.float64)[: k[q], : n[q]]
            want = 1.25 * (opA @ opB) - 0.5 * Cm[q].astype(np.float64)
            got = tc_[q].cpu().numpy().T.astype(np.float64)
            bound = 4 * max(k[q], 1) * u * (1.25 * np.abs(opA) @ np.abs(opB) + 0.5 * np.abs(Cm[q])) + 1e-300
            assert np.all(np.abs(got - want) <= bound), (q, m[q], n[q], k[q])


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_gemm_batch_alpha_zero_and_padded_ld(blas, dtype):
    """alpha = 0 gives C = beta C without reading A or B (NaN in A stays out); padded, odd
    leading dimensions (ld = rows + 3) take the element-wise copies; the padding rows of C
    stay untouched."""
    import torch
    rng = np.random.default_rng(99)
    cnt = 64
    m, n, k = (_loguniform(rng, 8, 300, cnt) for _ in range(3))
    npdt = np.float64 if dtype == "f64" else np.float32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    A = [rng.uniform(-1, 1, (m[q] + 3, k[q])).astype(npdt) for q in range(cnt)]
    B = [rng.uniform(-1, 1, (k[q] + 3, n[q])).astype(npdt) for q in range(cnt)]
    C0 = [rng.uniform(-1, 1, (m[q] + 3, n[q])).astype(npdt) for q in range(cnt)]
    ta_, pa, la = _pack(torch, A, tdt)
    tb_, pb, lb = _pack(torch, B, tdt)
    batch = blas.GemmBatch(m, n, k, dtype=dtype, tune=False)
    u = 2.0 ** -53 if dtype == "f64" else 2.0 ** -24
    for alpha in (0.0, 1.5):
        if alpha == 0.0:
            for q in range(cnt):
                ta_[q][0, 0] = float("nan")  # element (0, 0) of A: never read when alpha = 0
        else:
            for q in range(cnt):
                ta_[q].copy_(torch.from_numpy(np.ascontiguousarray(A[q].T)))
        tc_, pc, lc = _pack(torch, C0, tdt)
        batch.run(alpha, pa, la, pb, lb, 0.5, pc, lc)
        torch.cuda.synchronize()
        for q in range(cnt):
            got = tc_[q].cpu().numpy().T.astype(np.float64)
            c0 = C0[q].astype(np.float64)
            if alpha == 0.0:
                want = 0.5 * c0[: m[q]]
                assert np.array_equal(got[: m[q]], want.astype(npdt).astype(np.float64)), q
            else:
                a, b = A[q].astype(np.float64)[: m[q]], B[q].astype(np.float64)[: k[q]]
                want = 1.5 * (a @ b) + 0.5 * c0[: m[q]]
                bound = 4 * k[q] * u * (1.5 * np.abs(a) @ np.abs(b) + 0.5 * np.abs(c0[: m[q]])) + 1e-300
                assert np.all(np.abs(got[: m[q]] - want) <= bound), q
            assert np.array_equal(got[m[q]:], c0[m[q]:]), "padding rows of C changed"
    batch.close()


def test_gemm_batch_tune_cache(blas, tmp_path, monkeypatch):
    """The autotuner's table is written to the JSON cache named by ZYNUM_GPU_TUNE_CACHE (fresh process)."""
    import subprocess
    import sys
    from pathlib import Path
    cache = tmp_path / "tune.json"
    root = Path(__file__).resolve().parents[1]
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from zynum_b200 import blas\n"
        "b = blas.GemmBatch([300]*8 + [20]*8, [300]*8 + [24]*8, [200]*8 + [30]*8, tune=True)\n"
        "print(b.info())\n" % str(root))
    env = dict(__import__("os").environ, ZYNUM_GPU_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    table = json.loads(cache.read_text())
    # a tile config per bucket, or -1: the size rule stays
    assert len(table) >= 2 and all(v in (-1, 0, 1, 2) for v in table.values())


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("U", "N", "N"), ("L", "T", "N"), ("U", "T", "U")])
def test_trsm_batch(blas, oracle, dtype, uplo, trans, diag):
    """Sizes 16..300 plus a few large problems (several 64-row blocks and 64-row panel chunks,
    ragged last block), 1..64 right-hand sides, alpha = 0.5."""
    import torch
    rng = np.random.default_rng(sum(map(ord, dtype + uplo + trans + diag)))
    cnt = 120
    nn = _loguniform(rng, 16, 300, cnt)
    nn[:4] = [1100, 777, 640, 193]
    rr = rng.integers(1, 65, cnt).astype(np.int32)
    rr[:4] = [64, 33, 1, 17]
    npdt = np.float64 if dtype == "f64" else np.float32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    Ls = []
    for q in range(cnt):
        L = np.tril(rng.standard_normal((nn[q], nn[q])), -1) if uplo == "L" else \
            np.triu(rng.standard_normal((nn[q], nn[q])), 1)
        L = L * 0.5 / np.sqrt(nn[q]) + np.diag(2 + np.abs(rng.standard_normal(nn[q])))
        Ls.append(L.astype(npdt))
    Bs = [rng.standard_normal((nn[q], rr[q])).astype(npdt) for q in range(cnt)]
    tl, pa, la = _pack(torch, Ls, tdt)
    tbb, pb, lb = _pack(torch, Bs, tdt)
    batch = blas.TrsmBatch(nn, rr, dtype=dtype, uplo=uplo, transa=trans, diag=diag)
    batch.run(0.5, pa, la, pb, lb, use_graph=True)
    torch.cuda.synchronize()
    tol = 1e-11 if dtype == "f64" else 2e-4
    for q in range(cnt):
        ref = np.asfortranarray(Bs[q].copy())
        oracle.trsm("L", uplo, trans, diag, nn[q], rr[q], 0.5, np.asfortranarray(Ls[q]), nn[q], ref, nn[q])
        got = tbb[q].cpu().numpy().T
        assert np.all(np.abs(got - ref) <= tol * (1 + np.abs(ref))), q


def test_batch_argument_errors(blas):
    with pytest.raises(ValueError):
        blas.TrsmBatch([10], [65])  # more than 64 right-hand sides
    with pytest.raises(ValueError):
        blas.GemmBatch([4], [-1], [4])
