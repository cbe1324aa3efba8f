"""Adjoint kernels behind torch.autograd.Function (GPU).

The differentiation chain X = TRSM(L, B), C = SYRK(X^T) = X^T X, loss =
sum(sin(C)) is checked (a) by central finite differences on 64 random
directions and (b) against the gradient assembled from the CPU oracle's BLAS
calls (restated from the reference's trsm / gemm semantics); each Function is
also run through torch.autograd.gradcheck.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chain_inputs(torch, n, r, seed):
    g = torch.Generator().manual_seed(seed)
    L = torch.tril(torch.randn(n, n, generator=g, dtype=torch.float64) / np.sqrt(n), -1)
    L += torch.diag(1 + torch.randn(n, generator=g, dtype=torch.float64).abs())
    B = torch.randn(n, r, generator=g, dtype=torch.float64)
    return L.cuda(), B.cuda()


def _loss(torch, ag, L, B, recompute=True):
    return ag.chain_loss(L, B, recompute=recompute)


def test_chain_finite_differences_64_directions():
    import torch
    from zynum_b200 import autograd as ag
    n, r = 150, 24  # three 64-row diagonal blocks
    L, B = _chain_inputs(torch, n, r, 0)
    L.requires_grad_(True)
    B.requires_grad_(True)
    loss = _loss(torch, ag, L, B)
    gL, gB = torch.autograd.grad(loss, (L, B))
    gen = torch.Generator(device="cuda").manual_seed(1)
    h = 1e-6
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            VL = torch.tril(torch.randn(n, n, generator=gen, device="cuda", dtype=torch.float64))
            VB = torch.randn(n, r, generator=gen, device="cuda", dtype=torch.float64)
            fp = _loss(torch, ag, L + h * VL, B + h * VB)
            fm = _loss(torch, ag, L - h * VL, B - h * VB)
            fd = (fp - fm).item() / (2 * h)
            an = (gL * VL).sum().item() + (gB * VB).sum().item()
            worst = max(worst, abs(fd - an) / max(1.0, abs(an)))
    assert worst < 1e-6, worst


def test_chain_against_cpu_blas_adjoint(oracle):
    """Gradient assembled from CPU oracle calls: X = trsm(L,B); C = X^T X; G_C = cos(C);
    G_X = X (G_C + G_C^T); dB = trsm(L^T, G_X); dL = -tril(dB X^T)."""
    import torch
    from zynum_b200 import autograd as ag
    n, r = 200, 32
    L, B = _chain_inputs(torch, n, r, 3)
    L.requires_grad_(True)
    B.requires_grad_(True)
    gL, gB = torch.autograd.grad(_loss(torch, ag, L, B), (L, B))
    Lh = np.asfortranarray(L.detach().cpu().numpy())
    X = np.asfortranarray(B.detach().cpu().numpy())
    oracle.trsm("L", "L", "N", "N", n, r, 1.0, Lh, n, X, n)
    C = np.zeros((r, r), order="F")
    oracle.gemm("T", "N", r, r, n, 1.0, X, n, X, n, 0.0, C, r)
    GC = np.asfortranarray(np.cos(C))
    GX = np.zeros((n, r), order="F")
    oracle.gemm("N", "N", n, r, r, 1.0, X, n, GC, r, 0.0, GX, n)
    oracle.gemm("N", "T", n, r, r, 1.0, X, n, GC, r, 1.0, GX, n)
    dB = GX.copy(order="F")
    oracle.trsm("L", "L", "T", "N", n, r, 1.0, Lh, n, dB, n)
    dL = np.zeros((n, n), order="F")
    oracle.gemm("N", "T", n, n, r, -1.0, dB, n, X, n, 0.0, dL, n)
    dL = np.tril(dL)
    np.testing.assert_allclose(gB.cpu().numpy(), dB, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(gL.cpu().numpy(), dL, rtol=1e-9, atol=1e-10)


def test_recompute_matches_stored():
    import torch
    from zynum_b200 import autograd as ag
    L, B = _chain_inputs(torch, 130, 16, 5)
    grads = []
    for recompute in (False, True):
        l = L.clone().requires_grad_(True)
        b = B.clone().requires_grad_(True)
        grads.append(torch.autograd.grad(_loss(torch, ag, l, b, recompute), (l, b)))
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("U", "N", "N"), ("L", "T", "N"), ("U", "T", "U")])
def test_trsm_gradcheck(uplo, trans, diag):
    import torch
    from zynum_b200 import autograd as ag
    n, r = 70, 5
    g = torch.Generator().manual_seed(7)
    T = torch.randn(n, n, generator=g, dtype=torch.float64) * 0.2
    T = torch.tril(T) if uplo == "L" else torch.triu(T)
    T = T + torch.diag(2 + torch.rand(n, generator=g, dtype=torch.float64))
    L = T.cuda().requires_grad_(True)
    B = torch.randn(n, r, generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    mask = (torch.tril(torch.ones(n, n)) if uplo == "L" else torch.triu(torch.ones(n, n))).cuda().double()
    if diag == "U":
        mask = mask - torch.eye(n, device="cuda", dtype=torch.float64)

    def f(l, b):
        # only the stored triangle of L is a parameter
        return ag.trsm(l * mask + L.detach() * (1 - mask), b, uplo, trans, diag, 0.5)

    assert torch.autograd.gradcheck(f, (L, B), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_gemm_and_syrk_gradcheck():
    import torch
    from zynum_b200 import autograd as ag
    g = torch.Generator().manual_seed(9)
    A = torch.randn(33, 20, generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    Bm = torch.randn(20, 17, generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda a, b: ag.gemm(a, b, 1.5), (A, Bm), eps=1e-6, atol=1e-7)
    X = torch.randn(40, 12, generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: ag.syrk(x, True, 0.75), (X,), eps=1e-6, atol=1e-7)
    assert torch.autograd.gradcheck(lambda x: ag.syrk(x, False), (X,), eps=1e-6, atol=1e-7)


def test_auto_recompute_follows_free_memory(monkeypatch):
    """recompute="auto": X is kept when it is small against the free device memory and
    recomputed when it is not; the gradients agree either way."""
    import torch
    from zynum_b200 import autograd as ag
    L, B = _chain_inputs(torch, 256, 32, 5)
    grads = {}
    for free, expect in ((1 << 40, False), (256 * 32 * 8, True)):
        monkeypatch.setattr(torch.cuda, "mem_get_info", lambda device=None, f=free: (f, 1 << 40))
        Lr, Br = L.clone().requires_grad_(True), B.clone().requires_grad_(True)
        x = ag.trsm(Lr, Br)  # recompute="auto"
        assert x.grad_fn.recompute is expect
        torch.sin(ag.syrk(x)).sum().backward()
        grads[expect] = (Lr.grad, Br.grad)
    assert torch.allclose(grads[False][0], grads[True][0], rtol=1e-12, atol=1e-14)
    assert torch.allclose(grads[False][1], grads[True][1], rtol=1e-12, atol=1e-14)
