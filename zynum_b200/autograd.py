"""torch.autograd.Function adjoints for GEMM, TRSM and SYRK on the GPU backend.

All tensors are ordinary row-major torch tensors (float64, CUDA).  Every
forward and backward product is one of this library's own kernels, called
through its C ABI; a row-major matrix is the column-major transpose, so each
call swaps operands / flips side and uplo exactly like the reference's CBLAS
row-major wrappers (src/blas/abi/cblas.zig:1428-1438, :1729-1743).

Adjoints (G = upstream gradient):
  gemm   C = alpha A B             dA = alpha G B^T,  dB = alpha A^T G
  trsm   X = alpha op(L)^-1 B      dB = alpha op(L)^-T G
                                   dL = -mask(dB Y^T)  (op = N) or -mask(Y dB^T) (op = T),
                                   Y = op(L)^-1 B, mask = the stored triangle of L
                                   (strict when the diagonal is unit)
  syrk   C = alpha X^T X (trans)   dX = alpha X (G + G^T)
         C = alpha X X^T           dX = alpha (G + G^T) X
The inverses of L's diagonal blocks are formed once in the TRSM forward and
kept for the backward's adjoint solve and recomputation (all three solves use
the same L; an odd order or an unaligned L forms them per solve instead).
With recompute=True the TRSM backward solves Y again from (L, B) instead of
keeping X alive between forward and backward, on a second stream beside the
adjoint solve; recompute="auto" (the default of
trsm()) decides at forward time from the device memory still free: X is
recomputed when keeping it until backward would take more than
RECOMPUTE_FRACTION of the free bytes (recompute_policy).
"""
from __future__ import annotations

import torch

from . import blas

_FLIP = {"U": "L", "L": "U"}

# Share of the free device memory a saved TRSM output may take before the
# backward recomputes it instead.
RECOMPUTE_FRACTION = 0.25


def recompute_policy(nbytes: int, free_bytes: int, fraction: float | None = None) -> bool:
    """True when keeping `nbytes` alive from forward to backward would use more than
    `fraction` (default RECOMPUTE_FRACTION) of the `free_bytes` the device still has."""
    f = RECOMPUTE_FRACTION if fraction is None else fraction
    return nbytes > f * free_bytes


def _check(t):
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError("zynum_b200.autograd expects float64 CUDA tensors")
    return t.contiguous()


# -------------------------------------------------- row-major primitives
def rm_gemm(alpha, a, b, beta, c, ta=False, tb=False):
    """c (m x n, row-major) = alpha op(a) op(b) + beta c."""
    m, n = c.shape
    k = a.shape[0] if ta else a.shape[1]
    # column-major: C^T (n x m) = op(b)^T (n x k) op(a)^T (k x m)
    blas.dgemm_device("T" if tb else "N", "T" if ta else "N", n, m, k, alpha, b, b.shape[1], a, a.shape[1],
                      beta, c, n)
    return c


def rm_gemmt(uplo, alpha, a, b, beta, c, ta=False, tb=False):
    """Triangle uplo of c (n x n, row-major) = alpha op(a) op(b) + beta c (other triangle untouched)."""
    n = c.shape[0]
    k = a.shape[0] if ta else a.shape[1]
    st = blas.load().zynum_blas_gpu_dgemmt_device(
        _FLIP[uplo].encode(), b"T" if tb else b"N", b"T" if ta else b"N", n, k, float(alpha), b.data_ptr(),
        b.shape[1], a.data_ptr(), a.shape[1], float(beta), c.data_ptr(), n, blas._stream(None))
    blas.check(st, "zynum_blas_gpu_dgemmt_device")
    return c


_SIDE_STREAMS: dict = {}


def _side_stream(device):
    """One extra stream per device for work that overlaps the current stream's."""
    key = torch.device(device).index
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(device=device)
    return _SIDE_STREAMS[key]


def rm_trsm_inverse(uplo, diag, l):
    """The diagonal-block inverses of l (n x n, row-major) for rm_trsm_left, or None where the
    library forms them per solve (odd n, or l not 16-byte aligned)."""
    n = l.shape[0]
    if n % 2 or l.data_ptr() % 16:
        return None
    inv = torch.empty(blas.dtrsm_inverse_bytes(n) // 8, dtype=torch.float64, device=l.device)
    blas.dtrsm_inverse_device(_FLIP[uplo], diag, n, l, n, inv)
    return inv


def rm_trsm_left(uplo, trans, diag, alpha, l, b, inv=None):
    """In place on b (n x r, row-major): b := alpha op(l)^-1 b, l (n x n, row-major) triangular;
    inv: l's diagonal-block inverses from rm_trsm_inverse (same uplo and diag), or None."""
    n, r = b.shape
    # column-major: X^T (r x n) = alpha B^T op(L)^-T -> right-side solve with L^T (flipped triangle)
    if inv is not None:
        blas.dtrsm_with_inverse_device("R", _FLIP[uplo], trans, diag, r, n, alpha, l, n, b, r, inv)
    else:
        blas.dtrsm_device("R", _FLIP[uplo], trans, diag, r, n, alpha, l, n, b, r)
    return b


def rm_syrk_full(alpha, x, trans_first):
    """Full symmetric alpha X^T X (trans_first) or alpha X X^T, from the SYRK kernel + a triangle mirror."""
    if trans_first:
        k, n = x.shape
        t = "N"     # column-major X^T (n x k): C = X^T X = X_cm X_cm^T
    else:
        n, k = x.shape
        t = "T"     # column-major X^T (k x n): C = X X^T = X_cm^T X_cm
    c = torch.empty((n, n), dtype=x.dtype, device=x.device)
    blas.dsyrk_device("L", t, n, k, alpha, x, x.shape[1], 0.0, c, n)
    st = blas.load().zynum_blas_gpu_dsymmetrize_device(b"L", n, c.data_ptr(), n, blas._stream(None))
    blas.check(st, "zynum_blas_gpu_dsymmetrize_device")
    return c


# ------------------------------------------------------------- functions
class Gemm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, b, alpha=1.0):
        a, b = _check(a), _check(b)
        c = torch.empty((a.shape[0], b.shape[1]), dtype=a.dtype, device=a.device)
        rm_gemm(alpha, a, b, 0.0, c)
        ctx.save_for_backward(a, b)
        ctx.alpha = alpha
        return c

    @staticmethod
    def backward(ctx, g):
        a, b = ctx.saved_tensors
        g = g.contiguous()
        da = db = None
        if ctx.needs_input_grad[0]:
            da = rm_gemm(ctx.alpha, g, b, 0.0, torch.empty_like(a), tb=True)
        if ctx.needs_input_grad[1]:
            db = rm_gemm(ctx.alpha, a, g, 0.0, torch.empty_like(b), ta=True)
        return da, db, None


class Trsm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, l, b, uplo="L", trans="N", diag="N", alpha=1.0, recompute=False):
        l, b = _check(l), _check(b)
        x = b.clone()
        inv = rm_trsm_inverse(uplo, diag, l)
        rm_trsm_left(uplo, trans, diag, alpha, l, x, inv)
        if recompute == "auto":
            free, _ = torch.cuda.mem_get_info(x.device)
            recompute = recompute_policy(x.numel() * x.element_size(), free)
        ctx.uplo, ctx.trans, ctx.diag, ctx.alpha, ctx.recompute = uplo, trans, diag, alpha, recompute
        ctx.inv = inv  # not a differentiable input: kept on ctx for the backward's solves
        if recompute:
            ctx.save_for_backward(l, b)  # X is solved again in backward
        else:
            ctx.save_for_backward(l, x)
        return x

    @staticmethod
    def backward(ctx, g):
        l, saved = ctx.saved_tensors
        g = g.contiguous()
        flip = "T" if ctx.trans == "N" else "N"
        # dB = alpha op(L)^-T G
        db = g.clone()
        dl = None
        if ctx.needs_input_grad[0] and ctx.recompute:
            # Y = op(L)^-1 B and dB are independent solves, each a latency-bound
            # chain of small kernels: Y runs on a second stream beside dB.  Y is
            # allocated on this stream, which waits for the second one before it
            # (or any later kernel) touches Y.
            y = saved.clone()
            cur = torch.cuda.current_stream(y.device)
            side = _side_stream(y.device)
            side.wait_stream(cur)
            with torch.cuda.stream(side):
                rm_trsm_left(ctx.uplo, ctx.trans, ctx.diag, 1.0, l, y, ctx.inv)
            rm_trsm_left(ctx.uplo, flip, ctx.diag, ctx.alpha, l, db, ctx.inv)
            cur.wait_stream(side)
        else:
            rm_trsm_left(ctx.uplo, flip, ctx.diag, ctx.alpha, l, db, ctx.inv)
        if ctx.needs_input_grad[0]:
            if not ctx.recompute:
                y = saved / ctx.alpha if ctx.alpha != 1.0 else saved
            dl = torch.zeros_like(l)
            if ctx.trans == "N":
                rm_gemmt(ctx.uplo, -1.0, db, y, 0.0, dl, tb=True)     # -(dB Y^T) on the stored triangle
            else:
                rm_gemmt(ctx.uplo, -1.0, y, db, 0.0, dl, tb=True)     # -(Y dB^T) on the stored triangle
            if ctx.diag == "U":
                dl.diagonal().zero_()
        return dl, (db if ctx.needs_input_grad[1] else None), None, None, None, None, None


class Syrk(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, trans_first=True, alpha=1.0):
        x = _check(x)
        ctx.save_for_backward(x)
        ctx.trans_first, ctx.alpha = trans_first, alpha
        return rm_syrk_full(alpha, x, trans_first)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        g = g.contiguous()
        dx = torch.empty_like(x)
        s = g + g.t()  # G + G^T (n x n, small): one product instead of two
        if ctx.trans_first:   # dX = alpha X (G + G^T)
            rm_gemm(ctx.alpha, x, s, 0.0, dx)
        else:                 # dX = alpha (G + G^T) X
            rm_gemm(ctx.alpha, s, x, 0.0, dx)
        return dx, None, None


def gemm(a, b, alpha=1.0):
    return Gemm.apply(a, b, alpha)


def trsm(l, b, uplo="L", trans="N", diag="N", alpha=1.0, recompute="auto"):
    """X = alpha op(L)^-1 B (left side); recompute True / False / "auto" (from free device memory)."""
    return Trsm.apply(l, b, uplo, trans, diag, alpha, recompute)


def syrk(x, trans_first=True, alpha=1.0):
    """Full symmetric alpha X^T X (trans_first) or alpha X X^T."""
    return Syrk.apply(x, trans_first, alpha)


def chain_loss(l, b, recompute=True):
    """The differentiation workload: X = TRSM(L, B), C = SYRK(X^T) = X^T X, loss = sum(sin(C))."""
    x = trsm(l, b, "L", "N", "N", 1.0, recompute)
    c = syrk(x, trans_first=True)
    return torch.sin(c).sum()
