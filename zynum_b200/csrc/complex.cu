// Complex GEMM (ZGEMM / CGEMM) through real GEMMs.
//
//   C = alpha * op(A) * op(B) + beta * C,  op in {N, T, C},  interleaved (re, im)
//
// Replaces the reference's complex routes (core/matrix_matrix/gemm.zig):
//   * "expanded real" (gemm.zig:945-1005): one real GEMM of shape
//     (2m x 2k) * (2k x n):  [[Ar, -Ai], [Ai, Ar]] * [Br; Bi] = [Cr; Ci]   (4M flops)
//   * "3M" (gemm.zig:1039, planes :1173-1203): three real GEMMs
//     cr = Ar (Br + Bi), tmp = (Ar + Ai) Bi, ci = (Ai - Ar) Br,
//     Re C = cr - tmp, Im C = cr + ci                                       (3M flops)
// Unlike the reference (which takes these routes only for alpha = 1, beta = 0,
// gemm.zig:420-442), the combine kernel applies any complex alpha / beta, so
// every call takes the GPU route.  The real GEMMs are whatever the caller
// supplies (native FP64 / FP32, Ozaki INT8 or 3xBF16).
#include "common.cuh"
#include "complex.h"

namespace zb {
namespace {

inline int grid_for(long total) {
    long b = (total + 255) / 256;
    if (b > 148L * 32) b = 148L * 32;
    return b < 1 ? 1 : (int)b;
}

// op(X)[r, c] of an interleaved complex matrix stored with leading dimension ld.
template <typename T>
ZB_DEVICE void op_value(const T* x, long ld, char t, long r, long c, T& re, T& im) {
    const T* p = (t == 'N') ? x + 2 * (r + c * ld) : x + 2 * (c + r * ld);
    re = p[0];
    im = (t == 'C') ? -p[1] : p[1];
}

// A_exp (2m x 2k, ld 2m) = [[Ar, -Ai], [Ai, Ar]] of op(A) (m x k).
template <typename T>
__global__ void expand_a(const T* __restrict__ a, long lda, char ta, int m, int k, T* __restrict__ out) {
    const long total = (long)m * k;
    const long ld = 2L * m;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long i = q % m, p = q / m;
        T re, im;
        op_value(a, lda, ta, i, p, re, im);
        out[i + p * ld] = re;
        out[i + (k + p) * ld] = -im;
        out[m + i + p * ld] = im;
        out[m + i + (k + p) * ld] = re;
    }
}

// B_st (2k x n, ld 2k) = [Br; Bi] of op(B) (k x n).
template <typename T>
__global__ void stack_b(const T* __restrict__ b, long ldb, char tb, int k, int n, T* __restrict__ out) {
    const long total = (long)k * n;
    const long ld = 2L * k;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long p = q % k, j = q / k;
        T re, im;
        op_value(b, ldb, tb, p, j, re, im);
        out[p + j * ld] = re;
        out[k + p + j * ld] = im;
    }
}

// C = alpha (Cr + i Ci) + beta C, with Cr / Ci the two halves of a 2m x n real result.
template <typename T>
__global__ void combine_expanded(const T* __restrict__ cst, int m, int n, T ar, T ai, T br, T bi, T* __restrict__ c,
                                 long ldc, int tri) {
    const long total = (long)m * n;
    const bool beta0 = (br == T(0) && bi == T(0));
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long i = q % m, j = q / m;
        if (tri == 1 ? i > j : (tri == 2 && i < j)) continue;  // outside the computed triangle
        const T xr = cst[i + j * 2L * m], xi = cst[m + i + j * 2L * m];
        T* cp = c + 2 * (i + j * ldc);
        T rr = ar * xr - ai * xi, ri = ar * xi + ai * xr;
        if (!beta0) {
            const T cr = cp[0], ci = cp[1];
            rr += br * cr - bi * ci;
            ri += br * ci + bi * cr;
        }
        cp[0] = rr;
        cp[1] = ri;
    }
}

// 3M planes of op(A): ar = Re, as = Re + Im, am = Im - Re  (each m x k, ld m)
template <typename T>
__global__ void planes_a3(const T* __restrict__ a, long lda, char ta, int m, int k, T* __restrict__ out) {
    const long total = (long)m * k;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long i = q % m, p = q / m;
        T re, im;
        op_value(a, lda, ta, i, p, re, im);
        out[q] = re;
        out[total + q] = re + im;
        out[2 * total + q] = im - re;
    }
}

// 3M planes of op(B): br = Re, bi = Im, bp = Re + Im  (each k x n, ld k)
template <typename T>
__global__ void planes_b3(const T* __restrict__ b, long ldb, char tb, int k, int n, T* __restrict__ out) {
    const long total = (long)k * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long p = q % k, j = q / k;
        T re, im;
        op_value(b, ldb, tb, p, j, re, im);
        out[q] = re;
        out[total + q] = im;
        out[2 * total + q] = re + im;
    }
}

// Re = cr - tmp, Im = cr + ci, then alpha / beta.
template <typename T>
__global__ void combine_3m(const T* __restrict__ prod, int m, int n, T ar, T ai, T br, T bi, T* __restrict__ c,
                           long ldc, int tri) {
    const long total = (long)m * n;
    const bool beta0 = (br == T(0) && bi == T(0));
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long i = q % m, j = q / m;
        if (tri == 1 ? i > j : (tri == 2 && i < j)) continue;  // outside the computed triangle
        const T cr = prod[q], tmp = prod[total + q], ci = prod[2 * total + q];
        const T xr = cr - tmp, xi = cr + ci;
        T* cp = c + 2 * (i + j * ldc);
        T rr = ar * xr - ai * xi, ri = ar * xi + ai * xr;
        if (!beta0) {
            const T c0 = cp[0], c1 = cp[1];
            rr += br * c0 - bi * c1;
            ri += br * c1 + bi * c0;
        }
        cp[0] = rr;
        cp[1] = ri;
    }
}

}  // namespace

template <typename T>
size_t complex_plane_bytes(int method, int m, int n, int k) {
    const size_t e = sizeof(T);
    size_t b;
    if (method == COMPLEX_3M)
        b = e * (3ul * m * k + 3ul * k * n + 3ul * m * n);
    else
        b = e * (4ul * m * k + 2ul * k * n + 2ul * m * n);
    return (b + 1023) & ~size_t(1023);
}

template <typename T>
cudaError_t complex_gemm(const ComplexArgs<T>& g, int method, void* planes, const RealGemm<T>& real_gemm,
                         cudaStream_t st) {
    const int m = g.m, n = g.n, k = g.k;
    T* w = static_cast<T*>(planes);
    cudaError_t e;
    if (method == COMPLEX_3M) {
        T* pa = w;
        T* pb = pa + 3L * m * k;
        T* pc = pb + 3L * k * n;
        planes_a3<T><<<grid_for((long)m * k), 256, 0, st>>>(g.a, g.lda, g.transa, m, k, pa);
        count_launch();
        planes_b3<T><<<grid_for((long)k * n), 256, 0, st>>>(g.b, g.ldb, g.transb, k, n, pb);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const long mk = (long)m * k, kn = (long)k * n, mn = (long)m * n;
        // cr = ar * bp, tmp = as * bi, ci = am * br
        if ((e = real_gemm(m, n, k, pa, m, pb + 2 * kn, k, pc, m, g.tri)) != cudaSuccess) return e;
        if ((e = real_gemm(m, n, k, pa + mk, m, pb + kn, k, pc + mn, m, g.tri)) != cudaSuccess) return e;
        if ((e = real_gemm(m, n, k, pa + 2 * mk, m, pb, k, pc + 2 * mn, m, g.tri)) != cudaSuccess) return e;
        combine_3m<T><<<grid_for(mn), 256, 0, st>>>(pc, m, n, g.alpha[0], g.alpha[1], g.beta[0], g.beta[1], g.c,
                                                    g.ldc, g.tri);
        count_launch();
        return cudaGetLastError();
    }
    T* ax = w;
    T* bs = ax + 4L * m * k;
    T* cs = bs + 2L * k * n;
    expand_a<T><<<grid_for((long)m * k), 256, 0, st>>>(g.a, g.lda, g.transa, m, k, ax);
    count_launch();
    stack_b<T><<<grid_for((long)k * n), 256, 0, st>>>(g.b, g.ldb, g.transb, k, n, bs);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (g.tri == 0) {
        if ((e = real_gemm(2 * m, n, 2 * k, ax, 2 * m, bs, 2 * k, cs, 2 * m, 0)) != cudaSuccess) return e;
    } else {
        // one triangle: the real and imaginary halves as two m-row products in
        // triangle mode, [Ar, -Ai] [Br; Bi] and [Ai, Ar] [Br; Bi]
        if ((e = real_gemm(m, n, 2 * k, ax, 2 * m, bs, 2 * k, cs, 2 * m, g.tri)) != cudaSuccess) return e;
        if ((e = real_gemm(m, n, 2 * k, ax + m, 2 * m, bs, 2 * k, cs + m, 2 * m, g.tri)) != cudaSuccess) return e;
    }
    combine_expanded<T><<<grid_for((long)m * n), 256, 0, st>>>(cs, m, n, g.alpha[0], g.alpha[1], g.beta[0],
                                                               g.beta[1], g.c, g.ldc, g.tri);
    count_launch();
    return cudaGetLastError();
}

template size_t complex_plane_bytes<double>(int, int, int, int);
template size_t complex_plane_bytes<float>(int, int, int, int);
template cudaError_t complex_gemm<double>(const ComplexArgs<double>&, int, void*, const RealGemm<double>&,
                                          cudaStream_t);
template cudaError_t complex_gemm<float>(const ComplexArgs<float>&, int, void*, const RealGemm<float>&, cudaStream_t);

}  // namespace zb
