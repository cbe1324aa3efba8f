// Vector-edge routes of GEMM: n == 1 or m == 1 calls are matrix-vector
// products (the reference sends them to its GEMV path, gemm.zig:189-224 and
// :228-240) and are HBM-bound on B200: every matrix element is read once,
// 8 (FP64) or 4 (FP32) bytes for 2 flops.
//
// Two kernels cover every case; M is the matrix, R the outputs, K the reduction:
//   gemv_n: y_r = alpha sum_k M[r + k ld] x_k + beta y_r   (outputs contiguous in M)
//   gemv_t: y_r = alpha sum_k M[k + r ld] x_k + beta y_r   (each output a contiguous dot product)
// n == 1:  op(A) = A -> gemv_n over A (m x k);  op(A) = A^T -> gemv_t over A (k x m).
// m == 1:  op(B) = B -> gemv_t over B (k x n);  op(B) = B^T -> gemv_n over B (n x k);
//          x = row 0 of op(A), y = row 0 of C (stride ldc).
// The matrix is read with 16-byte streaming loads when its base and ld allow.
// Sums run in a fixed order (per-thread column order, then a fixed tree or warp
// order), so results are identical run to run.  When R alone cannot fill the
// GPU the planner splits K over blockIdx.y into partials that a second kernel
// adds in split order.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kGvThreads = 256;
constexpr int kGvWarps = kGvThreads / 32;
constexpr int kGvUnroll = 8;   // gemv_n: columns in flight per thread
constexpr int kGvRowsT = 4;    // gemv_t: outputs per lane group
constexpr int kGvChunk = 256;  // K split granularity (a multiple of every strip)

template <typename T, int VEC>
struct VecOf;
template <>
struct VecOf<double, 1> {
    using type = double;
};
template <>
struct VecOf<double, 2> {
    using type = double2;
};
template <>
struct VecOf<float, 1> {
    using type = float;
};
template <>
struct VecOf<float, 4> {
    using type = float4;
};

// VEC consecutive elements at p (16-byte aligned when VEC > 1), streamed.
template <typename T, int VEC>
__device__ __forceinline__ void load_vec(const T* p, T (&v)[VEC]) {
    using V = typename VecOf<T, VEC>::type;
    const V w = __ldcs(reinterpret_cast<const V*>(p));
    if constexpr (VEC == 1) {
        v[0] = w;
    } else if constexpr (VEC == 2) {
        v[0] = w.x;
        v[1] = w.y;
    } else {
        v[0] = w.x;
        v[1] = w.y;
        v[2] = w.z;
        v[3] = w.w;
    }
}

template <typename T>
__device__ __forceinline__ void store_y(T* y, long incy, int r, T s, T alpha, T beta) {
    T* yp = y + (long)r * incy;
    *yp = beta == T(0) ? alpha * s : fma(beta, *yp, alpha * s);
}

// gemv_n: a block owns 32 * VEC consecutive outputs; lane l holds outputs
// l*VEC .. l*VEC+VEC-1, warp w takes column groups w, w + 8, ... of kGvUnroll
// columns within this block's K chunk; warps are then added in order.
template <typename T, int VEC>
__global__ void __launch_bounds__(kGvThreads)
gemv_n_kernel(int R, int K, int kchunk, const T* __restrict__ M, long ld, const T* __restrict__ x, long incx, T alpha,
              T beta, T* __restrict__ y, long incy, T* __restrict__ part) {
    constexpr int RB = 32 * VEC;
    constexpr int U = kGvUnroll;
    __shared__ T red[kGvWarps][RB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = blockIdx.x * RB + lane * VEC;
    const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
    T acc[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) acc[e] = T(0);
    if (r0 < R) {
        const int nr = min(VEC, R - r0);
        const T* mr = M + r0;
        int k = k0 + U * warp;
        for (; k + U <= k1; k += kGvWarps * U) {
            T v[U][VEC], xv[U];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const T* p = mr + (long)(k + j) * ld;
                if (nr == VEC) {
                    load_vec<T, VEC>(p, v[j]);
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) v[j][e] = e < nr ? p[e] : T(0);
                }
                xv[j] = x[(long)(k + j) * incx];
            }
#pragma unroll
            for (int j = 0; j < U; ++j)
#pragma unroll
                for (int e = 0; e < VEC; ++e) acc[e] = fma(v[j][e], xv[j], acc[e]);
        }
        for (; k < k1; ++k) {  // this warp's last group, cut short by k1
            const T* p = mr + (long)k * ld;
            const T xk = x[(long)k * incx];
#pragma unroll
            for (int e = 0; e < VEC; ++e)
                if (e < nr) acc[e] = fma(p[e], xk, acc[e]);
        }
    }
#pragma unroll
    for (int e = 0; e < VEC; ++e) red[warp][lane * VEC + e] = acc[e];
    __syncthreads();
    for (int i = threadIdx.x; i < RB; i += kGvThreads) {
        const int r = blockIdx.x * RB + i;
        if (r >= R) break;
        T s = red[0][i];
#pragma unroll
        for (int w = 1; w < kGvWarps; ++w) s += red[w][i];
        if (part)
            part[(long)blockIdx.y * R + r] = s;
        else
            store_y(y, incy, r, s, alpha, beta);
    }
}

// gemv_t: a group of LPR lanes owns kGvRowsT consecutive outputs (one
// contiguous K run each; 32 / LPR groups per warp, LPR chosen from K so short
// runs still use 16-byte loads); lane l of a group reads elements l*VEC .. of
// every LPR*VEC strip, two strips in flight, and shares the x values across
// the group's outputs.  Per-output sums close with a butterfly over the group.
template <typename T, int VEC, int LPR>
__global__ void __launch_bounds__(kGvThreads)
gemv_t_kernel(int R, int K, int kchunk, const T* __restrict__ M, long ld, const T* __restrict__ x, long incx, T alpha,
              T beta, T* __restrict__ y, long incy, T* __restrict__ part) {
    constexpr int RW = kGvRowsT;
    constexpr int GPW = 32 / LPR;
    constexpr int STRIP = LPR * VEC;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wrow = (blockIdx.x * kGvWarps + warp) * GPW * RW;
    if (wrow >= R) return;  // whole warp; the kernel has no block-wide barrier
    const int sl = lane % LPR;
    const int rb = wrow + (lane / LPR) * RW;
    const int nr = max(0, min(RW, R - rb));  // 0: an idle group (still joins the shuffles)
    const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
    const T* mc[RW];
#pragma unroll
    for (int i = 0; i < RW; ++i) mc[i] = M + (long)(nr ? rb + min(i, nr - 1) : 0) * ld;
    T acc[RW];
#pragma unroll
    for (int i = 0; i < RW; ++i) acc[i] = T(0);
    int k = k0 + sl * VEC;
    for (; k + STRIP + VEC <= k1; k += 2 * STRIP) {
        T v[2][RW][VEC], xv[2][VEC];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int kk = k + h * STRIP;
#pragma unroll
            for (int i = 0; i < RW; ++i)
                if (i < nr) load_vec<T, VEC>(mc[i] + kk, v[h][i]);
#pragma unroll
            for (int e = 0; e < VEC; ++e) xv[h][e] = x[(long)(kk + e) * incx];
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int i = 0; i < RW; ++i)
                if (i < nr)
#pragma unroll
                    for (int e = 0; e < VEC; ++e) acc[i] = fma(v[h][i][e], xv[h][e], acc[i]);
    }
    if (k + VEC <= k1) {  // one whole strip left for this lane
        T v[RW][VEC], xv[VEC];
#pragma unroll
        for (int i = 0; i < RW; ++i)
            if (i < nr) load_vec<T, VEC>(mc[i] + k, v[i]);
#pragma unroll
        for (int e = 0; e < VEC; ++e) xv[e] = x[(long)(k + e) * incx];
#pragma unroll
        for (int i = 0; i < RW; ++i)
            if (i < nr)
#pragma unroll
                for (int e = 0; e < VEC; ++e) acc[i] = fma(v[i][e], xv[e], acc[i]);
        k += STRIP;
    }
    if (k < k1) {  // fewer than VEC elements left
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            if (k + e >= k1) break;
            const T xk = x[(long)(k + e) * incx];
#pragma unroll
            for (int i = 0; i < RW; ++i)
                if (i < nr) acc[i] = fma(mc[i][k + e], xk, acc[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < RW; ++i) {
#pragma unroll
        for (int o = LPR / 2; o; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    if (sl < nr) {
        T s = acc[0];
#pragma unroll
        for (int i = 1; i < RW; ++i)
            if (sl == i) s = acc[i];
        const int r = rb + sl;
        if (part)
            part[(long)blockIdx.y * R + r] = s;
        else
            store_y(y, incy, r, s, alpha, beta);
    }
}

// y_r = alpha sum_q part[q][r] + beta y_r, partials added in split order.
template <typename T>
__global__ void gemv_reduce_kernel(int R, int splits, const T* __restrict__ part, T alpha, T beta, T* __restrict__ y,
                                   long incy) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        T s = part[r];
        for (int q = 1; q < splits; ++q) s += part[(long)q * R + r];
        store_y(y, incy, r, s, alpha, beta);
    }
}

struct GemvShape {
    bool contiguous_outputs;  // gemv_n when true, gemv_t otherwise
    int R, K;
    const void* M;
    long ld;
    const void* x;
    long incx;
    void* y;
    long incy;
};

template <typename T>
GemvShape gemv_shape(const GemmArgs<T>& g) {
    GemvShape s{};
    s.K = g.k;
    s.y = g.c;
    if (g.n == 1) {
        // x = column 0 of op(B): op = N -> B(0:k, 0), op = T -> B(0, 0:k) with stride ldb
        s.x = g.b;
        s.incx = g.transb == 'N' ? 1 : g.ldb;
        s.incy = 1;
        s.R = g.m;
        s.M = g.a;
        s.ld = g.lda;
        s.contiguous_outputs = g.transa == 'N';
    } else {
        // m == 1: x = row 0 of op(A): op = N -> A(0, 0:k) with stride lda, op = T -> A(0:k, 0)
        s.x = g.a;
        s.incx = g.transa == 'N' ? g.lda : 1;
        s.incy = g.ldc;
        s.R = g.n;
        s.M = g.b;
        s.ld = g.ldb;
        s.contiguous_outputs = g.transb != 'N';
    }
    return s;
}

template <typename T, int VEC, int LPR>
void launch_gemv_t(const GemvShape& s, int kchunk, int used, T alpha, T beta, T* part, cudaStream_t st) {
    const int rb = kGvWarps * (32 / LPR) * kGvRowsT;
    dim3 grid((s.R + rb - 1) / rb, used);
    gemv_t_kernel<T, VEC, LPR><<<grid, kGvThreads, 0, st>>>(s.R, s.K, kchunk, static_cast<const T*>(s.M), s.ld,
                                                            static_cast<const T*>(s.x), s.incx, alpha, beta,
                                                            static_cast<T*>(s.y), s.incy, part);
}

template <typename T, int VEC>
void launch_gemv(const GemvShape& s, int kchunk, int used, T alpha, T beta, T* part, cudaStream_t st) {
    if (s.contiguous_outputs) {
        const int rb = 32 * VEC;
        dim3 grid((s.R + rb - 1) / rb, used);
        gemv_n_kernel<T, VEC><<<grid, kGvThreads, 0, st>>>(s.R, s.K, kchunk, static_cast<const T*>(s.M), s.ld,
                                                           static_cast<const T*>(s.x), s.incx, alpha, beta,
                                                           static_cast<T*>(s.y), s.incy, part);
        return;
    }
    // lanes per output: the widest group that still gives every lane two
    // strips (LPR * VEC elements each) of the K run in flight
    const int run = std::min(s.K, kchunk);
    if (run >= 64 * VEC)
        launch_gemv_t<T, VEC, 32>(s, kchunk, used, alpha, beta, part, st);
    else if (run >= 32 * VEC)
        launch_gemv_t<T, VEC, 16>(s, kchunk, used, alpha, beta, part, st);
    else if (run >= 16 * VEC)
        launch_gemv_t<T, VEC, 8>(s, kchunk, used, alpha, beta, part, st);
    else
        launch_gemv_t<T, VEC, 4>(s, kchunk, used, alpha, beta, part, st);
}

template <typename T>
cudaError_t gemv_run(const GemmArgs<T>& g, int splits, T* workspace, cudaStream_t st) {
    constexpr int VEC = 16 / (int)sizeof(T);
    const GemvShape s = gemv_shape(g);
    splits = std::max(1, splits);
    int kchunk = (s.K + splits - 1) / splits;
    kchunk = (kchunk + kGvChunk - 1) / kGvChunk * kGvChunk;
    const int used = (s.K + kchunk - 1) / kchunk;
    T* part = used > 1 ? workspace : nullptr;
    if (used > 1 && !part) return cudaErrorInvalidValue;
    const bool vec = reinterpret_cast<uintptr_t>(s.M) % 16 == 0 && s.ld % VEC == 0;
    prof_begin(st);
    if (vec)
        launch_gemv<T, VEC>(s, kchunk, used, g.alpha, g.beta, part, st);
    else
        launch_gemv<T, 1>(s, kchunk, used, g.alpha, g.beta, part, st);
    count_launch();
    prof_end(st);
    if (used > 1) {
        const int blocks = std::max(1, std::min((s.R + 255) / 256, 148 * 8));
        gemv_reduce_kernel<T><<<blocks, 256, 0, st>>>(s.R, used, part, g.alpha, g.beta, static_cast<T*>(s.y), s.incy);
        count_launch();
    }
    return cudaGetLastError();
}

}  // namespace

bool gemv_applies(int m, int n, int k, int tri) { return tri == 0 && k >= 1 && (n == 1 || m == 1); }

int gemv_split_count(int rows, int k) {
    // Split K until outputs x splits reaches kGemvSplitTarget (several waves of
    // blocks for every kernel variant, so the last wave's imbalance stays
    // small), each split >= kGvChunk deep and at most 64 of them; the partials
    // stay below kGemvMaxPartials elements.
    if (rows >= kGemvSplitTarget || k < 4 * kGvChunk) return 1;
    long sp = (kGemvSplitTarget + rows - 1) / rows;
    sp = std::min<long>(sp, k / kGvChunk);
    sp = std::min<long>(sp, 64);
    sp = std::min<long>(sp, kGemvMaxPartials / std::max(1, rows));
    return (int)std::max<long>(1, sp);
}

int gemv_used_splits(int k, int splits) {
    splits = std::max(1, splits);
    int kchunk = (k + splits - 1) / splits;
    kchunk = (kchunk + kGvChunk - 1) / kGvChunk * kGvChunk;
    return (k + kchunk - 1) / kchunk;
}

cudaError_t dgemv_route(const GemmArgsF64& g, int splits, double* ws, cudaStream_t st) {
    return gemv_run<double>(g, splits, ws, st);
}
cudaError_t sgemv_route(const GemmArgsF32& g, int splits, float* ws, cudaStream_t st) {
    return gemv_run<float>(g, splits, ws, st);
}

}  // namespace zb
