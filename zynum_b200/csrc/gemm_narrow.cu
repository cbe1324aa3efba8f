// FP32 GEMM with at most 16 columns (or rows) of C: n <= 16 ("narrow N") or
// m <= 16 ("narrow M").  These shapes are HBM-bound on B200 -- the wide operand
// is read once and each of its elements feeds at most 16 FMAs -- so a 128 x 128
// FFMA tile would spend most of its time on padding.  Both cases are one
// problem, "R outputs x NV vectors":
//
//   y_v(r) = alpha sum_k M(r, k) x_v(k) + beta y_v(r),   v < nv <= 16
//
//   narrow N: R = m, M = op(A), x_v = column v of op(B), y_v = column v of C
//   narrow M: R = n, M = op(B)^T, x_v = row v of op(A),  y_v = row v of C
//
// M is "R-fast" (r contiguous in memory) or "K-fast" (k contiguous); both are
// copied global -> shared in their stored orientation with cp.async (16-byte
// copies when the base and ld allow), so global reads stay coalesced.  A CTA
// owns 128 outputs; its 8 warps take 4 of every 32 k of a stage, each lane
// holds 4 outputs x NV accumulators and reads the x values as shared-memory
// broadcasts.  The warps' partial sums are then added in warp order (fixed, so
// results repeat run to run).  Split K writes partials in C coordinates and a
// second kernel adds them in split order.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kNwThreads = 256;
constexpr int kNwRows = 128;  // outputs per CTA
constexpr int kNwBK = 32;     // k per stage (4 per warp)
constexpr int kNwStages = 4;

struct NarrowArgs {
    int R, K, nv, k_chunk;
    const float* M;  // R-fast: M(r, k) = M[r + k ld]; K-fast: M[k + r ld]
    long ld;
    const float* X;  // x_v(k) = X[k incx + v xs]
    long incx, xs;
    float alpha, beta;
    float* Y;  // y_v(r) = Y[r incy + v ys]
    long incy, ys;
    float* W;  // split z partial of (r, v): W[z wz + r wr + v wv] (C coordinates)
    long wz, wr, wv;
};

template <bool KFAST>
struct NarrowGeom {
    static constexpr int MROWS = KFAST ? kNwRows : kNwBK;   // shared tile rows
    static constexpr int MCOLS = KFAST ? kNwBK : kNwRows;   // contiguous dimension
    static constexpr int MP = MCOLS + 4;                    // pitch: 16-byte rows, conflict-free reads
    static constexpr int MSTAGE = MROWS * MP;
};

template <int NV>
constexpr size_t narrow_smem_bytes(bool kfast) {
    const int mstage = kfast ? NarrowGeom<true>::MSTAGE : NarrowGeom<false>::MSTAGE;
    const size_t pipe = (size_t)kNwStages * (mstage + kNwBK * NV) * sizeof(float);
    const size_t red = (size_t)kNwThreads / 32 * kNwRows * NV * sizeof(float);
    return pipe > red ? pipe : red;
}

template <bool KFAST, int NV, int VEC>
__global__ void __launch_bounds__(kNwThreads, 2) narrow_ffma_kernel(NarrowArgs a) {
    using G = NarrowGeom<KFAST>;
    constexpr int XSTAGE = kNwBK * NV;
    extern __shared__ __align__(16) float nsm[];
    float* Ms = nsm;
    float* Xs = nsm + kNwStages * G::MSTAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = blockIdx.x * kNwRows;
    const int kb = blockIdx.y * a.k_chunk, ke = min(a.K, kb + a.k_chunk);
    const int KT = (ke - kb + kNwBK - 1) / kNwBK;

    auto load_stage = [&](int s, int kt) {
        const int k0 = kb + kt * kNwBK;
        float* ms = Ms + s * G::MSTAGE;
        constexpr int CPR = G::MCOLS / VEC;  // copies per shared row
#pragma unroll
        for (int it = 0; it < G::MROWS * CPR / kNwThreads; ++it) {
            const int q = it * kNwThreads + tid;
            const int row = q / CPR, col = (q % CPR) * VEC;
            int valid;
            const float* src;
            if (KFAST) {  // shared row = output r, columns k
                const int gr = r0 + row, gk = k0 + col;
                valid = gr < a.R ? max(0, min(VEC, ke - gk)) : 0;
                src = a.M + (long)gr * a.ld + gk;
            } else {  // shared row = k, columns r
                const int gk = k0 + row, gr = r0 + col;
                valid = gk < ke ? max(0, min(VEC, a.R - gr)) : 0;
                src = a.M + (long)gk * a.ld + gr;
            }
            const uint32_t dst = smem_u32(ms + row * G::MP + col);
            if (VEC == 4)
                cp_async_16(dst, valid ? src : a.M, valid * 4);
            else
                cp_async_4(dst, valid ? src : a.M, valid * 4);
        }
        float* xs = Xs + s * XSTAGE;
        for (int q = tid; q < XSTAGE; q += kNwThreads) {
            const int kk = q / NV, v = q % NV, gk = k0 + kk;
            const bool ok = gk < ke && v < a.nv;
            cp_async_4(smem_u32(xs + q), ok ? a.X + (long)gk * a.incx + (long)v * a.xs : a.X, ok ? 4 : 0);
        }
    };

    float acc[4][NV];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[i][v] = 0.f;

#pragma unroll
    for (int s = 0; s < kNwStages - 1; ++s) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<kNwStages - 2>();
        __syncthreads();
        {
            const int nk = kt + kNwStages - 1;
            if (nk < KT) load_stage(nk % kNwStages, nk);
            cp_async_commit();
        }
        const float* ms = Ms + (kt % kNwStages) * G::MSTAGE;
        const float* xs = Xs + (kt % kNwStages) * XSTAGE;
        // mv[i][j]: output i of this lane at k = 4 warp + j
        float mv[4][4];
        if (KFAST) {  // outputs lane + 32 i; lanes 36 floats apart: conflict-free 16-byte reads
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 t = *reinterpret_cast<const float4*>(ms + (lane + 32 * i) * G::MP + 4 * warp);
                mv[i][0] = t.x, mv[i][1] = t.y, mv[i][2] = t.z, mv[i][3] = t.w;
            }
        } else {  // outputs 4 lane + i; consecutive 16-byte reads
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float4 t = *reinterpret_cast<const float4*>(ms + (4 * warp + j) * G::MP + 4 * lane);
                mv[0][j] = t.x, mv[1][j] = t.y, mv[2][j] = t.z, mv[3][j] = t.w;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float* xr = xs + (4 * warp + j) * NV;  // the same address in every lane: broadcast
            float xv[NV];
            if constexpr (NV % 4 == 0) {
#pragma unroll
                for (int v = 0; v < NV; v += 4) {
                    const float4 t = *reinterpret_cast<const float4*>(xr + v);
                    xv[v] = t.x, xv[v + 1] = t.y, xv[v + 2] = t.z, xv[v + 3] = t.w;
                }
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) xv[v] = xr[v];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int v = 0; v < NV; ++v) acc[i][v] = fmaf(mv[i][j], xv[v], acc[i][v]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();

    // red[w][v][r]: warp w's partial of output r0 + r, vector v
    float* red = nsm;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = KFAST ? lane + 32 * i : 4 * lane + i;
#pragma unroll
        for (int v = 0; v < NV; ++v) red[(warp * NV + v) * kNwRows + r] = acc[i][v];
    }
    __syncthreads();
    for (int q = tid; q < kNwRows * NV; q += kNwThreads) {
        const int r = q % kNwRows, v = q / kNwRows, gr = r0 + r;
        if (gr >= a.R || v >= a.nv) continue;
        float s = red[v * kNwRows + r];
#pragma unroll
        for (int w = 1; w < kNwThreads / 32; ++w) s += red[(w * NV + v) * kNwRows + r];
        if (a.W) {
            a.W[(long)blockIdx.y * a.wz + (long)gr * a.wr + (long)v * a.wv] = s;
        } else {
            float* yp = a.Y + (long)gr * a.incy + (long)v * a.ys;
            *yp = a.beta == 0.f ? a.alpha * s : fmaf(a.beta, *yp, a.alpha * s);
        }
    }
}

// C(i, j) = alpha sum_z W[z m n + j m + i] + beta C(i, j), splits added in order.
__global__ void narrow_reduce_kernel(int m, int n, int splits, const float* __restrict__ W, float alpha, float beta,
                                     float* __restrict__ C, long ldc) {
    const long total = (long)m * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int i = (int)(q % m), j = (int)(q / m);
        float s = W[q];
        for (int z = 1; z < splits; ++z) s += W[(long)z * total + q];
        float* cp = C + (long)j * ldc + i;
        *cp = beta == 0.f ? alpha * s : fmaf(beta, *cp, alpha * s);
    }
}

template <bool KFAST, int NV, int VEC>
cudaError_t launch_narrow(const NarrowArgs& a, int used, cudaStream_t st) {
    auto kern = narrow_ffma_kernel<KFAST, NV, VEC>;
    const int smem = (int)narrow_smem_bytes<NV>(KFAST);
    cudaError_t e = ensure_dynamic_smem(kern, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.R + kNwRows - 1) / kNwRows, used);
    kern<<<grid, kNwThreads, smem, st>>>(a);
    return cudaSuccess;
}

template <bool KFAST, int VEC>
cudaError_t launch_nv(const NarrowArgs& a, int used, cudaStream_t st) {
    if (a.nv <= 2) return launch_narrow<KFAST, 2, VEC>(a, used, st);
    if (a.nv <= 4) return launch_narrow<KFAST, 4, VEC>(a, used, st);
    if (a.nv <= 8) return launch_narrow<KFAST, 8, VEC>(a, used, st);
    return launch_narrow<KFAST, 16, VEC>(a, used, st);
}

}  // namespace

bool narrow_gemm_applies(int m, int n, int tri) {
    return tri == 0 && ((n <= 16 && m >= 512) || (m <= 16 && n >= 512)) && m > 1 && n > 1;
}

int narrow_split_count(int m, int n, int k, int sm_count) {
    // K split until about eight CTAs per SM are queued (two run per SM, so the
    // last wave is short), each slice >= 256 deep, at most 64 slices, and the
    // partials within kGemvMaxPartials elements.
    const long tiles = n <= 16 ? (m + kNwRows - 1) / kNwRows : (n + kNwRows - 1) / kNwRows;
    const long want = 8L * sm_count;
    if (tiles >= want || k < 1024) return 1;
    long s = (want + tiles - 1) / tiles;
    s = std::min<long>(s, k / 256);
    s = std::min<long>(s, 64);
    s = std::min<long>(s, kGemvMaxPartials / std::max<long>(1, (long)m * n));
    return (int)std::max<long>(1, s);
}

cudaError_t sgemm_narrow(const GemmArgsF32& g, int splits, float* workspace, cudaStream_t st) {
    NarrowArgs a{};
    a.K = g.k;
    a.alpha = g.alpha;
    a.beta = g.beta;
    bool kfast;
    if (g.n <= 16 && g.m >= 512) {  // outputs = rows of C
        a.R = g.m;
        a.nv = g.n;
        a.M = g.a;
        a.ld = g.lda;
        kfast = g.transa != 'N';
        a.X = g.b;
        a.incx = g.transb == 'N' ? 1 : g.ldb;
        a.xs = g.transb == 'N' ? g.ldb : 1;
        a.Y = g.c;
        a.incy = 1;
        a.ys = g.ldc;
        a.wr = 1;
        a.wv = g.m;
    } else {  // outputs = columns of C
        a.R = g.n;
        a.nv = g.m;
        a.M = g.b;
        a.ld = g.ldb;
        kfast = g.transb == 'N';
        a.X = g.a;
        a.incx = g.transa == 'N' ? g.lda : 1;
        a.xs = g.transa == 'N' ? 1 : g.lda;
        a.Y = g.c;
        a.incy = g.ldc;
        a.ys = 1;
        a.wr = g.m;
        a.wv = 1;
    }
    splits = std::max(1, splits);
    int kchunk = (a.K + splits - 1) / splits;
    kchunk = (kchunk + kNwBK - 1) / kNwBK * kNwBK;
    const int used = (a.K + kchunk - 1) / kchunk;
    a.k_chunk = kchunk;
    if (used > 1) {
        if (!workspace) return cudaErrorInvalidValue;
        a.W = workspace;
        a.wz = (long)g.m * g.n;
    }
    const bool vec = reinterpret_cast<uintptr_t>(a.M) % 16 == 0 && a.ld % 4 == 0;
    prof_begin(st);
    cudaError_t e;
    if (kfast)
        e = vec ? launch_nv<true, 4>(a, used, st) : launch_nv<true, 1>(a, used, st);
    else
        e = vec ? launch_nv<false, 4>(a, used, st) : launch_nv<false, 1>(a, used, st);
    if (e != cudaSuccess) return e;
    count_launch();
    prof_end(st);
    if (used > 1) {
        const long total = (long)g.m * g.n;
        const int blocks = (int)std::min<long>((total + 255) / 256, 148L * 8);
        narrow_reduce_kernel<<<blocks, 256, 0, st>>>(g.m, g.n, used, workspace, g.alpha, g.beta, g.c, g.ldc);
        count_launch();
    }
    return cudaGetLastError();
}

}  // namespace zb
