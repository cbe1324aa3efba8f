// Tall-skinny GEMM: C (m x n) = alpha op(A) (m x k) op(B) (k x n) + beta C for
// n <= 64, k <= 64 and large m (e.g. 131072 x 64 x 64), the reference's
// HBM-bound sweep shape (bench/gemm_sweep.zig) on the packed-SIMD path of
// kernels/shared/matrix_matrix/packed_simd.zig:306.
//
// The generic 128 x 128 / 128 x 64 tiles re-stage op(B) for every output tile
// and run a full K pipeline prologue and epilogue per 128 rows.  Here every
// persistent CTA (two per SM) stages op(B) once (zero-padded to 64 x 64) and
// streams row blocks of op(A) through a two-stage cp.async ring, so the only
// HBM traffic is op(A) once, C once (twice with beta != 0) and op(B) per CTA.
//   FP64: 64-row blocks, DMMA m16n8k8; warp w computes rows 16 (w & 3) .. +15,
//         columns 32 (w >> 2) .. +31 (four n-fragments).
//   FP32: 128-row blocks, FFMA; thread t computes rows 8 (t >> 4) .. +7 and
//         columns 4 (t & 15) .. +3, storing 8 consecutive rows as 16-byte vectors.
// op(A) is staged in its global orientation: [k][128] (m fast) for op = N,
// [128][k] (k fast) for op = T; pitches are 4 mod 16 elements, which keeps
// the fragment loads free of bank conflicts.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kSkK = 64, kSkN = 64, kSkThreads = 256;

template <typename T, bool AKF>
struct SkinnyGeom {
    static constexpr int BM = sizeof(T) == 8 ? 64 : 128;  // rows per block
    // A stage: AKF ? [BM][kSkK + 4] : [kSkK][BM + 4]
    static constexpr int A_ROWS = AKF ? BM : kSkK;
    static constexpr int A_PITCH = AKF ? kSkK + 4 : BM + 4;
    static constexpr int A_STAGE = A_ROWS * A_PITCH;
    static constexpr int B_PITCH = kSkN + 4;  // Bs[k][n]
    static constexpr size_t SMEM = (size_t)(2 * A_STAGE + kSkK * B_PITCH) * sizeof(T);
};

template <typename T>
ZB_DEVICE void cp_el(T* dst, const T* src, bool ok, const T* fallback) {
    if (sizeof(T) == 8)
        cp_async_8(smem_u32(dst), ok ? src : fallback, ok ? 8 : 0);
    else
        cp_async_4(smem_u32(dst), ok ? src : fallback, ok ? 4 : 0);
}

// Stage rows [i0, i0 + BM) of op(A) (all k < K) into one A stage.
template <typename T, bool AKF>
ZB_DEVICE void load_a_block(T* As, const T* __restrict__ A, long lda, int i0, int M, int K) {
    using G = SkinnyGeom<T, AKF>;
    constexpr int kSkM = G::BM;
    if (!AKF) {
        // op(A) = A (m x k, column-major): column kk holds BM contiguous rows
        for (int e = threadIdx.x; e < kSkK * kSkM; e += kSkThreads) {
            const int kk = e / kSkM, i = e % kSkM;
            cp_el(As + kk * G::A_PITCH + i, A + (i0 + i) + (long)kk * lda, kk < K && i0 + i < M, A);
        }
    } else {
        // op(A) = A^T (A is k x m): row i of op(A) is column i of A, k contiguous
        for (int e = threadIdx.x; e < kSkK * kSkM; e += kSkThreads) {
            const int i = e / kSkK, kk = e % kSkK;
            cp_el(As + i * G::A_PITCH + kk, A + kk + (long)(i0 + i) * lda, kk < K && i0 + i < M, A);
        }
    }
    cp_async_commit();
}

template <typename T>
ZB_DEVICE T a_at(const T* As, int i, int kk, int pitch, bool akf) {
    return akf ? As[i * pitch + kk] : As[kk * pitch + i];
}

template <typename T, bool AKF, bool BKF>
__global__ void __launch_bounds__(kSkThreads, 2)
gemm_skinny_kernel(int M, int N, int K, T alpha, const T* __restrict__ A, long lda, const T* __restrict__ B, long ldb,
                   T beta, T* __restrict__ C, long ldc) {
    using G = SkinnyGeom<T, AKF>;
    constexpr int kSkM = G::BM;
    extern __shared__ __align__(16) unsigned char sk_smem[];
    T* As = reinterpret_cast<T*>(sk_smem);
    T* Bs = As + 2 * G::A_STAGE;
    const int nblk = (M + kSkM - 1) / kSkM;
    if ((int)blockIdx.x >= nblk) return;
    // op(B) (k x n) -> Bs[kk][j], zero outside k < K, j < N
    for (int e = threadIdx.x; e < kSkK * kSkN; e += kSkThreads) {
        int kk, j;
        const T* src;
        if (BKF) {  // op(B) = B (k x n, column-major): k contiguous
            j = e / kSkK;
            kk = e % kSkK;
            src = B + kk + (long)j * ldb;
        } else {  // op(B) = B^T (B is n x k): n contiguous
            kk = e / kSkN;
            j = e % kSkN;
            src = B + j + (long)kk * ldb;
        }
        cp_el(Bs + kk * G::B_PITCH + j, src, kk < K && j < N, B);
    }
    load_a_block<T, AKF>(As, A, lda, blockIdx.x * kSkM, M, K);  // commit group 0 holds B and block 0
    const int ksteps = (K + 7) / 8;
    int stage = 0;
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x, stage ^= 1) {
        const int i0 = blk * kSkM;
        if (blk + (int)gridDim.x < nblk) {
            load_a_block<T, AKF>(As + (stage ^ 1) * G::A_STAGE, A, lda, i0 + gridDim.x * kSkM, M, K);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const T* as = As + stage * G::A_STAGE;
        if (sizeof(T) == 8) {
            // ---- FP64: DMMA, warp w -> rows 16 (w & 3) .. +15, columns 32 (w >> 2) .. +31
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
            const int r0 = (warp & 3) * 16, n0 = (warp >> 2) * 32;
            double acc[4][4];
#pragma unroll
            for (int jn = 0; jn < 4; ++jn)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[jn][v] = 0.0;
            for (int s = 0; s < ksteps; ++s) {
                double af[4];
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    af[v] = (double)a_at(as, r0 + g + 8 * (v & 1), s * 8 + t + 4 * (v >> 1), G::A_PITCH, AKF);
#pragma unroll
                for (int jn = 0; jn < 4; ++jn) {
                    double bf[2];
#pragma unroll
                    for (int v = 0; v < 2; ++v) bf[v] = (double)Bs[(s * 8 + t + 4 * v) * G::B_PITCH + n0 + jn * 8 + g];
                    dmma_16x8x8(acc[jn], af, bf);
                }
            }
            // epilogue: c[v0 + 2 v1] at (row g + 8 v1, col 2 t + v0); C reads before stores
            double cin[4][4];
#pragma unroll
            for (int jn = 0; jn < 4; ++jn)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = i0 + r0 + g + 8 * (v >> 1), col = n0 + jn * 8 + 2 * t + (v & 1);
                    cin[jn][v] = (beta != T(0) && row < M && col < N) ? (double)C[row + (long)col * ldc] : 0.0;
                }
#pragma unroll
            for (int jn = 0; jn < 4; ++jn)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = i0 + r0 + g + 8 * (v >> 1), col = n0 + jn * 8 + 2 * t + (v & 1);
                    if (row < M && col < N) {
                        double out = (double)alpha * acc[jn][v];
                        if (beta != T(0)) out = fma((double)beta, cin[jn][v], out);
                        C[row + (long)col * ldc] = (T)out;
                    }
                }
        } else {
            // ---- FP32: FFMA, thread -> rows 8 ty .. 8 ty + 7, columns 4 tx .. 4 tx + 3
            // a warp spans 2 row groups x 16 column groups: the 8 A values of a
            // thread are a broadcast within each half-warp
            const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
            float acc[8][4];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
            for (int kk = 0; kk < K; ++kk) {
                float av[8], bv[4];
#pragma unroll
                for (int i = 0; i < 8; ++i) av[i] = (float)a_at(as, 8 * ty + i, kk, G::A_PITCH, AKF);
#pragma unroll
                for (int j = 0; j < 4; ++j) bv[j] = (float)Bs[kk * G::B_PITCH + 4 * tx + j];
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
            }
            // 8 consecutive rows of a column: two 16-byte accesses when aligned
            const int row0 = i0 + 8 * ty;
            const bool vec = row0 + 8 <= M && (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = 4 * tx + j;
                if (col >= N) break;
                float* cp = reinterpret_cast<float*>(C) + row0 + (long)col * ldc;
                float out[8];
                float cin[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (vec) {
                    if (beta != T(0)) {
                        const float4 c0 = reinterpret_cast<const float4*>(cp)[0], c1 = reinterpret_cast<const float4*>(cp)[1];
                        cin[0] = c0.x; cin[1] = c0.y; cin[2] = c0.z; cin[3] = c0.w;
                        cin[4] = c1.x; cin[5] = c1.y; cin[6] = c1.z; cin[7] = c1.w;
                    }
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        out[i] = beta != T(0) ? fmaf((float)beta, cin[i], (float)alpha * acc[i][j]) : (float)alpha * acc[i][j];
                    reinterpret_cast<float4*>(cp)[0] = make_float4(out[0], out[1], out[2], out[3]);
                    reinterpret_cast<float4*>(cp)[1] = make_float4(out[4], out[5], out[6], out[7]);
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (row0 + i < M && beta != T(0)) cin[i] = cp[i];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (row0 + i < M)
                            cp[i] = beta != T(0) ? fmaf((float)beta, cin[i], (float)alpha * acc[i][j]) : (float)alpha * acc[i][j];
                }
            }
        }
        __syncthreads();  // this stage is refilled by the next iteration's prefetch
    }
}

template <typename T, bool AKF, bool BKF>
cudaError_t launch_skinny(const GemmArgs<T>& g, cudaStream_t st) {
    using G = SkinnyGeom<T, AKF>;
    auto kern = gemm_skinny_kernel<T, AKF, BKF>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)G::SMEM);
    if (e != cudaSuccess) return e;
    static const int sms = [] {
        int dev = 0, n = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    const int nblk = (g.m + G::BM - 1) / G::BM;
    const int grid = std::min(nblk, 2 * sms);  // two CTAs per SM
    prof_begin(st);
    kern<<<grid, kSkThreads, G::SMEM, st>>>(g.m, g.n, g.k, g.alpha, g.a, g.lda, g.b, g.ldb, g.beta, g.c, g.ldc);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

template <typename T>
cudaError_t skinny_dispatch(const GemmArgs<T>& g, cudaStream_t st) {
    const bool akf = g.transa != 'N', bkf = g.transb == 'N';
    if (!akf && bkf) return launch_skinny<T, false, true>(g, st);
    if (!akf && !bkf) return launch_skinny<T, false, false>(g, st);
    if (akf && bkf) return launch_skinny<T, true, true>(g, st);
    return launch_skinny<T, true, false>(g, st);
}

}  // namespace

bool skinny_gemm_applies(int m, int n, int k, int tri) {
    return tri == 0 && n >= 1 && n <= kSkN && k >= 1 && k <= kSkK && m >= 2048;
}

cudaError_t dgemm_skinny(const GemmArgsF64& g, cudaStream_t st) { return skinny_dispatch<double>(g, st); }
cudaError_t sgemm_skinny(const GemmArgsF32& g, cudaStream_t st) { return skinny_dispatch<float>(g, st); }

}  // namespace zb
