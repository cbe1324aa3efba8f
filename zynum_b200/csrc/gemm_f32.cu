// Native FP32 GEMM (SGEMM) for sm_100a.
//
//   C = alpha * op(A) * op(B) + beta * C     (column-major, any lda/ldb/ldc)
//
// Replaces the f32 instantiation of the reference's packed-SIMD body
// (kernels/shared/matrix_matrix/packed_simd.zig:306, x86 AVX-512 tile
// 16 lanes x 2 row groups x 12 columns, packed_params.zig:45-66).
//
// IEEE FP32 has no exact tensor-core kind (kind::tf32 drops mantissa bits), so
// the native SGEMM is a CUDA-core FFMA kernel: 128 x 128 block tile, 256
// threads, an 8 x 8 register tile per thread split into two 4-row and two
// 4-column halves so that every shared load is a conflict-free float4.
// Operands are staged with cp.async; a K-fast global operand (op = T for A,
// op = N for B) is transposed on the fly by per-element copies.
#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kBM = 128, kBN = 128, kBK = 16, kStages = 3, kThreads = 256;
constexpr int kPitch = 128 + 4;  // floats per shared row ([k][mn], mn fast)

// Copy a kBK x 128 tile (rows k, columns mn) into shared memory.
// MN_FAST: global element (mn, k) at base[mn + k*ld]; else at base[k + mn*ld].
template <bool MN_FAST, int VEC>
ZB_DEVICE void load_tile_f32(float* s, const float* __restrict__ base, long ld, int mn0, int k0, int mn_lim,
                             int k_lim) {
    if (MN_FAST) {
        constexpr int CPR = 128 / VEC;
#pragma unroll
        for (int it = 0; it < (kBK * CPR) / kThreads; ++it) {
            int q = it * kThreads + threadIdx.x;
            int kk = q / CPR, mm = (q % CPR) * VEC;
            int gk = k0 + kk, gm = mn0 + mm;
            int valid = 0;
            if (gk < k_lim) {
                valid = mn_lim - gm;
                valid = valid < 0 ? 0 : (valid > VEC ? VEC : valid);
            }
            const float* src = valid ? base + (long)gk * ld + gm : base;
            uint32_t dst = smem_u32(s + kk * kPitch + mm);
            if (VEC == 4)
                cp_async_16(dst, src, valid * 4);
            else
                cp_async_4(dst, src, valid * 4);
        }
    } else {
        // K-fast: consecutive threads walk k (contiguous in global), then mn.
#pragma unroll
        for (int it = 0; it < (kBK * 128) / kThreads; ++it) {
            int q = it * kThreads + threadIdx.x;
            int kk = q % kBK, mm = q / kBK;
            int gk = k0 + kk, gm = mn0 + mm;
            bool ok = gk < k_lim && gm < mn_lim;
            const float* src = ok ? base + (long)gm * ld + gk : base;
            cp_async_4(smem_u32(s + kk * kPitch + mm), src, ok ? 4 : 0);
        }
    }
}

template <bool A_MNFAST, bool B_MNFAST, int VEC, bool PARTIAL>
__global__ void __launch_bounds__(kThreads, 2)
sgemm_ffma_kernel(int M, int N, int K, int k_chunk, float alpha, const float* __restrict__ A, long lda,
                  const float* __restrict__ B, long ldb, float beta, float* __restrict__ C, long ldc,
                  float* __restrict__ W, int tri) {
    extern __shared__ __align__(128) float smf[];
    float* As = smf;
    float* Bs = smf + kStages * kBK * kPitch;

    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    // triangle mode: skip tiles that hold no element of the stored triangle
    if ((tri == 1 && m0 > n0 + kBN - 1) || (tri == 2 && m0 + kBM - 1 < n0)) return;
    const int kb = blockIdx.z * k_chunk;
    const int ke = min(K, kb + k_chunk);
    const int KT = (ke - kb + kBK - 1) / kBK;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    auto load_stage = [&](int stage, int kt) {
        int k0 = kb + kt * kBK;
        load_tile_f32<A_MNFAST, (A_MNFAST ? VEC : 1)>(As + stage * kBK * kPitch, A, lda, m0, k0, M, ke);
        load_tile_f32<B_MNFAST, (B_MNFAST ? VEC : 1)>(Bs + stage * kBK * kPitch, B, ldb, n0, k0, N, ke);
    };

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        {
            int nk = kt + kStages - 1;
            if (nk < KT) load_stage(nk % kStages, nk);
            cp_async_commit();
        }
        const float* as = As + (kt % kStages) * kBK * kPitch;
        const float* bs = Bs + (kt % kStages) * kBK * kPitch;
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            float a[8], b[8];
            *reinterpret_cast<float4*>(a) = *reinterpret_cast<const float4*>(as + kk * kPitch + ty * 4);
            *reinterpret_cast<float4*>(a + 4) = *reinterpret_cast<const float4*>(as + kk * kPitch + 64 + ty * 4);
            *reinterpret_cast<float4*>(b) = *reinterpret_cast<const float4*>(bs + kk * kPitch + tx * 4);
            *reinterpret_cast<float4*>(b + 4) = *reinterpret_cast<const float4*>(bs + kk * kPitch + 64 + tx * 4);
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
        if (col >= N) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
            if (row >= M) continue;
            if (tri == 1 ? row > col : (tri == 2 && row < col)) continue;
            if (PARTIAL) {
                W[(long)blockIdx.z * M * N + (long)col * M + row] = acc[i][j];
            } else {
                float* cp = C + (long)col * ldc + row;
                float out = alpha * acc[i][j];
                if (beta != 0.f) out = fmaf(beta, *cp, out);
                *cp = out;
            }
        }
    }
}

__global__ void sgemm_splitk_reduce(int M, int N, int splits, const float* __restrict__ W, float alpha, float beta,
                                    float* __restrict__ C, long ldc, int tri) {
    long total = (long)M * N;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        int row = (int)(q % M), col = (int)(q / M);
        if (tri == 1 ? row > col : (tri == 2 && row < col)) continue;
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += W[(long)z * total + q];
        float* cp = C + (long)col * ldc + row;
        float out = alpha * s;
        if (beta != 0.f) out = fmaf(beta, *cp, out);
        *cp = out;
    }
}

template <bool AM, bool BM_, int VEC, bool PARTIAL>
cudaError_t launch_f32(const GemmArgsF32& g, int splits, int k_chunk, float* W, cudaStream_t st) {
    constexpr size_t SMEM = (size_t)2 * kStages * kBK * kPitch * sizeof(float);
    auto kern = sgemm_ffma_kernel<AM, BM_, VEC, PARTIAL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if (e != cudaSuccess) return e;
    dim3 grid((g.m + kBM - 1) / kBM, (g.n + kBN - 1) / kBN, splits);
    prof_begin(st);
    kern<<<grid, kThreads, SMEM, st>>>(g.m, g.n, g.k, k_chunk, g.alpha, g.a, g.lda, g.b, g.ldb, g.beta, g.c, g.ldc, W,
                                       g.tri);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

template <bool PARTIAL>
cudaError_t dispatch_f32(const GemmArgsF32& g, int vec, int splits, int k_chunk, float* W, cudaStream_t st) {
    // A is MN-fast when stored untransposed; B is MN-fast when stored transposed.
    const bool am = g.transa == 'N', bm = g.transb != 'N';
#define ZB_CASE(AM, BMF, V) \
    if (am == AM && bm == BMF && vec == V) return launch_f32<AM, BMF, V, PARTIAL>(g, splits, k_chunk, W, st);
    ZB_CASE(false, false, 1) ZB_CASE(false, true, 1) ZB_CASE(true, false, 1) ZB_CASE(true, true, 1)
    ZB_CASE(false, true, 4) ZB_CASE(true, false, 4) ZB_CASE(true, true, 4)
#undef ZB_CASE
    if (!am && !bm) return launch_f32<false, false, 1, PARTIAL>(g, splits, k_chunk, W, st);
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t sgemm_native(const GemmArgsF32& g, const GemmPlan& plan, float* workspace, cudaStream_t st) {
    // 16-byte copies need 16-byte aligned bases and ld % 4 == 0 on every MN-fast operand.
    bool aligned = true;
    if (g.transa == 'N') aligned = aligned && (reinterpret_cast<uintptr_t>(g.a) % 16 == 0) && (g.lda % 4 == 0);
    if (g.transb != 'N') aligned = aligned && (reinterpret_cast<uintptr_t>(g.b) % 16 == 0) && (g.ldb % 4 == 0);
    const int vec = aligned ? 4 : 1;
    const int splits = plan.splits < 1 ? 1 : plan.splits;
    int k_chunk = (g.k + splits - 1) / splits;
    k_chunk = (k_chunk + kBK - 1) / kBK * kBK;
    const int used = (g.k + k_chunk - 1) / k_chunk;
    if (used > 1) {
        if (!workspace) return cudaErrorInvalidValue;
        cudaError_t e = dispatch_f32<true>(g, vec, used, k_chunk, workspace, st);
        if (e != cudaSuccess) return e;
        long total = (long)g.m * g.n;
        int blocks = (int)((total + 255) / 256);
        if (blocks > 148 * 16) blocks = 148 * 16;
        sgemm_splitk_reduce<<<blocks, 256, 0, st>>>(g.m, g.n, used, workspace, g.alpha, g.beta, g.c, g.ldc, g.tri);
        count_launch();
        return cudaGetLastError();
    }
    return dispatch_f32<false>(g, vec, 1, k_chunk, nullptr, st);
}

}  // namespace zb
