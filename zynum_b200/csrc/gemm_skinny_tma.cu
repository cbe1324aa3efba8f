// Tall-skinny FP64 GEMM, TMA-fed and warp-specialised (sm_100a):
// C (m x n) = alpha op(A) (m x k) op(B) (k x n) + beta C for n <= 64,
// k <= 64 and large m (131072 x 64 x 64 in the reference's sweep,
// bench/gemm_sweep.zig, on the packed-SIMD path of
// kernels/shared/matrix_matrix/packed_simd.zig:306 via gemm.zig:168).
//
// At k = n = 64 the product sits at the FP64 ridge (2 k flop per 8-byte
// element of A: 1.07 GFLOP against 134-201 MB), so both the DMMA pipe and
// HBM have to be kept busy.  One persistent CTA per SM stages op(B) once
// (zero-padded to 64 x 64, K-major, 128-byte swizzle) and a producer warp
// streams 64-row blocks of op(A) through a four-stage TMA ring; eight math
// warps each own a 32 x 16 piece of the 64 x 64 block of C, issue its
// beta * C loads before the block's products, run K / 8 DMMA steps and write
// C straight from registers.  There is no block-wide barrier after the
// prologue.  Fragment layouts and the row / k / column bijections are those
// of the 128 x 128 TMA kernel (gemm_f64_tma.cu) on 64-row boxes.
//
// Used for FP64 when op(A)'s base is 16-byte aligned and lda is even (TMA);
// otherwise the cp.async kernel of gemm_skinny.cu runs.
#include <algorithm>
#include <cudaTypedefs.h>

#include "bounded_wait.cuh"
#include "common.cuh"
#include "kernels.h"
#include "ozaki.h"

namespace zb {
namespace {

constexpr int kKBM = 64, kKK = 64, kKN = 64, kKStages = 4;
constexpr int kKMathWarps = 8;                     // 2 (M) x 4 (N) warps of 32 x 16
constexpr int kKThreads = (kKMathWarps + 1) * 32;  // + the TMA producer warp
constexpr int kKABytes = kKBM * kKK * 8;           // 32 KB per stage
constexpr int kKBBytes = kKN * kKK * 8;            // 32 KB, resident
constexpr size_t kKSmem = 1024 + (size_t)kKStages * kKABytes + kKBBytes + 256;
constexpr unsigned long long kKWaitNs = 4000000000ull;

struct SkinnyParams {
    int M, N, K, nblk;
    double alpha, beta;
    const double* B;
    long ldb;
    int b_kfast;  // op(B) = B (k x n, k contiguous); else B^T (n contiguous)
    double* C;
    long ldc;
    int* report;
    unsigned long long wait_ns;
};

// 64-row boxes of 128 B with the 128-byte swizzle (chunk index ^ row mod 8).
ZB_DEVICE uint32_t mn_off64(int mn, int k) {  // [mn / 16][k][16 mn]
    return (uint32_t)((mn >> 4) * 8192 + k * 128 + ((((mn & 15) >> 1) ^ (k & 7)) << 4) + ((mn & 1) << 3));
}
ZB_DEVICE uint32_t k_off64(int mn, int k) {  // [k / 16][mn][16 k]
    return (uint32_t)((k >> 4) * 8192 + mn * 128 + ((((k & 15) >> 1) ^ (mn & 7)) << 4) + ((k & 1) << 3));
}

template <bool A_MN>
__global__ void __launch_bounds__(kKThreads, 1)
dgemm_skinny_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ SkinnyParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sB = smem + kKStages * kKABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kKBBytes);
    uint64_t* empty = full + kKStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kKStages);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // op(B), zero-padded to 64 x 64, K-major and swizzled like the A boxes
    for (int e = threadIdx.x; e < kKK * kKN; e += kKThreads) {
        int kk, j;
        if (P.b_kfast) {
            j = e / kKK;
            kk = e % kKK;
        } else {
            kk = e / kKN;
            j = e % kKN;
        }
        double v = 0.0;
        if (kk < P.K && j < P.N) v = P.b_kfast ? P.B[kk + (long)j * P.ldb] : P.B[j + (long)kk * P.ldb];
        *reinterpret_cast<double*>(sB + k_off64(j, kk)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kKStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kKMathWarps);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const WaitCtl W{abort_flag, nullptr, P.report, P.wait_ns};

    if (warp == kKMathWarps) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            prefetch_tmap(&tmA);
            Issued issued;
            bool ok = true;
            int s = 0;
            uint32_t ph = 0;
            for (int blk = blockIdx.x; blk < P.nblk; blk += gridDim.x) {
                if (!(ok = wait_phase(&empty[s], ph ^ 1u, W, WAIT_PRODUCER_EMPTY_A))) break;
                const uint32_t sa = smem_u32(smem + s * kKABytes);
                const int i0 = blk * kKBM;
                mbar_arrive_expect_tx(&full[s], kKABytes);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    if (A_MN)  // rows k, 16 m per box
                        tma_load_2d(sa + b * 8192, &tmA, &full[s], i0 + 16 * b, 0);
                    else  // rows m, 16 k per box
                        tma_load_2d(sa + b * 8192, &tmA, &full[s], 16 * b, i0);
                }
                issued.note(s, ph);
                if (++s == kKStages) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            if (!ok) issued.drain(full, kKStages, P.wait_ns);
        }
        return;
    }

    // ---------------------------------------------------------- math warps
    const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
    const int g = lane >> 2, t = lane & 3;
    const int ks8 = (P.K + 7) / 8;
    const bool busy1 = wn + 8 < P.N;  // second 8-column fragment inside op(B)
    const bool busy = wn < P.N;
    uint32_t a_off[2][2], b_off[2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int v = 0; v < 2; ++v)
            a_off[i][v] = A_MN ? mn_off64(wm + 16 * i + 2 * g, 2 * t + v) : k_off64(wm + 16 * i + 2 * g + v, 2 * t);
#pragma unroll
    for (int j = 0; j < 2; ++j) b_off[j] = k_off64(wn + 8 * j + ((g >> 1) | ((g & 1) << 2)), 2 * t);
    const bool use_c = P.beta != 0.0;

    bool ok = true;
    int s = 0;
    uint32_t ph = 0;
    for (int blk = blockIdx.x; blk < P.nblk; blk += gridDim.x) {
        const int i0 = blk * kKBM;
        // beta * C loads first: their latency overlaps this block's products
        double cin[2][2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = i0 + wm + 16 * i + 2 * g + (v >> 1);
                    const int col = wn + 8 * j + t + 4 * (v & 1);
                    cin[i][j][v] = (use_c && row < P.M && col < P.N) ? __ldcs(P.C + row + (long)col * P.ldc) : 0.0;
                }
        if (!(ok = wait_phase(&full[s], ph, W, WAIT_MMA_FULL_A))) break;
        const uint8_t* sa = smem + s * kKABytes;
        double acc[2][2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
        if (busy) {
#pragma unroll 2
            for (int q = 0; q < ks8; ++q) {
                const int ks = q * 8;
                const uint32_t mn_step = ks * 128;
                const uint32_t k_xor = ((ks & 15) >> 1) << 4, k_box = (ks >> 4) * 8192;
                double af[2][4], bf[2][2];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    if (A_MN) {
                        const double2 p0 = *reinterpret_cast<const double2*>(sa + a_off[i][0] + mn_step);
                        const double2 p1 = *reinterpret_cast<const double2*>(sa + a_off[i][1] + mn_step);
                        af[i][0] = p0.x, af[i][1] = p0.y, af[i][2] = p1.x, af[i][3] = p1.y;
                    } else {
                        const double2 p0 = *reinterpret_cast<const double2*>(sa + ((a_off[i][0] ^ k_xor) + k_box));
                        const double2 p1 = *reinterpret_cast<const double2*>(sa + ((a_off[i][1] ^ k_xor) + k_box));
                        af[i][0] = p0.x, af[i][2] = p0.y, af[i][1] = p1.x, af[i][3] = p1.y;
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const double2 qv = *reinterpret_cast<const double2*>(sB + ((b_off[j] ^ k_xor) + k_box));
                    bf[j][0] = qv.x, bf[j][1] = qv.y;
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    dmma_16x8x8(acc[i][0], af[i], bf[0]);
                    if (busy1) dmma_16x8x8(acc[i][1], af[i], bf[1]);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (++s == kKStages) {
            s = 0;
            ph ^= 1u;
        }
        // c[v0 + 2 v1]: row 2 g + v1, column t + 4 v0 of the fragment
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = i0 + wm + 16 * i + 2 * g + (v >> 1);
                    const int col = wn + 8 * j + t + 4 * (v & 1);
                    if (row < P.M && col < P.N) {
                        double out = P.alpha * acc[i][j][v];
                        if (use_c) out = fma(P.beta, cin[i][j][v], out);
                        __stcs(P.C + row + (long)col * P.ldc, out);
                    }
                }
    }
    (void)ok;
}

// ---------------------------------------------------------------- FP32
// 128-row blocks of op(A) (32 KB per stage, four stages), op(B) resident as
// [k][64 n] floats; eight FFMA warps, thread (tm = tid mod 16, tn = tid / 16)
// owns 8 rows x columns 4 tn .. 4 tn + 3 of the 128 x 64 block of C.
//   op(A) m-contiguous (boxes of 32 m x 64 k): rows 4 tm + {0..3} and
//     64 + 4 tm + {0..3}, two 16-byte loads per k;
//   op(A) k-contiguous (boxes of 128 m x 32 k): rows tm + 16 i, i < 8, one
//     16-byte load of 4 k per row.
// Either way a quarter-warp reads 8 distinct 16-byte chunks of the swizzle.
constexpr int kFBM = 128;
constexpr int kFABytes = kFBM * kKK * 4;  // 32 KB per stage
constexpr int kFBBytes = kKK * kKN * 4;   // 16 KB, resident
constexpr size_t kFSmem = 1024 + (size_t)kKStages * kFABytes + kFBBytes + 256;

struct SkinnyParamsF {
    int M, N, K, nblk;
    float alpha, beta;
    const float* B;
    long ldb;
    int b_kfast;
    float* C;
    long ldc;
    int* report;
    unsigned long long wait_ns;
};

template <bool A_MN>
ZB_DEVICE int f32_row(int tm, int i) {
    return A_MN ? ((i < 4) ? 4 * tm + i : 64 + 4 * tm + (i - 4)) : tm + 16 * i;
}

template <bool A_MN>
__global__ void __launch_bounds__(kKThreads, 1)
sgemm_skinny_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ SkinnyParamsF P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float* sB = reinterpret_cast<float*>(smem + kKStages * kFABytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kKStages * kFABytes + kFBBytes);
    uint64_t* empty = full + kKStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kKStages);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int e = threadIdx.x; e < kKK * kKN; e += kKThreads) {
        int kk, j;
        if (P.b_kfast) {
            j = e / kKK;
            kk = e % kKK;
        } else {
            kk = e / kKN;
            j = e % kKN;
        }
        float v = 0.f;
        if (kk < P.K && j < P.N) v = P.b_kfast ? P.B[kk + (long)j * P.ldb] : P.B[j + (long)kk * P.ldb];
        sB[kk * kKN + j] = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kKStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kKMathWarps);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const WaitCtl W{abort_flag, nullptr, P.report, P.wait_ns};

    if (warp == kKMathWarps) {
        if (lane == 0) {
            prefetch_tmap(&tmA);
            Issued issued;
            bool ok = true;
            int s = 0;
            uint32_t ph = 0;
            for (int blk = blockIdx.x; blk < P.nblk; blk += gridDim.x) {
                if (!(ok = wait_phase(&empty[s], ph ^ 1u, W, WAIT_PRODUCER_EMPTY_A))) break;
                const uint32_t sa = smem_u32(smem + s * kFABytes);
                const int i0 = blk * kFBM;
                mbar_arrive_expect_tx(&full[s], kFABytes);
                if (A_MN) {  // 4 boxes of 64 k-rows x 32 m
#pragma unroll
                    for (int b = 0; b < 4; ++b) tma_load_2d(sa + b * 8192, &tmA, &full[s], i0 + 32 * b, 0);
                } else {  // 2 boxes of 128 m-rows x 32 k
#pragma unroll
                    for (int b = 0; b < 2; ++b) tma_load_2d(sa + b * 16384, &tmA, &full[s], 32 * b, i0);
                }
                issued.note(s, ph);
                if (++s == kKStages) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            if (!ok) issued.drain(full, kKStages, P.wait_ns);
        }
        return;
    }

    const int tm = threadIdx.x & 15, tn = threadIdx.x >> 4;
    const bool busy = 4 * tn < P.N;
    const bool use_c = P.beta != 0.0f;
    bool ok = true;
    int s = 0;
    uint32_t ph = 0;
    for (int blk = blockIdx.x; blk < P.nblk; blk += gridDim.x) {
        const int i0 = blk * kFBM;
        float cin[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int row = i0 + f32_row<A_MN>(tm, i), col = 4 * tn + j;
                cin[i][j] = (use_c && row < P.M && col < P.N) ? __ldcs(P.C + row + (long)col * P.ldc) : 0.f;
            }
        if (!(ok = wait_phase(&full[s], ph, W, WAIT_MMA_FULL_A))) break;
        const uint8_t* sa = smem + s * kFABytes;
        float acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
        if (busy) {
            if (A_MN) {
                // element (m, k) at (m / 32) * 8192 + k * 128 + (((m mod 32) / 4 ^ k mod 8) * 16) + (m mod 4) * 4
                const uint32_t lo = (uint32_t)((tm >> 3) * 8192), hi = lo + 2 * 8192;
#pragma unroll 4
                for (int k = 0; k < P.K; ++k) {
                    const uint32_t chunk = (uint32_t)(((tm & 7) ^ (k & 7)) << 4) + k * 128;
                    const float4 a0 = *reinterpret_cast<const float4*>(sa + lo + chunk);
                    const float4 a1 = *reinterpret_cast<const float4*>(sa + hi + chunk);
                    const float4 bv = *reinterpret_cast<const float4*>(sB + k * kKN + 4 * tn);
                    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                    const float bw[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
                    for (int i = 0; i < 8; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bw[j], acc[i][j]);
                }
            } else {
                // element (m, k) at (k / 32) * 16384 + m * 128 + (((k mod 32) / 4 ^ m mod 8) * 16) + (k mod 4) * 4
#pragma unroll 2
                for (int kq = 0; kq < (P.K + 3) / 4; ++kq) {
                    const uint32_t box = (uint32_t)((kq >> 3) * 16384), c = (uint32_t)(((kq & 7) ^ (tm & 7)) << 4);
                    float4 a[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        a[i] = *reinterpret_cast<const float4*>(sa + box + (tm + 16 * i) * 128 + c);
                    float4 b[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) b[u] = *reinterpret_cast<const float4*>(sB + (4 * kq + u) * kKN + 4 * tn);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float ak[4] = {a[i].x, a[i].y, a[i].z, a[i].w};
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            acc[i][0] = fmaf(ak[u], b[u].x, acc[i][0]);
                            acc[i][1] = fmaf(ak[u], b[u].y, acc[i][1]);
                            acc[i][2] = fmaf(ak[u], b[u].z, acc[i][2]);
                            acc[i][3] = fmaf(ak[u], b[u].w, acc[i][3]);
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (++s == kKStages) {
            s = 0;
            ph ^= 1u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int col = 4 * tn + j;
            if (col >= P.N) break;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int row = i0 + f32_row<A_MN>(tm, i);
                if (row < P.M) {
                    float out = P.alpha * acc[i][j];
                    if (use_c) out = fmaf(P.beta, cin[i][j], out);
                    __stcs(P.C + row + (long)col * P.ldc, out);
                }
            }
        }
    }
    (void)ok;
}

// op(A)'s tensor map: 128-byte wide boxes (16 doubles / 32 floats) of
// `box_outer` rows in its global orientation, 128-byte swizzle, zero fill.
template <typename T>
cudaError_t make_a_map(CUtensorMap* map, const GemmArgs<T>& g, int box_outer) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return cudaErrorNotSupported;
    const bool a_mn = g.transa == 'N';
    cuuint64_t dims[2] = {(cuuint64_t)(a_mn ? g.m : g.k), (cuuint64_t)(a_mn ? g.k : g.m)};
    cuuint64_t strides[1] = {(cuuint64_t)(g.lda * sizeof(T))};
    cuuint32_t box[2] = {(cuuint32_t)(128 / sizeof(T)), (cuuint32_t)box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                     const_cast<T*>(g.a), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int sm_count_skinny() {
    static const int sms = [] {
        int dev = 0, n = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    return sms;
}

}  // namespace

bool dgemm_skinny_tma_applies(const GemmArgsF64& g) {
    return reinterpret_cast<uintptr_t>(g.a) % 16 == 0 && g.lda % 2 == 0 && tensor_map_encoder() != nullptr;
}

bool sgemm_skinny_tma_applies(const GemmArgsF32& g) {
    return reinterpret_cast<uintptr_t>(g.a) % 16 == 0 && g.lda % 4 == 0 && tensor_map_encoder() != nullptr;
}

cudaError_t sgemm_skinny_tma(const GemmArgsF32& g, cudaStream_t st) {
    const bool a_mn = g.transa == 'N';
    CUtensorMap ma;
    cudaError_t e = make_a_map(&ma, g, a_mn ? 64 : kFBM);
    if (e != cudaSuccess) return e;
    SkinnyParamsF P{};
    P.M = g.m;
    P.N = g.n;
    P.K = g.k;
    P.nblk = (g.m + kFBM - 1) / kFBM;
    P.alpha = g.alpha;
    P.beta = g.beta;
    P.B = g.b;
    P.ldb = g.ldb;
    P.b_kfast = g.transb == 'N';
    P.C = g.c;
    P.ldc = g.ldc;
    P.wait_ns = kKWaitNs;
    if ((e = wait_report_word(&P.report)) != cudaSuccess) return e;
    const int grid = std::min(P.nblk, sm_count_skinny());
    auto kern = a_mn ? sgemm_skinny_tma_kernel<true> : sgemm_skinny_tma_kernel<false>;
    if ((e = ensure_dynamic_smem(kern, (int)kFSmem)) != cudaSuccess) return e;
    prof_begin(st);
    kern<<<grid, kKThreads, kFSmem, st>>>(ma, P);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

cudaError_t dgemm_skinny_tma(const GemmArgsF64& g, cudaStream_t st) {
    CUtensorMap ma;
    cudaError_t e = make_a_map(&ma, g, 64);
    if (e != cudaSuccess) return e;
    SkinnyParams P{};
    P.M = g.m;
    P.N = g.n;
    P.K = g.k;
    P.nblk = (g.m + kKBM - 1) / kKBM;
    P.alpha = g.alpha;
    P.beta = g.beta;
    P.B = g.b;
    P.ldb = g.ldb;
    P.b_kfast = g.transb == 'N';
    P.C = g.c;
    P.ldc = g.ldc;
    P.wait_ns = kKWaitNs;
    if ((e = wait_report_word(&P.report)) != cudaSuccess) return e;
    const int grid = std::min(P.nblk, sm_count_skinny());
    auto kern = g.transa == 'N' ? dgemm_skinny_tma_kernel<true> : dgemm_skinny_tma_kernel<false>;
    if ((e = ensure_dynamic_smem(kern, (int)kKSmem)) != cudaSuccess) return e;
    prof_begin(st);
    kern<<<grid, kKThreads, kKSmem, st>>>(ma, P);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

}  // namespace zb
