// Tall-skinny GEMM, TMA-fed (sm_100a):
// C (m x n) = alpha op(A) (m x k) op(B) (k x n) + beta C for n <= 64,
// k <= 64 and large m (131072 x 64 x 64 in the reference's sweep,
// bench/gemm_sweep.zig, on the packed-SIMD path of
// kernels/shared/matrix_matrix/packed_simd.zig:306 via gemm.zig:168).
//
// At k = n = 64 the product sits at the ridge of both pipes (2 k flop per
// element of op(A)), so the math pipe has to keep working while HBM streams.
// One persistent CTA of sixteen warps per SM stages op(B) once (zero-padded
// to 64 x 64).  The warps form four independent groups of four, one warp of
// each group per SM sub-partition; group g takes the CTA's row blocks g,
// g + 4, ... and owns its own shared-memory stages, so the groups drift apart
// and one group's loads and epilogue overlap the others' products.  There is
// no producer warp: the group's first lane issues the group's TMA loads
// (128-byte swizzle, zero fill past m and k) as soon as its four warps are
// done with a stage, and the group's warps leave together through one
// bar.red.and per block (bounded mbarrier waits; an abort drains the loads).
//
// FP64: 32-row blocks, two stages per group (one block computed while the
// next lands), DMMA m16n8k8 with each warp a 16 x 32 piece of the block;
// fragment layouts and row / k / column bijections as in the 128 x 128 TMA
// kernel (gemm_f64_tma.cu); beta * C is read into registers before the
// block's products and C leaves by 16-byte streaming stores.  FP32: 128-row
// blocks, one stage per group, FFMA with each thread an 8 x 8 register tile
// fed by 16-byte shared loads.
//
// Measured at 131072 x 64 x 64 (timed in CUDA graphs) against cuBLAS on the
// same layout: FP64 47.5 / 57.7 us (beta 0 / 1; cuBLAS 48.4 / 55.8), FP32
// 35.1 / 36.5 us (cuBLAS 30.1 / 33.5).  Variants measured slower: a
// dedicated producer warp with one or two groups of eight math warps (the
// DMMA pipe idled while the lock-stepped warps ran their epilogues), TMA
// stores of C from shared memory (the next load had to wait for the store to
// read the stage), and L2 prefetches of C's blocks ahead of the epilogue.
//
// Used when op(A)'s base is 16-byte aligned and its leading dimension a
// multiple of 16 bytes (TMA); otherwise the cp.async kernel of
// gemm_skinny.cu runs.
#include <algorithm>
#include <cudaTypedefs.h>

#include "bounded_wait.cuh"
#include "common.cuh"
#include "kernels.h"
#include "ozaki.h"

namespace zb {
namespace {

constexpr int kKK = 64, kKN = 64;
constexpr int kGroups = 4, kGroupWarps = 4, kGroupStages = 2;  // group g owns stages 2 g, 2 g + 1
constexpr int kStagesAll = kGroups * kGroupStages;
constexpr int kKThreads = kGroups * kGroupWarps * 32;
constexpr int kKBM = 32;                                    // FP64 rows per block
constexpr int kKABytes = kKBM * kKK * 8;                    // 16 KB per stage
constexpr int kKBBytes = kKN * kKK * 8;                     // 32 KB, resident
constexpr size_t kKSmem = 1024 + (size_t)kStagesAll * kKABytes + kKBBytes + 256;
constexpr unsigned long long kKWaitNs = 4000000000ull;
static_assert(kKK * kKN % kKThreads == 0, "op(B) staging: whole elements per thread");

// Named barrier 1 + grp over the group's four warps; true iff every thread passed `ok`.
ZB_DEVICE bool group_bar_and(int grp, bool ok) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(1 + grp), "n"(kGroupWarps * 32)
        : "memory");
    return r != 0;
}

// Loads row block `blk` (rows blk bm ..) of op(A) into a stage: one TMA
// transaction of `stage_bytes`, issued by the calling thread through `boxes`.
template <typename BoxFn>
ZB_DEVICE void feed_stage(uint64_t* bar, uint32_t stage, int stage_bytes, int blk, int bm, int nblk, BoxFn boxes) {
    if (blk >= nblk) return;
    mbar_arrive_expect_tx(bar, (uint32_t)stage_bytes);
    boxes(stage, bar, blk * bm);
}

struct SkinnyParams {
    int M, N, K, nblk;
    double alpha, beta;
    const double* B;
    long ldb;
    int b_kfast;  // op(B) = B (k x n, k contiguous); else B^T (n contiguous)
    int vec_c;    // C 16-byte aligned with an even ldc: row pairs move as double2
    double* C;
    long ldc;
    int* report;
    unsigned long long wait_ns;
};

// 128-byte swizzled boxes (16-byte chunk index ^ row mod 8):
//   mn_off: op(A) / op(B) m-contiguous, boxes of 16 mn x 64 k: [mn / 16][k][16 mn]
//   k_off<R>: k-contiguous, boxes of R rows x 16 k: [k / 16][R rows][16 k]
ZB_DEVICE uint32_t mn_off(int mn, int k) {
    return (uint32_t)((mn >> 4) * 8192 + k * 128 + ((((mn & 15) >> 1) ^ (k & 7)) << 4) + ((mn & 1) << 3));
}
template <int R>
ZB_DEVICE uint32_t k_off(int mn, int k) {
    return (uint32_t)((k >> 4) * (R * 128) + mn * 128 + ((((k & 15) >> 1) ^ (mn & 7)) << 4) + ((k & 1) << 3));
}

// FP64: group g takes the CTA's row blocks g, g + 4, ... (32 rows each) and
// holds two of them in flight, one being computed while the next one's TMA
// load lands.  Its four warps each own 16 rows x 32 columns of the block
// (2 x 2 warps): four independent 16 x 8 DMMA accumulators per warp, and
// sixteen per sub-partition with the four groups.
template <bool A_MN, bool USE_C>
__global__ void __launch_bounds__(kKThreads, 1)
dgemm_skinny_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ SkinnyParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sB = smem + kStagesAll * kKABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kKBBytes);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(full + kStagesAll);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / kGroupWarps, wq = warp % kGroupWarps;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStagesAll; ++s) mbar_init(&full[s], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const WaitCtl W{abort_flag, nullptr, P.report, P.wait_ns};
    uint8_t* const stage0 = smem + grp * kGroupStages * kKABytes;
    auto boxes = [&](uint32_t st, uint64_t* bar, int i0) {
        if (A_MN) {  // 2 boxes of 64 k-rows x 16 m
#pragma unroll
            for (int b = 0; b < kKBM / 16; ++b) tma_load_2d(st + b * 8192, &tmA, bar, i0 + 16 * b, 0);
        } else {  // 4 boxes of 32 m-rows x 16 k
#pragma unroll
            for (int b = 0; b < kKK / 16; ++b) tma_load_2d(st + b * (kKBM * 128), &tmA, bar, 16 * b, i0);
        }
    };
    const int step = kGroups * gridDim.x;
    const int blk0 = blockIdx.x + grp * gridDim.x;
    if (wq == 0 && lane == 0) {
        prefetch_tmap(&tmA);
#pragma unroll
        for (int q = 0; q < kGroupStages; ++q)
            feed_stage(&full[grp * kGroupStages + q], smem_u32(stage0 + q * kKABytes), kKABytes, blk0 + q * step, kKBM,
                       P.nblk, boxes);
    }

    // op(B), zero-padded to 64 x 64, K-major and swizzled like the k-contiguous A boxes;
    // every thread's loads are issued before its stores (one memory round trip)
    {
        double v[kKK * kKN / kKThreads];
#pragma unroll
        for (int r = 0; r < kKK * kKN / kKThreads; ++r) {
            const int e = threadIdx.x + r * kKThreads;
            const int j = P.b_kfast ? e / kKK : e % kKN, kk = P.b_kfast ? e % kKK : e / kKN;
            v[r] = (kk < P.K && j < P.N) ? (P.b_kfast ? P.B[kk + (long)j * P.ldb] : P.B[j + (long)kk * P.ldb]) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < kKK * kKN / kKThreads; ++r) {
            const int e = threadIdx.x + r * kKThreads;
            const int j = P.b_kfast ? e / kKK : e % kKN, kk = P.b_kfast ? e % kKK : e / kKN;
            *reinterpret_cast<double*>(sB + k_off<kKN>(j, kk)) = v[r];
        }
    }
    __syncthreads();

    const int wm = (wq >> 1) * 16, wn = (wq & 1) * 32;
    const int g = lane >> 2, t = lane & 3;
    const int ks8 = (P.K + 7) / 8;
    const int nfrag = max(0, min(4, (P.N - wn + 7) / 8));  // 8-column fragments inside op(B)
    uint32_t a_off[2], b_off[4];
#pragma unroll
    for (int v = 0; v < 2; ++v) a_off[v] = A_MN ? mn_off(wm + 2 * g, 2 * t + v) : k_off<kKBM>(wm + 2 * g + v, 2 * t);
#pragma unroll
    for (int j = 0; j < 4; ++j) b_off[j] = k_off<kKN>(wn + 8 * j + ((g >> 1) | ((g & 1) << 2)), 2 * t);

    bool ok = true;
    int n = 0;
    // acc[j][v0 + 2 v1]: row 2 g + v1 of the warp's 16 rows, column t + 4 v0 of fragment j
    for (int blk = blk0; blk < P.nblk; blk += step, ++n) {
        const int q = n & (kGroupStages - 1);
        const uint32_t ph = (uint32_t)(n / kGroupStages) & 1u;
        const uint8_t* sa = stage0 + q * kKABytes;
        const int row = blk * kKBM + wm + 2 * g;
        // beta * C loads first: their latency overlaps this block's products
        double cin[4][2][2];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v0 = 0; v0 < 2; ++v0) {
                const int col = wn + 8 * j + t + 4 * v0;
                const double* p = P.C + row + (long)col * P.ldc;
                double x0 = 0.0, x1 = 0.0;
                if (USE_C && col < P.N) {
                    if (P.vec_c && row + 1 < P.M) {
                        const double2 x = __ldcs(reinterpret_cast<const double2*>(p));
                        x0 = x.x, x1 = x.y;
                    } else {
                        if (row < P.M) x0 = __ldcs(p);
                        if (row + 1 < P.M) x1 = __ldcs(p + 1);
                    }
                }
                cin[j][v0][0] = x0;
                cin[j][v0][1] = x1;
            }
        double acc[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[j][v] = 0.0;
        ok = wait_phase(&full[grp * kGroupStages + q], ph, W, WAIT_MMA_FULL_A);
        if (ok && nfrag > 0) {
#pragma unroll 4
            for (int kq = 0; kq < ks8; ++kq) {
                const int ks = kq * 8;
                const uint32_t k_xor = ((ks & 15) >> 1) << 4, k_box = (ks >> 4) * (kKBM * 128),
                               b_box = (ks >> 4) * (kKN * 128);
                double af[4], bf[4][2];
                if (A_MN) {
                    const double2 p0 = *reinterpret_cast<const double2*>(sa + a_off[0] + ks * 128);
                    const double2 p1 = *reinterpret_cast<const double2*>(sa + a_off[1] + ks * 128);
                    af[0] = p0.x, af[1] = p0.y, af[2] = p1.x, af[3] = p1.y;
                } else {
                    const double2 p0 = *reinterpret_cast<const double2*>(sa + ((a_off[0] ^ k_xor) + k_box));
                    const double2 p1 = *reinterpret_cast<const double2*>(sa + ((a_off[1] ^ k_xor) + k_box));
                    af[0] = p0.x, af[2] = p0.y, af[1] = p1.x, af[3] = p1.y;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double2 qv = *reinterpret_cast<const double2*>(sB + ((b_off[j] ^ k_xor) + b_box));
                    bf[j][0] = qv.x, bf[j][1] = qv.y;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (j < nfrag) dmma_16x8x8(acc[j], af, bf[j]);
            }
        }
        // the group's four warps are done with the stage (or leave together)
        if (!(ok = group_bar_and(grp, ok))) break;
        if (wq == 0 && lane == 0)
            feed_stage(&full[grp * kGroupStages + q], smem_u32(sa), kKABytes, blk + kGroupStages * step, kKBM,
                       P.nblk, boxes);
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v0 = 0; v0 < 2; ++v0) {
                const int col = wn + 8 * j + t + 4 * v0;
                if (col >= P.N) continue;
                double o0 = P.alpha * acc[j][v0], o1 = P.alpha * acc[j][v0 + 2];
                if (USE_C) {
                    o0 = fma(P.beta, cin[j][v0][0], o0);
                    o1 = fma(P.beta, cin[j][v0][1], o1);
                }
                double* p = P.C + row + (long)col * P.ldc;
                if (P.vec_c && row + 1 < P.M) {
                    __stcs(reinterpret_cast<double2*>(p), make_double2(o0, o1));
                } else {
                    if (row < P.M) __stcs(p, o0);
                    if (row + 1 < P.M) __stcs(p + 1, o1);
                }
            }
    }
    // abort: the loads this group issued and has not consumed land before exit
    if (!ok && wq == 0 && lane == 0) {
        for (int q = 0; q < kGroupStages; ++q) {
            const int nn = n + q;  // block n (waited for) and n + 1 (loaded ahead)
            if (blk0 + nn * step < P.nblk)
                drain_phase(&full[grp * kGroupStages + (nn & (kGroupStages - 1))], (uint32_t)(nn / kGroupStages) & 1u,
                            P.wait_ns);
        }
    }
}

// ---------------------------------------------------------------- FP32
// 128-row blocks of op(A) (32 KB per stage), op(B) resident as [k][64 n]
// floats.  Thread u of a group (tm = u mod 16, tn = u / 16) owns 8 rows x
// columns 8 tn .. 8 tn + 7 of the 128 x 64 block of C:
//   op(A) m-contiguous (boxes of 32 m x 64 k): rows 4 tm + {0..3} and
//     64 + 4 tm + {0..3}, two 16-byte loads per k;
//   op(A) k-contiguous (boxes of 128 m x 32 k): rows tm + 16 i, i < 8, one
//     16-byte load of 4 k per row.
// Either way a quarter-warp reads 8 distinct 16-byte chunks of the swizzle.
constexpr int kFBM = 128;
constexpr int kFABytes = kFBM * kKK * 4;  // 32 KB per stage
constexpr int kFBBytes = kKK * kKN * 4;   // 16 KB, resident
constexpr size_t kFSmem = 1024 + (size_t)kGroups * kFABytes + kFBBytes + 256;

struct SkinnyParamsF {
    int M, N, K, nblk;
    float alpha, beta;
    const float* B;
    long ldb;
    int b_kfast;
    int vec_c;  // C 16-byte aligned with ldc a multiple of 4 (m-contiguous op(A) only)
    float* C;
    long ldc;
    int* report;
    unsigned long long wait_ns;
};

template <bool A_MN, bool USE_C>
__global__ void __launch_bounds__(kKThreads, 1)
sgemm_skinny_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ SkinnyParamsF P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float* sB = reinterpret_cast<float*>(smem + kGroups * kFABytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kGroups * kFABytes + kFBBytes);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(full + kGroups);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / kGroupWarps, wq = warp % kGroupWarps;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGroups; ++s) mbar_init(&full[s], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const WaitCtl W{abort_flag, nullptr, P.report, P.wait_ns};
    const uint8_t* sa = smem + grp * kFABytes;
    auto boxes = [&](uint32_t st, uint64_t* bar, int i0) {
        if (A_MN) {  // 4 boxes of 64 k-rows x 32 m
#pragma unroll
            for (int b = 0; b < 4; ++b) tma_load_2d(st + b * 8192, &tmA, bar, i0 + 32 * b, 0);
        } else {  // 2 boxes of 128 m-rows x 32 k
#pragma unroll
            for (int b = 0; b < 2; ++b) tma_load_2d(st + b * 16384, &tmA, bar, 32 * b, i0);
        }
    };
    const int step = kGroups * gridDim.x;
    int blk = blockIdx.x + grp * gridDim.x;
    if (wq == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        feed_stage(&full[grp], smem_u32(sa), kFABytes, blk, kFBM, P.nblk, boxes);
    }

    {
        float v[kKK * kKN / kKThreads];
#pragma unroll
        for (int r = 0; r < kKK * kKN / kKThreads; ++r) {
            const int e = threadIdx.x + r * kKThreads;
            const int j = P.b_kfast ? e / kKK : e % kKN, kk = P.b_kfast ? e % kKK : e / kKN;
            v[r] = (kk < P.K && j < P.N) ? (P.b_kfast ? P.B[kk + (long)j * P.ldb] : P.B[j + (long)kk * P.ldb]) : 0.f;
        }
#pragma unroll
        for (int r = 0; r < kKK * kKN / kKThreads; ++r) {
            const int e = threadIdx.x + r * kKThreads;
            const int j = P.b_kfast ? e / kKK : e % kKN, kk = P.b_kfast ? e % kKK : e / kKN;
            sB[kk * kKN + j] = v[r];
        }
    }
    __syncthreads();

    const int u = threadIdx.x % (kGroupWarps * 32);
    const int tm = u & 15, tn = u >> 4;
    const bool busy = 8 * tn < P.N;
    uint32_t ph = 0;
    bool ok = true;
    for (; blk < P.nblk; blk += step) {
        float acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
        ok = wait_phase(&full[grp], ph, W, WAIT_MMA_FULL_A);
        if (ok && busy) {
            if (A_MN) {
                // element (m, k) at (m / 32) * 8192 + k * 128 + (((m mod 32) / 4 ^ k mod 8) * 16) + (m mod 4) * 4
                const uint32_t lo = (uint32_t)((tm >> 3) * 8192), hi = lo + 2 * 8192;
#pragma unroll 4
                for (int k = 0; k < P.K; ++k) {
                    const uint32_t chunk = (uint32_t)(((tm & 7) ^ (k & 7)) << 4) + k * 128;
                    const float4 a0 = *reinterpret_cast<const float4*>(sa + lo + chunk);
                    const float4 a1 = *reinterpret_cast<const float4*>(sa + hi + chunk);
                    const float4 b0 = *reinterpret_cast<const float4*>(sB + k * kKN + 8 * tn);
                    const float4 b1 = *reinterpret_cast<const float4*>(sB + k * kKN + 8 * tn + 4);
                    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                    const float bw[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int i = 0; i < 8; ++i)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bw[j], acc[i][j]);
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
#pragma unroll
                    for (int uu = 0; uu < 4; ++uu) {
                        const float4 b0 = *reinterpret_cast<const float4*>(sB + (4 * kq + uu) * kKN + 8 * tn);
                        const float4 b1 = *reinterpret_cast<const float4*>(sB + (4 * kq + uu) * kKN + 8 * tn + 4);
                        const float bw[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const float ak = uu == 0 ? a[i].x : uu == 1 ? a[i].y : uu == 2 ? a[i].z : a[i].w;
#pragma unroll
                            for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(ak, bw[j], acc[i][j]);
                        }
                    }
                }
            }
        }
        if (!(ok = group_bar_and(grp, ok))) break;
        ph ^= 1u;
        const int i0 = blk * kFBM;
        if (wq == 0 && lane == 0) feed_stage(&full[grp], smem_u32(sa), kFABytes, blk + step, kFBM, P.nblk, boxes);
        // epilogue in two halves of four rows per thread: every beta * C load of a
        // half is issued before its stores (L2 hits after the prefetch)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float cin[4][8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = 8 * tn + j;
                if (A_MN) {
                    const int row = i0 + 64 * h + 4 * tm;
                    const float* p = P.C + row + (long)col * P.ldc;
                    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (USE_C && col < P.N) {
                        if (P.vec_c && row + 3 < P.M) {
                            x = __ldcs(reinterpret_cast<const float4*>(p));
                        } else {
                            if (row < P.M) x.x = __ldcs(p);
                            if (row + 1 < P.M) x.y = __ldcs(p + 1);
                            if (row + 2 < P.M) x.z = __ldcs(p + 2);
                            if (row + 3 < P.M) x.w = __ldcs(p + 3);
                        }
                    }
                    cin[0][j] = x.x, cin[1][j] = x.y, cin[2][j] = x.z, cin[3][j] = x.w;
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int row = i0 + tm + 16 * (4 * h + v);
                        cin[v][j] = (USE_C && row < P.M && col < P.N) ? __ldcs(P.C + row + (long)col * P.ldc) : 0.f;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = 8 * tn + j;
                if (col >= P.N) break;
                float o[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    o[v] = P.alpha * acc[4 * h + v][j];
                    if (USE_C) o[v] = fmaf(P.beta, cin[v][j], o[v]);
                }
                if (A_MN) {
                    const int row = i0 + 64 * h + 4 * tm;
                    float* p = P.C + row + (long)col * P.ldc;
                    if (P.vec_c && row + 3 < P.M) {
                        __stcs(reinterpret_cast<float4*>(p), make_float4(o[0], o[1], o[2], o[3]));
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            if (row + v < P.M) __stcs(p + v, o[v]);
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int row = i0 + tm + 16 * (4 * h + v);
                        if (row < P.M) __stcs(P.C + row + (long)col * P.ldc, o[v]);
                    }
                }
            }
        }
    }
    if (!ok && wq == 0 && lane == 0) drain_phase(&full[grp], ph, P.wait_ns);
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
    const bool c_al = reinterpret_cast<uintptr_t>(g.c) % 16 == 0 && g.ldc % 4 == 0;
    const bool use_c = g.beta != 0.0f;
    P.vec_c = a_mn && c_al;
    auto kern = a_mn ? (use_c ? sgemm_skinny_tma_kernel<true, true> : sgemm_skinny_tma_kernel<true, false>)
                     : (use_c ? sgemm_skinny_tma_kernel<false, true> : sgemm_skinny_tma_kernel<false, false>);
    if ((e = ensure_dynamic_smem(kern, (int)kFSmem)) != cudaSuccess) return e;
    prof_begin(st);
    kern<<<grid, kKThreads, kFSmem, st>>>(ma, P);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

cudaError_t dgemm_skinny_tma(const GemmArgsF64& g, cudaStream_t st) {
    CUtensorMap ma;
    cudaError_t e = make_a_map(&ma, g, g.transa == 'N' ? kKK : kKBM);
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
    P.vec_c = reinterpret_cast<uintptr_t>(g.c) % 16 == 0 && g.ldc % 2 == 0;
    const bool use_c = g.beta != 0.0;
    auto kern = g.transa == 'N'
                    ? (use_c ? dgemm_skinny_tma_kernel<true, true> : dgemm_skinny_tma_kernel<true, false>)
                    : (use_c ? dgemm_skinny_tma_kernel<false, true> : dgemm_skinny_tma_kernel<false, false>);
    if ((e = ensure_dynamic_smem(kern, (int)kKSmem)) != cudaSuccess) return e;
    prof_begin(st);
    kern<<<grid, kKThreads, kKSmem, st>>>(ma, P);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

}  // namespace zb
