// Native FP64 GEMM on 128 x 128 tiles, TMA-fed and warp-specialised (sm_100a).
//
//   C = alpha * op(A) * op(B) + beta * C     (column-major)
//
// The same contraction as dgemm_dmma_kernel (the reference's packed-SIMD
// body, kernels/shared/matrix_matrix/packed_simd.zig:306 noTransReal and
// planner.zig:327 noTransRealWithBLayout) for operands that TMA can describe:
// 16-byte aligned base addresses and even leading dimensions.  One producer
// warp issues cp.async.bulk.tensor loads of 32-deep K slices of op(A) and
// op(B) into a three-stage ring (64 KB per stage, 128-byte swizzle); eight
// math warps wait on the stage's "full" mbarrier, run warp-level DMMA
// (mma.sync m16n8k8 .f64; tcgen05 has no FP64 kind) and release the stage on
// its "empty" mbarrier.  No block-wide barrier sits in the main loop.
//
// Shared tiles keep the orientation of global memory:
//   MN-major (A 'N', B 'T'): 8 boxes of 32 k-rows x 16 elements (128 B);
//   K-major  (A 'T', B 'N'): 2 boxes of 128 rows x 16 k (128 B).
// Within a k8 step the MMA's k index kappa reads physical k = 2 (kappa mod 4)
// + kappa / 4, and within a 16-row fragment MMA row r = g + 8 v reads
// physical row 2 g + v (g = lane / 4); for a K-major op(B) the MMA's column n
// reads physical column (n >> 1) | ((n & 1) << 2) of its 8-column block.  All
// are bijections, applied to A, B and C alike, so the product is unchanged;
// they make every A fragment pair and every K-major B fragment pair one
// 16-byte shared load, and with the 128-byte swizzle every fragment load runs
// at the minimum number of shared-memory wavefronts (the two rows of a K-major
// quarter-warp fall in opposite halves of the swizzle).
//
// Every mbarrier wait is bounded in time; a wait that runs out records its
// site in the device's report word and the warp leaves its part of C alone.
#include <cudaTypedefs.h>

#include "bounded_wait.cuh"
#include "common.cuh"
#include "kernels.h"
#include "ozaki.h"

namespace zb {
namespace {

constexpr int kTBM = 128, kTBN = 128, kTBK = 32, kTStages = 3;
constexpr int kTMathWarps = 8;                     // 2 (M) x 4 (N) warps of 64 x 32
constexpr int kTThreads = (kTMathWarps + 4) * 32;  // + a producer warpgroup (one TMA thread)
// Register split: 384 threads launch with 168 registers each (64512); the
// producer warpgroup drops to 40 and the two math warpgroups rise to 232:
// 128 x 40 + 256 x 232 = 64512.  Per SM sub-partition: 2 x 32 x 232 + 32 x 40
// = 16128 of its 16384 registers.
constexpr int kTProducerRegs = 40, kTMathRegs = 232;
static_assert(128 * kTProducerRegs + 256 * kTMathRegs <= kTThreads * 168, "register split exceeds the launch");
constexpr int kTWM = 64, kTWN = 32;
constexpr int kTOpBytes = kTBM * kTBK * 8;  // 32 KB per operand and stage
constexpr int kTStageBytes = 2 * kTOpBytes;
constexpr size_t kTSmem = 1024 + (size_t)kTStages * kTStageBytes + 256;
constexpr unsigned long long kTWaitNs = 4000000000ull;

struct TmaGemmParams {
    int M, N, K, k_chunk, tri;
    double alpha, beta;
    double* C;
    long ldc;
    double* W;  // split-K partials, slice blockIdx.z (ld = M)
    int* report;
    unsigned long long wait_ns;
};

// Byte offsets of an element in the two tile orientations (128-byte swizzle:
// the 16-byte chunk index is XORed with the row index mod 8).
ZB_DEVICE uint32_t mn_major_off(int mn, int k) {
    return (uint32_t)((mn >> 4) * 4096 + k * 128 + ((((mn & 15) >> 1) ^ (k & 7)) << 4) + ((mn & 1) << 3));
}
ZB_DEVICE uint32_t k_major_off(int mn, int k) {
    return (uint32_t)((k >> 4) * 16384 + mn * 128 + ((((k & 15) >> 1) ^ (mn & 7)) << 4) + ((k & 1) << 3));
}

// A_MN: op(A) is stored m-contiguous (transa 'N'); B_K: op(B) is stored
// k-contiguous (transb 'N').  PARTIAL: raw sums to the split-K workspace.
template <bool A_MN, bool B_K, bool PARTIAL>
__global__ void __launch_bounds__(kTThreads, 1)
dgemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ TmaGemmParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kTStages * kTStageBytes);
    uint64_t* empty = full + kTStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kTStages);

    const int m0 = blockIdx.x * kTBM, n0 = blockIdx.y * kTBN;
    // triangle mode (SYRK): tiles holding no element of the stored triangle
    if ((P.tri == 1 && m0 > n0 + kTBN - 1) || (P.tri == 2 && m0 + kTBM - 1 < n0)) return;
    const int kb = blockIdx.z * P.k_chunk;
    const int ke = min(P.K, kb + P.k_chunk);
    const int KT = (ke - kb + kTBK - 1) / kTBK;  // k_chunk is a multiple of kTBK

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTMathWarps);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == kTMathWarps && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    __syncthreads();
    // launched during the tail of the kernel before it (which may write A, B or C)
    grid_dependency_wait();
    const WaitCtl W{abort_flag, nullptr, P.report, P.wait_ns};

    if (warp >= kTMathWarps) {
        // ------------------------------------------------------ TMA producer
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kTProducerRegs));
        if (warp == kTMathWarps && lane == 0) {
            Issued issued;
            bool ok = true;
            int s = 0;
            uint32_t ph = 0;
            for (int kt = 0; kt < KT; ++kt) {
                if (!(ok = wait_phase(&empty[s], ph ^ 1u, W, WAIT_PRODUCER_EMPTY_A))) break;
                const uint32_t sa = smem_u32(smem + s * kTStageBytes), sb = sa + kTOpBytes;
                const int k0 = kb + kt * kTBK;
                mbar_arrive_expect_tx(&full[s], kTStageBytes);
                if (A_MN) {
#pragma unroll
                    for (int b = 0; b < kTBM / 16; ++b) tma_load_2d(sa + b * 4096, &tmA, &full[s], m0 + 16 * b, k0);
                } else {
#pragma unroll
                    for (int b = 0; b < kTBK / 16; ++b) tma_load_2d(sa + b * 16384, &tmA, &full[s], k0 + 16 * b, m0);
                }
                if (B_K) {
#pragma unroll
                    for (int b = 0; b < kTBK / 16; ++b) tma_load_2d(sb + b * 16384, &tmB, &full[s], k0 + 16 * b, n0);
                } else {
#pragma unroll
                    for (int b = 0; b < kTBN / 16; ++b) tma_load_2d(sb + b * 4096, &tmB, &full[s], n0 + 16 * b, k0);
                }
                issued.note(s, ph);
                if (++s == kTStages) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            // aborted: the bytes of every issued copy land before the CTA can retire
            if (!ok) issued.drain(full, kTStages, P.wait_ns);
        }
        return;
    }

    // ---------------------------------------------------------- math warps
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kTMathRegs));
    const int wm = (warp >> 2) * kTWM, wn = (warp & 3) * kTWN;
    const int g = lane >> 2, t = lane & 3;
    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    // per-thread fragment offsets within a stage (k8 step 0; step ks adds a
    // multiple of 8 to k, which leaves k mod 8 and the swizzle unchanged)
    uint32_t a_off[4][2], b_off[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int v = 0; v < 2; ++v)
            a_off[i][v] = A_MN ? mn_major_off(wm + 16 * i + 2 * g, 2 * t + v)       // v = v1: rows 2g, 2g+1
                               : k_major_off(wm + 16 * i + 2 * g + v, 2 * t);       // v = v0: k 2t, 2t+1
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int v = 0; v < 2; ++v)
            b_off[j][v] = B_K ? k_major_off(wn + 8 * j + ((g >> 1) | ((g & 1) << 2)), 2 * t)
                              : mn_major_off(wn + 8 * j + g, 2 * t + v);

    bool ok = true;
    int s = 0;
    uint32_t ph = 0;
    for (int kt = 0; kt < KT; ++kt) {
        if (!(ok = wait_phase(&full[s], ph, W, WAIT_MMA_FULL_A))) break;
        const uint8_t* sa = smem + s * kTStageBytes;
        const uint8_t* sb = sa + kTOpBytes;
        // one k8 step per iteration (deeper unrolling spilled and measured up to 0.7 % slower)
#pragma unroll 1
        for (int ks = 0; ks < kTBK; ks += 8) {
            // k8 step ks: MN-major tiles advance 8 rows of 128 B; K-major tiles
            // move 4 chunks within a 16-k box (an XOR on the chunk index, as
            // t < 4) and to the second box from ks = 16
            const uint32_t mn_step = ks * 128;
            const uint32_t k_xor = ((ks & 15) >> 1) << 4, k_box = (ks >> 4) * 16384;
            double af[4][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (A_MN) {
                    // a[0], a[1]: rows 2g, 2g+1 at k 2t; a[2], a[3]: at k 2t+1
                    const double2 p0 = *reinterpret_cast<const double2*>(sa + a_off[i][0] + mn_step);
                    const double2 p1 = *reinterpret_cast<const double2*>(sa + a_off[i][1] + mn_step);
                    af[i][0] = p0.x, af[i][1] = p0.y, af[i][2] = p1.x, af[i][3] = p1.y;
                } else {
                    // a[0], a[2]: row 2g at k 2t, 2t+1; a[1], a[3]: row 2g+1
                    const double2 p0 = *reinterpret_cast<const double2*>(sa + ((a_off[i][0] ^ k_xor) + k_box));
                    const double2 p1 = *reinterpret_cast<const double2*>(sa + ((a_off[i][1] ^ k_xor) + k_box));
                    af[i][0] = p0.x, af[i][2] = p0.y, af[i][1] = p1.x, af[i][3] = p1.y;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (B_K) {
                    const double2 q = *reinterpret_cast<const double2*>(sb + ((b_off[j][0] ^ k_xor) + k_box));
                    bf[j][0] = q.x, bf[j][1] = q.y;
                } else {
                    bf[j][0] = *reinterpret_cast<const double*>(sb + b_off[j][0] + mn_step);
                    bf[j][1] = *reinterpret_cast<const double*>(sb + b_off[j][1] + mn_step);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (++s == kTStages) {
            s = 0;
            ph ^= 1u;
        }
    }
    if (!ok || *abort_flag) return;  // an incomplete sum is never written

    // Epilogue: c[v0 + 2 v1] holds physical row 2 g + v1 and column 2 t + v0 of
    // the fragment (K-major op(B): column t + 4 v0).  The beta * C reads of a
    // fragment row are issued before its stores.
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double cin[4][4];
        if (!PARTIAL && P.beta != 0.0) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = m0 + wm + 16 * i + 2 * g + (v >> 1);
                    const int col = n0 + wn + 8 * j + (B_K ? t + 4 * (v & 1) : 2 * t + (v & 1));
                    const bool in_tri = P.tri == 0 || (P.tri == 1 ? row <= col : row >= col);
                    cin[j][v] = (row < P.M && col < P.N && in_tri) ? P.C[(long)col * P.ldc + row] : 0.0;
                }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int row = m0 + wm + 16 * i + 2 * g + (v >> 1);
                const int col = n0 + wn + 8 * j + (B_K ? t + 4 * (v & 1) : 2 * t + (v & 1));
                const bool in_tri = P.tri == 0 || (P.tri == 1 ? row <= col : row >= col);
                if (row < P.M && col < P.N && in_tri) {
                    if (PARTIAL) {
                        P.W[(long)blockIdx.z * P.M * P.N + (long)col * P.M + row] = acc[i][j][v];
                    } else {
                        double out = P.alpha * acc[i][j][v];
                        if (P.beta != 0.0) out = fma(P.beta, cin[j][v], out);
                        P.C[(long)col * P.ldc + row] = out;
                    }
                }
            }
    }
}

// 2-D FP64 tensor map over a column-major matrix with `inner` contiguous
// elements per column (leading dimension ld) and `outer` columns; box
// 16 x box_outer elements with 128-byte swizzle; out-of-range elements read 0.
cudaError_t make_f64_map(CUtensorMap* map, const double* base, long inner, long outer, long ld, int box_outer) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return cudaErrorNotSupported;
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 8)};
    cuuint32_t box[2] = {16, (cuuint32_t)box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <bool A_MN, bool B_K, bool PARTIAL>
cudaError_t launch_tma(const CUtensorMap& ma, const CUtensorMap& mb, const TmaGemmParams& P, int splits,
                       cudaStream_t st) {
    auto kern = dgemm_tma_kernel<A_MN, B_K, PARTIAL>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)kTSmem);
    if (e != cudaSuccess) return e;
    dim3 grid((P.M + kTBM - 1) / kTBM, (P.N + kTBN - 1) / kTBN, splits);
    prof_begin(st);
    e = launch_dependent(kern, grid, dim3(kTThreads), kTSmem, st, ma, mb, P);
    count_launch();
    prof_end(st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <bool PARTIAL>
cudaError_t dispatch_tma(bool a_mn, bool b_k, const CUtensorMap& ma, const CUtensorMap& mb, const TmaGemmParams& P,
                         int splits, cudaStream_t st) {
    if (a_mn && b_k) return launch_tma<true, true, PARTIAL>(ma, mb, P, splits, st);
    if (a_mn) return launch_tma<true, false, PARTIAL>(ma, mb, P, splits, st);
    if (b_k) return launch_tma<false, true, PARTIAL>(ma, mb, P, splits, st);
    return launch_tma<false, false, PARTIAL>(ma, mb, P, splits, st);
}

}  // namespace

bool dgemm_tma_applies(const GemmArgsF64& g) {
    const uintptr_t bits = reinterpret_cast<uintptr_t>(g.a) | reinterpret_cast<uintptr_t>(g.b);
    return bits % 16 == 0 && g.lda % 2 == 0 && g.ldb % 2 == 0 && tensor_map_encoder() != nullptr;
}

int dgemm_tma_k_chunk(int k, int splits) {
    splits = splits < 1 ? 1 : splits;
    const int c = (k + splits - 1) / splits;
    return (c + kTBK - 1) / kTBK * kTBK;
}

cudaError_t dgemm_tma(const GemmArgsF64& g, int splits, double* workspace, cudaStream_t st) {
    const bool a_mn = g.transa == 'N', b_k = g.transb == 'N';
    CUtensorMap ma, mb;
    cudaError_t e = a_mn ? make_f64_map(&ma, g.a, g.m, g.k, g.lda, kTBK) : make_f64_map(&ma, g.a, g.k, g.m, g.lda, kTBM);
    if (e != cudaSuccess) return e;
    e = b_k ? make_f64_map(&mb, g.b, g.k, g.n, g.ldb, kTBN) : make_f64_map(&mb, g.b, g.n, g.k, g.ldb, kTBK);
    if (e != cudaSuccess) return e;
    TmaGemmParams P{};
    P.M = g.m;
    P.N = g.n;
    P.K = g.k;
    P.k_chunk = dgemm_tma_k_chunk(g.k, splits);
    P.tri = g.tri;
    P.alpha = g.alpha;
    P.beta = g.beta;
    P.C = g.c;
    P.ldc = g.ldc;
    P.W = workspace;
    P.wait_ns = kTWaitNs;
    if ((e = wait_report_word(&P.report)) != cudaSuccess) return e;
    const int used = (g.k + P.k_chunk - 1) / P.k_chunk;
    if (used == 1) return dispatch_tma<false>(a_mn, b_k, ma, mb, P, 1, st);
    if (!workspace) return cudaErrorInvalidValue;
    return dispatch_tma<true>(a_mn, b_k, ma, mb, P, used, st);
}

}  // namespace zb
