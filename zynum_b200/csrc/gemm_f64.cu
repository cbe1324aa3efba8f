// Native FP64 GEMM (DGEMM) for sm_100a.
//
//   C = alpha * op(A) * op(B) + beta * C     (column-major, any lda/ldb/ldc)
//
// Replaces the reference's packed-SIMD real GEMM body
// (kernels/shared/matrix_matrix/packed_simd.zig:306 noTransReal, its
// accumulatePackedP :140 FMA loop and epilogue.applyVector epilogue.zig:35)
// and the A^T pack of planner.transposedAReal (planner.zig:360).
//
// Blackwell has no FP64 kind for tcgen05.mma, so the contraction runs on the
// FP64 tensor pipe through warp-level DMMA (mma.sync m16n8k8 .f64).  Operands
// are staged global -> shared memory with cp.async in a multi-stage ring.
// cp.async is used instead of TMA because the BLAS leading dimensions are
// arbitrary: TMA needs 16-byte aligned strides, and lda = 1031 (8248 B) is not.
//
// Transposes cost nothing: every operand tile is copied in the orientation it
// has in global memory (so global reads stay contiguous) and the fragment
// loader reads either "K-fast" or "MN-fast" shared tiles; both orientations
// use a row pitch of 4 (mod 16) doubles, which keeps all fragment loads free of
// bank conflicts.
//
// Split-K (for K-dominant shapes, e.g. 256 x 256 x 262144) writes per-split
// partial tiles to a workspace; dgemm_splitk_reduce sums them in split order
// (deterministic) and applies alpha/beta.
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kBK = 16;

template <int ROWS, int COLS, int PITCH, int VEC, int NTHREADS>
ZB_DEVICE void load_tile(double* smem, const double* __restrict__ base, long ld, int r0, int c0, int r_lim,
                         int c_lim) {
    constexpr int CHUNKS_PER_ROW = COLS / VEC;
    constexpr int CHUNKS = ROWS * CHUNKS_PER_ROW;
    static_assert(CHUNKS % NTHREADS == 0 || CHUNKS < NTHREADS, "tile copy must divide evenly over the block");
#pragma unroll
    for (int it = 0; it < (CHUNKS + NTHREADS - 1) / NTHREADS; ++it) {
        int q = it * NTHREADS + threadIdx.x;
        if (CHUNKS < NTHREADS && q >= CHUNKS) break;  // narrow tiles: fewer chunks than threads
        int r = q / CHUNKS_PER_ROW;
        int c = (q % CHUNKS_PER_ROW) * VEC;
        int gr = r0 + r, gc = c0 + c;
        uint32_t dst = smem_u32(smem + r * PITCH + c);
        int valid = 0;
        if (gr < r_lim) {
            valid = c_lim - gc;
            valid = valid < 0 ? 0 : (valid > VEC ? VEC : valid);
        }
        const double* src = valid ? base + (long)gr * ld + gc : base;
        if (VEC == 2)
            cp_async_16(dst, src, valid * 8);
        else
            cp_async_8(dst, src, valid * 8);
    }
}

// BM x BN block tile, WM x WN warp tile, STAGES-deep cp.async ring of BK-deep slices.
// A_KFAST: A's shared tile is [m][k] (A stored transposed in global memory).
// B_KFAST: B's shared tile is [n][k] (B stored untransposed in global memory).
// PARTIAL: write raw accumulators to workspace slice blockIdx.z (ld = M).
template <int BM, int BN, int WM, int WN, int STAGES, bool A_KFAST, bool B_KFAST, int VEC, bool PARTIAL, int BK>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32, 1)
dgemm_dmma_kernel(int M, int N, int K, int k_chunk, double alpha, const double* __restrict__ A, long lda,
                  const double* __restrict__ B, long ldb, double beta, double* __restrict__ C, long ldc,
                  double* __restrict__ W, int tri) {
    constexpr int NTHREADS = (BM / WM) * (BN / WN) * 32;
    constexpr int WARPS_N = BN / WN;
    constexpr int MI = WM / 16;
    constexpr int NI = WN / 8;
    // Shared tile geometry (pitch = 4 mod 16 doubles).
    constexpr int A_ROWS = A_KFAST ? BM : BK, A_COLS = A_KFAST ? BK : BM, A_PITCH = A_COLS + 4;
    constexpr int B_ROWS = B_KFAST ? BN : BK, B_COLS = B_KFAST ? BK : BN, B_PITCH = B_COLS + 4;
    constexpr int A_STAGE = A_ROWS * A_PITCH, B_STAGE = B_ROWS * B_PITCH;

    extern __shared__ __align__(128) double smem[];
    double* As = smem;
    double* Bs = smem + STAGES * A_STAGE;

    const int m0 = blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    // triangle mode: skip tiles that hold no element of the stored triangle
    if ((tri == 1 && m0 > n0 + BN - 1) || (tri == 2 && m0 + BM - 1 < n0)) return;
    const int kb = blockIdx.z * k_chunk;
    const int ke = min(K, kb + k_chunk);
    const int KT = (ke - kb + BK - 1) / BK;
    // launched during the tail of the kernel before it (which may write A, B or C)
    grid_dependency_wait();

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wm = (warp / WARPS_N) * WM;
    const int wn = (warp % WARPS_N) * WN;
    const int g = lane >> 2, t = lane & 3;

    double acc[MI][NI][4];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kb + kt * BK;
        if (A_KFAST)  // A stored k x m (op = T): rows m, contiguous k
            load_tile<A_ROWS, A_COLS, A_PITCH, VEC, NTHREADS>(As + stage * A_STAGE, A, lda, m0, k0, M, ke);
        else  // A stored m x k: rows k, contiguous m
            load_tile<A_ROWS, A_COLS, A_PITCH, VEC, NTHREADS>(As + stage * A_STAGE, A, lda, k0, m0, ke, M);
        if (B_KFAST)  // B stored k x n: rows n, contiguous k
            load_tile<B_ROWS, B_COLS, B_PITCH, VEC, NTHREADS>(Bs + stage * B_STAGE, B, ldb, n0, k0, N, ke);
        else  // B stored n x k (op = T): rows k, contiguous n
            load_tile<B_ROWS, B_COLS, B_PITCH, VEC, NTHREADS>(Bs + stage * B_STAGE, B, ldb, k0, n0, ke, N);
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }

    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            int nk = kt + STAGES - 1;
            if (nk < KT) load_stage(nk % STAGES, nk);
            cp_async_commit();
        }
        const double* as = As + (kt % STAGES) * A_STAGE;
        const double* bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            double af[MI][4], bf[NI][2];
#pragma unroll
            for (int i = 0; i < MI; ++i) {
                const int r = wm + i * 16 + g;
#pragma unroll
                for (int v1 = 0; v1 < 2; ++v1) {
                    const int kk = ks + t + 4 * v1;
#pragma unroll
                    for (int v0 = 0; v0 < 2; ++v0) {
                        const int rr = r + 8 * v0;
                        af[i][v0 + 2 * v1] = A_KFAST ? as[rr * A_PITCH + kk] : as[kk * A_PITCH + rr];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NI; ++j) {
                const int c = wn + j * 8 + g;
#pragma unroll
                for (int v = 0; v < 2; ++v) {
                    const int kk = ks + t + 4 * v;
                    bf[j][v] = B_KFAST ? bs[c * B_PITCH + kk] : bs[kk * B_PITCH + c];
                }
            }
#pragma unroll
            for (int i = 0; i < MI; ++i)
#pragma unroll
                for (int j = 0; j < NI; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();

    // Epilogue: c[v0 + 2 v1] sits at (row g + 8 v1, col 2 t + v0) of each 16x8 fragment.
    // The beta * C reads of one fragment row are all issued before its stores
    // (a store to C would otherwise order every later C load behind it).
#pragma unroll
    for (int i = 0; i < MI; ++i) {
        double cin[NI][4];
        if (!PARTIAL && beta != 0.0) {
#pragma unroll
            for (int j = 0; j < NI; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = m0 + wm + i * 16 + g + 8 * (v >> 1);
                    const int col = n0 + wn + j * 8 + 2 * t + (v & 1);
                    const bool in_tri = tri == 0 || (tri == 1 ? row <= col : row >= col);
                    cin[j][v] = (row < M && col < N && in_tri) ? C[(long)col * ldc + row] : 0.0;
                }
        }
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int row = m0 + wm + i * 16 + g + 8 * (v >> 1);
                const int col = n0 + wn + j * 8 + 2 * t + (v & 1);
                const bool in_tri = tri == 0 || (tri == 1 ? row <= col : row >= col);
                if (row < M && col < N && in_tri) {
                    if (PARTIAL) {
                        W[(long)blockIdx.z * M * N + (long)col * M + row] = acc[i][j][v];
                    } else {
                        double out = alpha * acc[i][j][v];
                        if (beta != 0.0) out = fma(beta, cin[j][v], out);
                        C[(long)col * ldc + row] = out;
                    }
                }
            }
    }
}

__global__ void dgemm_splitk_reduce(int M, int N, int splits, const double* __restrict__ W, double alpha, double beta,
                                    double* __restrict__ C, long ldc, int tri) {
    grid_dependency_wait();  // launched during the tail of the product that writes W
    long total = (long)M * N;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        int row = (int)(q % M), col = (int)(q / M);
        if (tri == 1 ? row > col : (tri == 2 && row < col)) continue;
        double s = 0.0;
        for (int z = 0; z < splits; ++z) s += W[(long)z * total + q];
        double* cp = C + (long)col * ldc + row;
        double out = alpha * s;
        if (beta != 0.0) out = fma(beta, *cp, out);
        *cp = out;
    }
}

template <int BM, int BN, int WM, int WN, int STAGES, bool AK, bool BK_, int VEC, bool PARTIAL, int BK>
cudaError_t launch_one(const GemmArgsF64& g, int splits, int k_chunk, double* W, cudaStream_t st) {
    constexpr int NTHREADS = (BM / WM) * (BN / WN) * 32;
    constexpr int A_ROWS = AK ? BM : BK, A_COLS = AK ? BK : BM;
    constexpr int B_ROWS = BK_ ? BN : BK, B_COLS = BK_ ? BK : BN;
    constexpr size_t SMEM = (size_t)STAGES * (A_ROWS * (A_COLS + 4) + B_ROWS * (B_COLS + 4)) * sizeof(double);
    auto kern = dgemm_dmma_kernel<BM, BN, WM, WN, STAGES, AK, BK_, VEC, PARTIAL, BK>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)SMEM);
    if (e != cudaSuccess) return e;
    dim3 grid((g.m + BM - 1) / BM, (g.n + BN - 1) / BN, splits);
    prof_begin(st);
    e = launch_dependent(kern, grid, dim3(NTHREADS), SMEM, st, g.m, g.n, g.k, k_chunk, g.alpha, g.a, g.lda, g.b,
                         g.ldb, g.beta, g.c, g.ldc, W, g.tri);
    count_launch();
    prof_end(st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int STAGES, bool PARTIAL, int BK>
cudaError_t dispatch_layout(const GemmArgsF64& g, int vec, int splits, int k_chunk, double* W, cudaStream_t st) {
    const bool ak = g.transa != 'N', bk = g.transb == 'N';
#define ZB_CASE(AK, BKF, V)                                                                              \
    if (ak == AK && bk == BKF && vec == V)                                                               \
        return launch_one<BM, BN, WM, WN, STAGES, AK, BKF, V, PARTIAL, BK>(g, splits, k_chunk, W, st);
    ZB_CASE(false, false, 1) ZB_CASE(false, true, 1) ZB_CASE(true, false, 1) ZB_CASE(true, true, 1)
    ZB_CASE(false, false, 2) ZB_CASE(false, true, 2) ZB_CASE(true, false, 2) ZB_CASE(true, true, 2)
#undef ZB_CASE
    return cudaErrorInvalidValue;
}

cudaError_t splitk_reduce(const GemmArgsF64& g, int used_splits, double* workspace, cudaStream_t st) {
    long total = (long)g.m * g.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    cudaError_t e = launch_dependent(dgemm_splitk_reduce, dim3(blocks), dim3(256), 0, st, g.m, g.n, used_splits,
                                     (const double*)workspace, g.alpha, g.beta, g.c, g.ldc, g.tri);
    count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int STAGES, int BK = kBK>
cudaError_t run_tiles(const GemmArgsF64& g, int vec, int used_splits, int k_chunk, double* workspace,
                      cudaStream_t st) {
    if (used_splits == 1) return dispatch_layout<BM, BN, WM, WN, STAGES, false, BK>(g, vec, 1, k_chunk, nullptr, st);
    if (!workspace) return cudaErrorInvalidValue;
    cudaError_t e = dispatch_layout<BM, BN, WM, WN, STAGES, true, BK>(g, vec, used_splits, k_chunk, workspace, st);
    if (e != cudaSuccess) return e;
    return splitk_reduce(g, used_splits, workspace, st);
}

}  // namespace

// The 128 x 128 route takes the TMA kernel for operands TMA can describe
// (ZYNUM_GPU_DGEMM_TMA=0 keeps the cp.async kernel, for comparisons).
static bool use_tma_tiles(const GemmArgsF64& g, const GemmPlan& plan) {
    static const bool enabled = [] {
        const char* v = std::getenv("ZYNUM_GPU_DGEMM_TMA");
        return !(v && v[0] == '0');
    }();
    return enabled && plan.tile == TILE_128x128 && dgemm_tma_applies(g);
}

int dgemm_native_used_splits(const GemmArgsF64& g, const GemmPlan& plan) {
    const int splits = plan.splits < 1 ? 1 : plan.splits;
    if (plan.tile == TILE_GEMV && gemv_applies(g.m, g.n, g.k, g.tri)) return gemv_used_splits(g.k, splits);
    if (skinny_gemm_applies(g.m, g.n, g.k, g.tri)) return 1;
    int k_chunk = use_tma_tiles(g, plan) ? dgemm_tma_k_chunk(g.k, splits) : (g.k + splits - 1) / splits;
    k_chunk = (k_chunk + kBK - 1) / kBK * kBK;
    return (g.k + k_chunk - 1) / k_chunk;
}

// Entry used by the planner: `tile` selects the block shape, `splits` > 1
// requires a workspace of splits * m * n doubles.
cudaError_t dgemm_native(const GemmArgsF64& g, const GemmPlan& plan, double* workspace, cudaStream_t st) {
    if (plan.tile == TILE_GEMV && gemv_applies(g.m, g.n, g.k, g.tri)) return dgemv_route(g, plan.splits, workspace, st);
    if (skinny_gemm_applies(g.m, g.n, g.k, g.tri)) {
        static const bool tma = [] {  // TMA-fed kernel unless ZYNUM_GPU_SKINNY_TMA=0
            const char* v = std::getenv("ZYNUM_GPU_SKINNY_TMA");
            return !(v && v[0] == '0');
        }();
        return (tma && dgemm_skinny_tma_applies(g)) ? dgemm_skinny_tma(g, st) : dgemm_skinny(g, st);
    }
    const bool aligned = ((reinterpret_cast<uintptr_t>(g.a) | reinterpret_cast<uintptr_t>(g.b)) % 16 == 0) &&
                         (g.lda % 2 == 0) && (g.ldb % 2 == 0);
    const int vec = aligned ? 2 : 1;
    const int splits = plan.splits < 1 ? 1 : plan.splits;
    int k_chunk = (g.k + splits - 1) / splits;
    k_chunk = (k_chunk + kBK - 1) / kBK * kBK;
    const int used = (g.k + k_chunk - 1) / k_chunk;
    switch (plan.tile) {
        case TILE_128x64:
            return run_tiles<128, 64, 64, 32, 4>(g, vec, used, k_chunk, workspace, st);
        case TILE_NARROW_N:  // n <= 16: 128 x 16 tiles, warps 4 x 2 of 32 x 8
            return run_tiles<128, 16, 32, 8, 4>(g, vec, used, k_chunk, workspace, st);
        case TILE_NARROW_M:  // m <= 16: 16 x 128 tiles, warps 1 x 8 of 16 x 16
            return run_tiles<16, 128, 16, 16, 4>(g, vec, used, k_chunk, workspace, st);
        case TILE_64x64:  // few output tiles: 64 x 64 tiles, warps 2 x 2 of 32 x 32
            return run_tiles<64, 64, 32, 32, 4>(g, vec, used, k_chunk, workspace, st);
        default:
            if (use_tma_tiles(g, plan)) {
                const int kc = dgemm_tma_k_chunk(g.k, splits);
                const int used_t = (g.k + kc - 1) / kc;
                if (used_t > 1 && !workspace) return cudaErrorInvalidValue;
                cudaError_t e = dgemm_tma(g, splits, workspace, st);
                if (e != cudaSuccess || used_t == 1) return e;
                return splitk_reduce(g, used_t, workspace, st);
            }
            // op(B) k-contiguous (transb N): three 32-deep stages (212 KB), half the block
            // barriers of 16-deep slices (+2 % measured at 2048-8192); otherwise four 16-deep
            // stages (32-deep slices measured 1 % slower there)
            if (g.transb == 'N') return run_tiles<128, 128, 64, 32, 3, 32>(g, vec, used, k_chunk, workspace, st);
            return run_tiles<128, 128, 64, 32, 4>(g, vec, used, k_chunk, workspace, st);
    }
}

}  // namespace zb
