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
#include <algorithm>

#include <cstdlib>

#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

constexpr int kBM = 128, kThreads = 256;

// Block tile 128 x BN (BN = 128: two CTAs per SM at 128 registers; a
// 128 x 256 tile with one CTA per SM measured slower at 8192^3).
template <int BN>
struct Cfg;
template <>
struct Cfg<128> {
    static constexpr int BK = 16, STAGES = 5, MINB = 2;
};
__host__ __device__ constexpr int pitch(int width) { return width + 4; }  // floats per shared row ([k][mn], mn fast)

// Copy a BK x WIDTH tile (rows k, columns mn) into shared memory.
// MN_FAST: global element (mn, k) at base[mn + k*ld]; else at base[k + mn*ld].
// `valid` (from init) says which mn indices of this thread lie inside the
// matrix, fixed for the whole K loop; CHECK_K guards the last, partial slab.
template <bool MN_FAST, int VEC, int WIDTH, int BK>
struct TileLoader {
    static constexpr int kCopies = MN_FAST ? (BK * WIDTH / VEC) / kThreads : (BK * WIDTH) / kThreads;
    static constexpr int kKH = BK / 8;  // K-fast: 8 k x 4 mn per warp instruction
    static constexpr int kPitch = pitch(WIDTH);
    static_assert(!MN_FAST || kThreads % (WIDTH / VEC) == 0, "mn index must repeat across copies");

    ZB_DEVICE static void coords(int it, int& kk, int& mm) {
        const int q = it * kThreads + threadIdx.x;
        if (MN_FAST) {
            constexpr int CPR = WIDTH / VEC;
            kk = q / CPR;
            mm = (q % CPR) * VEC;
        } else {
            // lane -> (k = lane % 8, mn = lane / 8): 32-byte global segments and
            // conflict-free shared stores (bank = 4 k + mn mod 32, pitch = 4 mod 32)
            const int lane = threadIdx.x & 31, idx = it * (kThreads / 32) + (threadIdx.x >> 5);
            kk = (idx % kKH) * 8 + (lane & 7);
            mm = (idx / kKH) * 4 + (lane >> 3);
        }
    }
    // MN-fast: bytes to copy (0 outside the matrix), the same in every copy
    // slot; K-fast: one validity bit per slot.
    ZB_DEVICE static uint32_t init(int mn0, int mn_lim) {
        uint32_t r = 0;
        if (MN_FAST) {
            int kk, mm;
            coords(0, kk, mm);
            int valid = mn_lim - (mn0 + mm);
            valid = valid < 0 ? 0 : (valid > VEC ? VEC : valid);
            r = (uint32_t)valid * 4u;
        } else {
#pragma unroll
            for (int it = 0; it < kCopies; ++it) {
                int kk, mm;
                coords(it, kk, mm);
                if (mn0 + mm < mn_lim) r |= 1u << it;
            }
        }
        return r;
    }
    template <bool CHECK_K>
    ZB_DEVICE static void load(float* s, const float* __restrict__ base, long ld, int mn0, int k0, int k_lim,
                               uint32_t valid) {
#pragma unroll
        for (int it = 0; it < kCopies; ++it) {
            int kk, mm;
            coords(it, kk, mm);
            const int gk = k0 + kk, gm = mn0 + mm;
            uint32_t nb = MN_FAST ? valid : ((valid >> it) & 1u) * 4u;
            if (CHECK_K && gk >= k_lim) nb = 0;
            const float* src = nb ? (MN_FAST ? base + (long)gk * ld + gm : base + (long)gm * ld + gk) : base;
            const uint32_t dst = smem_u32(s + kk * kPitch + mm);
            if (MN_FAST && VEC == 4)
                cp_async_16(dst, src, nb);
            else
                cp_async_4(dst, src, nb);
        }
    }
};

// Thread (tx, ty) owns rows {ty*4 + i, 64 + ty*4 + i} and columns
// {64 q + tx*4 + j}, q < BN / 64; a warp covers 4 ty x 8 tx, so each float4
// fragment load touches 4 (A) or 8 (B) distinct 16-byte words: one
// shared-memory wavefront.
template <bool A_MNFAST, bool B_MNFAST, int VEC, bool PARTIAL, int BN>
__global__ void __launch_bounds__(kThreads, Cfg<BN>::MINB)
sgemm_ffma_kernel(int M, int N, int K, int k_chunk, float alpha, const float* __restrict__ A, long lda,
                  const float* __restrict__ B, long ldb, float beta, float* __restrict__ C, long ldc,
                  float* __restrict__ W, int tri) {
    constexpr int BK = Cfg<BN>::BK, STAGES = Cfg<BN>::STAGES, JN = BN / 16, PA = pitch(kBM), PB = pitch(BN);
    extern __shared__ __align__(128) float smf[];
    float* As = smf;
    float* Bs = smf + STAGES * BK * PA;
    using LA = TileLoader<A_MNFAST, (A_MNFAST ? VEC : 1), kBM, BK>;
    using LB = TileLoader<B_MNFAST, (B_MNFAST ? VEC : 1), BN, BK>;

    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    // triangle mode: skip tiles that hold no element of the stored triangle
    if ((tri == 1 && m0 > n0 + BN - 1) || (tri == 2 && m0 + kBM - 1 < n0)) return;
    const int kb = blockIdx.z * k_chunk;
    const int ke = min(K, kb + k_chunk);
    const int KT = (ke - kb + BK - 1) / BK;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tx = (warp & 1) * 8 + (lane & 7), ty = (warp >> 1) * 4 + (lane >> 3);

    const uint32_t a_valid = LA::init(m0, M), b_valid = LB::init(n0, N);

    float acc[8][JN];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < JN; ++j) acc[i][j] = 0.f;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kb + kt * BK;
        float* as = As + stage * BK * PA;
        float* bs = Bs + stage * BK * PB;
        if (k0 + BK <= ke) {
            LA::template load<false>(as, A, lda, m0, k0, ke, a_valid);
            LB::template load<false>(bs, B, ldb, n0, k0, ke, b_valid);
        } else {
            LA::template load<true>(as, A, lda, m0, k0, ke, a_valid);
            LB::template load<true>(bs, B, ldb, n0, k0, ke, b_valid);
        }
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
        const float* as = As + (kt % STAGES) * BK * PA;
        const float* bs = Bs + (kt % STAGES) * BK * PB;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            float a[8], b[JN];
            *reinterpret_cast<float4*>(a) = *reinterpret_cast<const float4*>(as + kk * PA + ty * 4);
            *reinterpret_cast<float4*>(a + 4) = *reinterpret_cast<const float4*>(as + kk * PA + 64 + ty * 4);
#pragma unroll
            for (int q = 0; q < JN / 4; ++q)
                *reinterpret_cast<float4*>(b + 4 * q) = *reinterpret_cast<const float4*>(bs + kk * PB + 64 * q + tx * 4);
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < JN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
    }
    cp_async_wait<0>();

    // Rows ty*4 .. ty*4+3 of one column are contiguous in column-major C:
    // one 16-byte access when the destination allows it.
    float* out_base = PARTIAL ? W + (long)blockIdx.z * M * N : C;
    const long ldo = PARTIAL ? (long)M : ldc;
    const bool vec_ok = tri == 0 && (reinterpret_cast<uintptr_t>(out_base) % 16 == 0) && (ldo % 4 == 0);
#pragma unroll
    for (int j = 0; j < JN; ++j) {
        const int col = n0 + (j / 4) * 64 + tx * 4 + (j % 4);
        if (col >= N) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int row0 = m0 + h * 64 + ty * 4;
            float* cp = out_base + (long)col * ldo + row0;
            if (vec_ok && row0 + 3 < M) {
                float4 v;
                v.x = acc[h * 4 + 0][j];
                v.y = acc[h * 4 + 1][j];
                v.z = acc[h * 4 + 2][j];
                v.w = acc[h * 4 + 3][j];
                if (!PARTIAL) {
                    v.x *= alpha;
                    v.y *= alpha;
                    v.z *= alpha;
                    v.w *= alpha;
                    if (beta != 0.f) {
                        const float4 c0 = *reinterpret_cast<const float4*>(cp);
                        v.x = fmaf(beta, c0.x, v.x);
                        v.y = fmaf(beta, c0.y, v.y);
                        v.z = fmaf(beta, c0.z, v.z);
                        v.w = fmaf(beta, c0.w, v.w);
                    }
                }
                *reinterpret_cast<float4*>(cp) = v;
                continue;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int row = row0 + i;
                if (row >= M) continue;
                if (tri == 1 ? row > col : (tri == 2 && row < col)) continue;
                if (PARTIAL) {
                    cp[i] = acc[h * 4 + i][j];
                } else {
                    float out = alpha * acc[h * 4 + i][j];
                    if (beta != 0.f) out = fmaf(beta, cp[i], out);
                    cp[i] = out;
                }
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

template <bool AM, bool BM_, int VEC, bool PARTIAL, int BN>
cudaError_t launch_f32(const GemmArgsF32& g, int splits, int k_chunk, float* W, cudaStream_t st) {
    constexpr size_t SMEM =
        (size_t)Cfg<BN>::STAGES * Cfg<BN>::BK * (pitch(kBM) + pitch(BN)) * sizeof(float);
    auto kern = sgemm_ffma_kernel<AM, BM_, VEC, PARTIAL, BN>;
    cudaError_t e = ensure_dynamic_smem(kern, (int)SMEM);
    if (e != cudaSuccess) return e;
    dim3 grid((g.m + kBM - 1) / kBM, (g.n + BN - 1) / BN, splits);
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
    if (am == AM && bm == BMF && vec == V) return launch_f32<AM, BMF, V, PARTIAL, 128>(g, splits, k_chunk, W, st);
    ZB_CASE(false, false, 1) ZB_CASE(false, true, 1) ZB_CASE(true, false, 1) ZB_CASE(true, true, 1)
    ZB_CASE(false, true, 4) ZB_CASE(true, false, 4) ZB_CASE(true, true, 4)
#undef ZB_CASE
    if (!am && !bm) return launch_f32<false, false, 1, PARTIAL, 128>(g, splits, k_chunk, W, st);
    return cudaErrorInvalidValue;
}

}  // namespace

namespace {

// dst (cols x rows, column-major, ld ldd) = transpose of src (rows x cols, ld lds).
__global__ void __launch_bounds__(256) transpose_f32(int rows, int cols, const float* __restrict__ src, long lds,
                                                     float* __restrict__ dst, long ldd) {
    __shared__ float t[32][33];
    const int r0 = blockIdx.x * 32;
    for (long c0 = (long)blockIdx.y * 32; c0 < cols; c0 += (long)gridDim.y * 32) {
#pragma unroll
        for (int j = threadIdx.y; j < 32; j += 8) {
            const int r = r0 + threadIdx.x;
            const long c = c0 + j;
            if (r < rows && c < cols) t[j][threadIdx.x] = src[r + c * lds];
        }
        __syncthreads();
#pragma unroll
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long c = c0 + threadIdx.x;
            const int r = r0 + j;
            if (r < rows && c < cols) dst[c + (long)r * ldd] = t[threadIdx.x][j];
        }
        __syncthreads();
    }
}

cudaError_t transpose(int rows, int cols, const float* src, long lds, float* dst, long ldd, cudaStream_t st) {
    dim3 grid((rows + 31) / 32, (unsigned)std::min<long>((cols + 31) / 32, 65535));
    transpose_f32<<<grid, dim3(32, 8), 0, st>>>(rows, cols, src, lds, dst, ldd);
    count_launch();
    return cudaGetLastError();
}

constexpr size_t kAlignElems = 64;  // 256-byte alignment of the workspace parts
size_t align_elems(size_t x) { return (x + kAlignElems - 1) / kAlignElems * kAlignElems; }
long pad4(long x) { return (x + 3) & ~3L; }

// A K-contiguous operand (A with op = T, B with op = N) is copied out
// MN-contiguous first when the product is large enough for the copy (one
// HBM read + write of the operand, ~8 bytes per element) to cost less than
// the slower transposing tile loads (~12 % of the FFMA time at 8192^3):
// the other output dimension must be >= 1024 and the copy <= 1 GiB.
constexpr long kRelayoutMinOther = 1024;
constexpr size_t kRelayoutMaxBytes = size_t(1) << 30;

struct Relayout {
    bool a = false, b = false;
    size_t splitk = 0, a_elems = 0, b_elems = 0;  // workspace parts, in floats
};

Relayout relayout_plan(char transa, char transb, int m, int n, int k, const GemmPlan& plan) {
    Relayout r;
    r.splitk = align_elems(splitk_workspace_elems(m, n, plan.splits));
    // the matrix-vector, narrow and tall-skinny kernels read either layout directly (the
    // tall-skinny route, K <= 64, never splits K either, so it needs no workspace at all,
    // e.g. on a stream under graph capture)
    if (plan.tile == TILE_GEMV || plan.tile == TILE_NARROW_N || plan.tile == TILE_NARROW_M ||
        skinny_gemm_applies(m, n, k, 0))
        return r;
    const size_t a_elems = align_elems((size_t)pad4(m) * (size_t)k);
    const size_t b_elems = align_elems((size_t)pad4(n) * (size_t)k);
    r.a = transa != 'N' && n >= kRelayoutMinOther && a_elems * sizeof(float) <= kRelayoutMaxBytes;
    r.b = transb == 'N' && m >= kRelayoutMinOther && b_elems * sizeof(float) <= kRelayoutMaxBytes;
    r.a_elems = r.a ? a_elems : 0;
    r.b_elems = r.b ? b_elems : 0;
    return r;
}

}  // namespace

size_t sgemm_native_workspace_bytes(char transa, char transb, int m, int n, int k, const GemmPlan& plan) {
    const Relayout r = relayout_plan(transa, transb, m, n, k, plan);
    return (r.splitk + r.a_elems + r.b_elems) * sizeof(float);
}

size_t sgemm_native_workspace_bound(int m, int n, int k, int sm_count) {
    // split-K partials never exceed sm_count x 128 x 128 (GEMV partials
    // kGemvMaxPartials); both copies at most
    return (align_elems((size_t)std::max<long>((long)sm_count * 128 * 128, kGemvMaxPartials)) +
            align_elems((size_t)pad4(m) * k) +
            align_elems((size_t)pad4(n) * k)) * sizeof(float);
}

cudaError_t sgemm_native(const GemmArgsF32& g_in, const GemmPlan& plan, float* workspace, cudaStream_t st) {
    if (plan.tile == TILE_GEMV && gemv_applies(g_in.m, g_in.n, g_in.k, g_in.tri))
        return sgemv_route(g_in, plan.splits, workspace, st);
    if (skinny_gemm_applies(g_in.m, g_in.n, g_in.k, g_in.tri)) {
        static const bool tma = [] {  // TMA-fed kernel unless ZYNUM_GPU_SKINNY_TMA=0
            const char* v = std::getenv("ZYNUM_GPU_SKINNY_TMA");
            return !(v && v[0] == '0');
        }();
        return (tma && sgemm_skinny_tma_applies(g_in)) ? sgemm_skinny_tma(g_in, st) : sgemm_skinny(g_in, st);
    }
    if ((plan.tile == TILE_NARROW_N || plan.tile == TILE_NARROW_M) && narrow_gemm_applies(g_in.m, g_in.n, g_in.tri))
        return sgemm_narrow(g_in, plan.splits, workspace, st);
    GemmArgsF32 g = g_in;
    const Relayout r = relayout_plan(g.transa, g.transb, g.m, g.n, g.k, plan);
    if ((r.a || r.b || r.splitk) && !workspace) return cudaErrorInvalidValue;
    float* a_copy = workspace + r.splitk;
    float* b_copy = a_copy + r.a_elems;
    if (r.a) {  // A is k x m (op = T): copy out A' (m x k) and use op = N
        const long ld = pad4(g.m);
        cudaError_t e = transpose(g.k, g.m, g.a, g.lda, a_copy, ld, st);
        if (e != cudaSuccess) return e;
        g.transa = 'N';
        g.a = a_copy;
        g.lda = ld;
    }
    if (r.b) {  // B is k x n (op = N): copy out B' (n x k) and use op = T
        const long ld = pad4(g.n);
        cudaError_t e = transpose(g.k, g.n, g.b, g.ldb, b_copy, ld, st);
        if (e != cudaSuccess) return e;
        g.transb = 'T';
        g.b = b_copy;
        g.ldb = ld;
    }
    // 16-byte copies need 16-byte aligned bases and ld % 4 == 0 on every MN-fast operand.
    bool aligned = true;
    if (g.transa == 'N') aligned = aligned && (reinterpret_cast<uintptr_t>(g.a) % 16 == 0) && (g.lda % 4 == 0);
    if (g.transb != 'N') aligned = aligned && (reinterpret_cast<uintptr_t>(g.b) % 16 == 0) && (g.ldb % 4 == 0);
    const int vec = aligned ? 4 : 1;
    const int splits = plan.splits < 1 ? 1 : plan.splits;
    int k_chunk = (g.k + splits - 1) / splits;
    k_chunk = (k_chunk + 31) / 32 * 32;  // a multiple of every BK
    const int used = (g.k + k_chunk - 1) / k_chunk;
    if (used > 1) {
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
