// Variable-size batched GEMM and TRSM: one persistent kernel per batch.
//
// No counterpart in the reference (Zynum has no batched API); the per-problem
// semantics are those of gemm.zig:1392 and triangular.zig:233.
//
// GEMM: the host turns the batch into a list of work items (chunks of output
// tiles of one problem, with their tile config) ordered longest-first; the
// persistent CTAs claim items in that order from a counter the launch zeroes
// (a memset and the kernel, both graph-capturable and replayable).  Each size
// bucket gets its tile config from the autotuner (batched_host.cpp).  Both
// dtypes run on DMMA tiles (mma.sync m16n8k8 .f64): FP32 operands are widened
// exactly to FP64 in the fragments and C is rounded to FP32 once (18.8 against
// 15.4 TFLOP/s for FFMA tiles on the 20,000-problem batch, and more accurate).
// Operands are staged with cp.async (8- / 4-byte copies: per-problem leading
// dimensions need not be aligned).
//
// TRSM (left side): one CTA solves one whole problem B := alpha op(A)^-1 B:
// for every 64-row diagonal block, substitution on the block held in shared
// memory, then the rank-64 update of the rows below (above) it with the
// solved rows kept in shared memory.
#include <algorithm>

#include "batched.h"
#include "common.cuh"

namespace zb {
namespace {

constexpr int kThreads = 256;
constexpr int kBK = 16;
constexpr int kStagesD = 2;  // two cp.async stages (64 x 64 tiles: 20 KB FP64), four CTAs per SM

template <typename T>
struct Prob {
    int m, n, k, lda, ldb, ldc;
    const T* a;
    const T* b;
    T* c;
};

// ------------------------------------------------------------- loaders
// smem[r][c] (pitch `pitch`) = base[(r0 + r) * ld + c0 + c], zero outside
// r_lim x c_lim.  vec: 16-byte copies (base 16-byte aligned, ld and c0 a
// multiple of 16 / sizeof(T), pitch likewise), a partial copy zero-filling the
// ragged edge; otherwise one copy per element (any ld, any alignment).
template <typename T, int ROWS, int COLS>
ZB_DEVICE void load_tile(T* smem, int pitch, const T* __restrict__ base, long ld, int r0, int c0, int r_lim,
                         int c_lim, bool vec) {
    constexpr int V = 16 / sizeof(T);
    if (vec) {
        constexpr int CPR = COLS / V, TOTAL = ROWS * CPR;
#pragma unroll
        for (int it = 0; it < (TOTAL + kThreads - 1) / kThreads; ++it) {
            const int q = it * kThreads + threadIdx.x;
            if (TOTAL % kThreads != 0 && q >= TOTAL) break;
            const int r = q / CPR, c = (q % CPR) * V;
            const int gr = r0 + r, gc = c0 + c;
            const int valid = gr < r_lim ? max(0, min(V, c_lim - gc)) : 0;
            const T* src = valid ? base + (long)gr * ld + gc : base;
            cp_async_16(smem_u32(smem + r * pitch + c), src, valid * (int)sizeof(T));
        }
        return;
    }
    constexpr int TOTAL = ROWS * COLS;
#pragma unroll
    for (int it = 0; it < (TOTAL + kThreads - 1) / kThreads; ++it) {
        const int q = it * kThreads + threadIdx.x;
        if (TOTAL % kThreads != 0 && q >= TOTAL) break;
        const int r = q / COLS, c = q % COLS;
        const int gr = r0 + r, gc = c0 + c;
        const bool ok = gr < r_lim && gc < c_lim;
        const T* src = ok ? base + (long)gr * ld + gc : base;
        if (sizeof(T) == 8)
            cp_async_8(smem_u32(smem + r * pitch + c), src, ok ? 8 : 0);
        else
            cp_async_4(smem_u32(smem + r * pitch + c), src, ok ? 4 : 0);
    }
}

// 16-byte copies are possible for an operand whose base is 16-byte aligned and
// whose leading dimension is a multiple of 16 bytes.
template <typename T>
ZB_DEVICE bool vec_ok(const T* base, int ld) {
    return ((reinterpret_cast<uintptr_t>(base) & 15) == 0) && ((ld * (int)sizeof(T)) % 16 == 0);
}

// ------------------------------------------------------- FP64 DMMA tile
// One kBK-deep slice of a warp's products on its first MIV x NIV fragments
// (the others lie outside the problem).  The fragment counts are compile-time
// so that skipped fragments issue nothing at all: a run-time test around a
// DMMA becomes a predicated DMMA, which still occupies the pipe.
template <int MI, int NI, int MIV, int NIV, int A_PITCH, int B_PITCH, bool AK, bool BKF, typename T>
ZB_DEVICE void dmma_slice(double (&acc)[MI][NI][4], const T* as, const T* bs, int wm, int wn, int g, int t) {
#pragma unroll
    for (int ks = 0; ks < kBK; ks += 8) {
        double af[MIV][4], bf[NIV][2];
#pragma unroll
        for (int i = 0; i < MIV; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int rr = wm + i * 16 + g + 8 * (v & 1), kk = ks + t + 4 * (v >> 1);
                af[i][v] = (double)(AK ? as[rr * A_PITCH + kk] : as[kk * A_PITCH + rr]);
            }
#pragma unroll
        for (int j = 0; j < NIV; ++j)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const int cc = wn + j * 8 + g, kk = ks + t + 4 * v;
                bf[j][v] = (double)(BKF ? bs[cc * B_PITCH + kk] : bs[kk * B_PITCH + cc]);
            }
#pragma unroll
        for (int i = 0; i < MIV; ++i)
#pragma unroll
            for (int j = 0; j < NIV; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
    }
}

// Variant V = MIV * (NI + 1) + NIV, chosen by a chain of warp-uniform branches.
template <int MI, int NI, int V, int A_PITCH, int B_PITCH, bool AK, bool BKF, typename T>
ZB_DEVICE void dmma_slice_var(int var, double (&acc)[MI][NI][4], const T* as, const T* bs, int wm, int wn, int g,
                              int t) {
    constexpr int MIV = V / (NI + 1), NIV = V % (NI + 1);
    if (var == V) {
        if constexpr (MIV > 0 && NIV > 0)
            dmma_slice<MI, NI, MIV, NIV, A_PITCH, B_PITCH, AK, BKF>(acc, as, bs, wm, wn, g, t);
        return;
    }
    if constexpr (V > 0) dmma_slice_var<MI, NI, V - 1, A_PITCH, B_PITCH, AK, BKF>(var, acc, as, bs, wm, wn, g, t);
}


// One BM x BN output tile: 8 warps as WARPS_M x (8 / WARPS_M), warp tile
// WM x WN of 16 x 8 DMMA fragments, kStagesD cp.async stages of kBK-deep A and
// B slices (16-byte copies where the operand allows them).  T = float: FP32
// operands staged as FP32 and widened exactly to FP64 in the fragments; the
// products and sums are FP64 and C = alpha acc + beta C is rounded to FP32 once.
// Row pitches: 4 extra elements for k-contiguous rows; m- / n-contiguous rows
// 4 extra doubles or 8 extra floats, which keeps the fragment loads conflict-free.
template <typename T>
constexpr int mn_pad() {
    return sizeof(T) == 8 ? 4 : 8;
}
template <int BM, int BN, int WARPS_M, bool AK, bool BKF, typename T = double>
ZB_DEVICE void dgemm_tile(const Prob<T>& p, int m0, int n0, double alpha, double beta, T* smem) {
    constexpr int WARPS_N = 8 / WARPS_M;
    constexpr int WM = BM / WARPS_M, WN = BN / WARPS_N, MI = WM / 16, NI = WN / 8;
    constexpr int A_ROWS = AK ? BM : kBK, A_COLS = AK ? kBK : BM, A_PITCH = A_COLS + (AK ? 4 : mn_pad<T>());
    constexpr int B_ROWS = BKF ? BN : kBK, B_COLS = BKF ? kBK : BN, B_PITCH = B_COLS + (BKF ? 4 : mn_pad<T>());
    constexpr int A_STAGE = A_ROWS * A_PITCH, B_STAGE = B_ROWS * B_PITCH;
    T* As = smem;
    T* Bs = smem + kStagesD * A_STAGE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp / WARPS_N) * WM, wn = (warp % WARPS_N) * WN;
    const int g = lane >> 2, t = lane & 3;
    const int KT = (alpha == 0.0) ? 0 : (p.k + kBK - 1) / kBK;  // alpha == 0: A and B are not read
    const bool va = vec_ok(p.a, p.lda), vb = vec_ok(p.b, p.ldb);
    // fragments of this warp inside the problem: the first miv row and niv column fragments
    const int miv = max(0, min(MI, (p.m - m0 - wm + 15) / 16)), niv = max(0, min(NI, (p.n - n0 - wn + 7) / 8));
    const int var = miv * (NI + 1) + niv;
    double acc[MI][NI][4];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * kBK;
        if (AK)
            load_tile<T, A_ROWS, A_COLS>(As + stage * A_STAGE, A_PITCH, p.a, p.lda, m0, k0, p.m, p.k, va);
        else
            load_tile<T, A_ROWS, A_COLS>(As + stage * A_STAGE, A_PITCH, p.a, p.lda, k0, m0, p.k, p.m, va);
        if (BKF)
            load_tile<T, B_ROWS, B_COLS>(Bs + stage * B_STAGE, B_PITCH, p.b, p.ldb, n0, k0, p.n, p.k, vb);
        else
            load_tile<T, B_ROWS, B_COLS>(Bs + stage * B_STAGE, B_PITCH, p.b, p.ldb, k0, n0, p.k, p.n, vb);
    };
#pragma unroll
    for (int s = 0; s < kStagesD - 1; ++s) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<kStagesD - 2>();
        __syncthreads();
        if (kt + kStagesD - 1 < KT) load_stage((kt + kStagesD - 1) % kStagesD, kt + kStagesD - 1);
        cp_async_commit();
        const T* as = As + (kt % kStagesD) * A_STAGE;
        const T* bs = Bs + (kt % kStagesD) * B_STAGE;
        if (var == MI * (NI + 1) + NI)  // the whole warp tile inside the problem
            dmma_slice<MI, NI, MI, NI, A_PITCH, B_PITCH, AK, BKF>(acc, as, bs, wm, wn, g, t);
        else
            dmma_slice_var<MI, NI, MI * (NI + 1) + NI - 1, A_PITCH, B_PITCH, AK, BKF>(var, acc, as, bs, wm, wn, g, t);
    }
    cp_async_wait<0>();
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int row = m0 + wm + i * 16 + g + 8 * (v >> 1);
                const int col = n0 + wn + j * 8 + 2 * t + (v & 1);
                if (row < p.m && col < p.n) {
                    T* cp = p.c + (long)col * p.ldc + row;
                    double out = alpha * acc[i][j][v];
                    if (beta != 0.0) out = fma(beta, (double)*cp, out);
                    *cp = (T)out;
                }
            }
    __syncthreads();  // shared memory is reused by the next tile
}

// A chunk of `count` consecutive output tiles t0 .. t0 + count - 1 of one
// problem (tile t: rows (t % mt) BM.., columns (t / mt) BN.., mt = ceil(m / BM)):
// the problem's sizes, pointers and leading dimensions are read once per chunk.
// (Carrying the cp.async stream across the chunk's tile boundaries measured
// slower than restarting it per tile.)
template <int BM, int BN, int WARPS_M, bool AK, bool BKF, typename T = double>
ZB_DEVICE void dgemm_chunk(const Prob<T>& p, int t0, int count, double alpha, double beta, T* smem) {
    const int mt = (p.m + BM - 1) / BM;
    for (int tile = t0; tile < t0 + count; ++tile)
        dgemm_tile<BM, BN, WARPS_M, AK, BKF, T>(p, (tile % mt) * BM, (tile / mt) * BN, alpha, beta, smem);
}

// ------------------------------------------------- persistent kernels
// Work items are claimed in list order (the host sorts them longest first)
// from a device counter the launch zeroes: a CTA that finishes early takes
// the next item, so the batch ends within about one item of its ideal
// (greedy longest-first list scheduling).  Thread 0 claims the following item
// while the CTA works on the current one.  Every tile is computed the same
// way whichever CTA takes it, so results do not depend on the schedule.
template <typename Fn>
ZB_DEVICE void for_each_claimed(int* next, int n_work, Fn fn) {
    __shared__ int s_item[2];
    if (threadIdx.x == 0) s_item[0] = atomicAdd(next, 1);
    __syncthreads();
    int buf = 0;
    for (int w = s_item[0]; w < n_work;) {
        if (threadIdx.x == 0) s_item[buf ^ 1] = atomicAdd(next, 1);
        fn(w);
        __syncthreads();
        buf ^= 1;
        w = s_item[buf];
    }
}

// The same claiming as a loop header, for bodies that use `continue`:
//   ZB_CLAIMED_LOOP(w, next, count) { ... }
// (the increment step holds the CTA-wide barrier that publishes the next claim).
struct Claim {
    int* next;
    int* slot;  // two shared-memory slots
    int buf = 0;
    ZB_DEVICE int first() {
        if (threadIdx.x == 0) slot[0] = atomicAdd(next, 1);
        __syncthreads();
        return slot[0];
    }
    ZB_DEVICE void prefetch() {
        if (threadIdx.x == 0) slot[buf ^ 1] = atomicAdd(next, 1);
    }
    ZB_DEVICE int advance() {
        __syncthreads();
        buf ^= 1;
        return slot[buf];
    }
};

// FP64: 64 x 64 tiles at most, four CTAs per SM (measured: 4 CTAs x 2 stages of 64 x 64 >
// 3 x 3 of 64 x 64 > 2 x 3 with 128 x 64 tiles, 15.8 / 15.4 / 13.9 TFLOP/s on the 20,000-problem
// batch: more tiles in flight hide each tile's start-up latency)
template <bool AK, bool BKF>
__global__ void __launch_bounds__(kThreads, 4)
dgemm_batched_kernel(const BatchWork* __restrict__ work, int n_work, int* __restrict__ next,
                     const int* __restrict__ dims, const double* const* __restrict__ a, const int* __restrict__ lda,
                     const double* const* __restrict__ b, const int* __restrict__ ldb, double alpha, double beta,
                     double* const* __restrict__ c, const int* __restrict__ ldc) {
    extern __shared__ __align__(128) double sm_d[];
    for_each_claimed(next, n_work, [&](int w) {
        const BatchWork it = work[w];
        const int q = it.prob;
        Prob<double> p{dims[3 * q], dims[3 * q + 1], dims[3 * q + 2], lda[q], ldb[q], ldc[q], a[q], b[q], c[q]};
        // tile edges: batched_tile_m / batched_tile_n (FP64: TILE_CFG_128 runs as 64 x 64)
        if (it.cfg == TILE_CFG_128 || it.cfg == TILE_CFG_64)
            dgemm_chunk<64, 64, 2, AK, BKF>(p, it.t0, it.count, alpha, beta, sm_d);
        else
            dgemm_chunk<32, 32, 2, AK, BKF>(p, it.t0, it.count, alpha, beta, sm_d);
    });
}

// FP32 batches run on the same DMMA tiles: operands staged as FP32 and widened
// exactly to FP64, FP64 products and sums, one rounding of alpha acc + beta C
// to FP32 (on the 20,000-problem batch of sizes log-uniform in [8, 512]: 18.8
// TFLOP/s, against 15.4 for FFMA tiles).
template <bool AK, bool BKF>
__global__ void __launch_bounds__(kThreads, 4)
sgemm_batched_kernel(const BatchWork* __restrict__ work, int n_work, int* __restrict__ next,
                     const int* __restrict__ dims, const float* const* __restrict__ a, const int* __restrict__ lda,
                     const float* const* __restrict__ b, const int* __restrict__ ldb, float alpha, float beta,
                     float* const* __restrict__ c, const int* __restrict__ ldc) {
    extern __shared__ __align__(128) float sm_f[];
    for_each_claimed(next, n_work, [&](int w) {
        const BatchWork it = work[w];
        const int q = it.prob;
        Prob<float> p{dims[3 * q], dims[3 * q + 1], dims[3 * q + 2], lda[q], ldb[q], ldc[q], a[q], b[q], c[q]};
        if (it.cfg == TILE_CFG_128 || it.cfg == TILE_CFG_64)
            dgemm_chunk<64, 64, 2, AK, BKF, float>(p, it.t0, it.count, alpha, beta, sm_f);
        else
            dgemm_chunk<32, 32, 2, AK, BKF, float>(p, it.t0, it.count, alpha, beta, sm_f);
    });
}

size_t dsmem_bytes() {
    // largest FP64 config (64 x 64), worst orientation of each operand
    constexpr size_t a = 64 * (kBK + 4) > kBK * (64 + 4) ? 64 * (kBK + 4) : kBK * (64 + 4);
    constexpr size_t b = 64 * (kBK + 4) > kBK * (64 + 4) ? 64 * (kBK + 4) : kBK * (64 + 4);
    return kStagesD * (a + b) * sizeof(double);
}
size_t ssmem_bytes() {
    // FP32 DMMA tiles, largest config (64 x 64), worst orientation of each operand
    constexpr size_t a = 64 * (kBK + 4) > kBK * (64 + 8) ? 64 * (kBK + 4) : kBK * (64 + 8);
    return kStagesD * 2 * a * sizeof(float);
}

// -------------------------------------------------------- batched TRSM
constexpr int kTB = 64;  // diagonal block
constexpr int kMaxRhs = 64;

template <typename T>
ZB_DEVICE T tri_el(const T* a, long lda, char uplo, char trans, char diag, int r, int c) {
    const int ar = (trans == 'N') ? r : c, ac = (trans == 'N') ? c : r;
    if (ar == ac && diag == 'U') return T(1);
    if (uplo == 'U' && ar > ac) return T(0);
    if (uplo == 'L' && ar < ac) return T(0);
    return a[ar + (long)ac * lda];
}

// One CTA per problem (left side): B (n x r) := alpha op(A)^-1 B, r <= 64.
// For each 64-row diagonal block in solve order:
//  * D (the block of op(A), masked to the stored triangle / unit diagonal) and
//    the block rows X of B go to shared memory;
//  * warp-synchronous substitution: warp w owns right-hand sides w, w + 8, ...,
//    lane l owns block rows l and l + 32; the solved value of row i is
//    broadcast by shuffle and the lanes update their later rows (no block
//    barrier inside the substitution);
//  * the rank-64 update of the rows still to solve runs over 64-row chunks of
//    the op(A) panel staged in shared memory by coalesced cp.async copies:
//    thread (row, group of 16 right-hand sides) accumulates 16 products per
//    panel column from shared-memory operands.
constexpr int kTP = kTB + 1;  // pitch of the diagonal block (column reads conflict-free)
constexpr int kPP = kTB + 4;  // pitch of the transposed panel and of X (16-byte aligned rows)

// One element, zero-filled (and `fallback`, a valid address, not read) when !ok.
template <typename T>
ZB_DEVICE void cp_async_el(T* dst, const T* src, const T* fallback, bool ok) {
    if (sizeof(T) == 8)
        cp_async_8(smem_u32(dst), ok ? src : fallback, ok ? 8 : 0);
    else
        cp_async_4(smem_u32(dst), ok ? src : fallback, ok ? 4 : 0);
}

// Pt[cc][rr] = op(A)[c0 + rr][kb + cc] for rr < rows, cc < sz (zero elsewhere):
// the panel chunk transposed (K-major), loaded coalesced along A's contiguous index.
template <typename T>
ZB_DEVICE void load_panel(T (*Pt)[kPP], const T* A, long la, char trans, int c0, int rows, int kb, int sz) {
    for (int e = threadIdx.x; e < kTB * kTB; e += kThreads) {
        int rr, cc;
        const T* src;
        if (trans == 'N') {
            rr = e % kTB;
            cc = e / kTB;
            src = A + (c0 + rr) + (long)(kb + cc) * la;
        } else {
            cc = e % kTB;
            rr = e / kTB;
            src = A + (kb + cc) + (long)(c0 + rr) * la;
        }
        cp_async_el(&Pt[cc][rr], src, A, rr < rows && cc < sz);
    }
    cp_async_commit();
}

// Warp-synchronous substitution of one 64-row block for the right-hand sides
// w + 8 c, c < CM, of warp w: lane l owns block rows l and l + 32.  Row i's
// solved value (its fully updated value times 1 / D[i][i]) is broadcast by
// shuffle and the lanes update their later rows; a row gets no update after it
// is solved, so each lane keeps its rows' final unscaled values and scales them
// once at the end.  The solve runs in two halves (rows 0..31 and 32..63, in
// solve order) so every register index is known at compile time.
template <typename T, int CM, int HI, bool UPPER>
ZB_DEVICE void substitute_half(T (&x)[2][CM], const T (*D)[kTP], const T* dinv, int sz) {
    const int lane = threadIdx.x & 31;
    const int lo = 32 * HI, hi = min(sz, lo + 32);
    for (int it = lo; it < hi; ++it) {
        const int i = UPPER ? hi - 1 - (it - lo) : it;
        const int li = i & 31;
        const T di = dinv[i];
        T xi[CM];
#pragma unroll
        for (int c = 0; c < CM; ++c) xi[c] = __shfl_sync(0xffffffffu, x[HI][c] * di, li);
        // later rows: for a lower op(A) rows p > i, for an upper one rows p < i
        if (UPPER ? true : HI == 0) {  // the other half of this lane (rows lane + 32 (1 - HI)...)
            const int p = lane + 32 * (1 - HI);
            const bool upd = UPPER ? (HI == 1 && p < i) : (p < sz);
            if (upd) {
                const T dpi = D[p][i];
#pragma unroll
                for (int c = 0; c < CM; ++c) x[1 - HI][c] = fma(-dpi, xi[c], x[1 - HI][c]);
            }
        }
        {
            const int p = lane + 32 * HI;  // this half
            if (UPPER ? p < i : (p > i && p < sz)) {
                const T dpi = D[p][i];
#pragma unroll
                for (int c = 0; c < CM; ++c) x[HI][c] = fma(-dpi, xi[c], x[HI][c]);
            }
        }
    }
}

template <typename T, int CM>
ZB_DEVICE void substitute_block(T (*X)[kPP], const T (*D)[kTP], const T* dinv, int sz, bool upper) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T x[2][CM];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int c = 0; c < CM; ++c) x[h][c] = X[lane + 32 * h][warp + 8 * c];
    if (upper) {
        substitute_half<T, CM, 1, true>(x, D, dinv, sz);
        substitute_half<T, CM, 0, true>(x, D, dinv, sz);
    } else {
        substitute_half<T, CM, 0, false>(x, D, dinv, sz);
        substitute_half<T, CM, 1, false>(x, D, dinv, sz);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const T s = dinv[lane + 32 * h];
#pragma unroll
        for (int c = 0; c < CM; ++c) X[lane + 32 * h][warp + 8 * c] = x[h][c] * s;
    }
}

// Substitution for the warp's share of r right-hand sides (1, 2, 4 or 8 slots).
template <typename T>
ZB_DEVICE void substitute_rhs(T (*X)[kPP], const T (*D)[kTP], const T* dinv, int sz, bool upper, int r) {
    const int warp = threadIdx.x >> 5;
    const int cw = r > warp ? (r - warp + 7) / 8 : 0;
    if (cw > 4)
        substitute_block<T, 8>(X, D, dinv, sz, upper);
    else if (cw > 2)
        substitute_block<T, 4>(X, D, dinv, sz, upper);
    else if (cw > 1)
        substitute_block<T, 2>(X, D, dinv, sz, upper);
    else if (cw == 1)
        substitute_block<T, 1>(X, D, dinv, sz, upper);
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 2)
trsm_batched_kernel(const int* __restrict__ order, int count, int* __restrict__ next, const int* __restrict__ dims, char uplo, char trans,
                    char diag, T alpha, const T* const* __restrict__ a, const int* __restrict__ lda,
                    T* const* __restrict__ b, const int* __restrict__ ldb) {
    extern __shared__ __align__(16) unsigned char trsm_smem[];
    // Two 64 x kPP buffers: the diagonal block D (pitch kTP) during the
    // substitution, then the second buffer of transposed panel chunks.
    T* buf0 = reinterpret_cast<T*>(trsm_smem);
    T(*D)[kTP] = reinterpret_cast<T(*)[kTP]>(buf0);
    T(*Pd)[kPP] = reinterpret_cast<T(*)[kPP]>(buf0);
    T(*X)[kPP] = reinterpret_cast<T(*)[kPP]>(buf0 + kTB * kPP);      // block rows of B
    T(*Pn)[kPP] = reinterpret_cast<T(*)[kPP]>(buf0 + 2 * kTB * kPP);  // panel chunk (transposed)
    T* dinv = buf0 + 3 * kTB * kPP;                                     // 1 / D[i][i]
    const bool upper = (trans == 'N' && uplo == 'U') || (trans != 'N' && uplo == 'L');
    const bool unit = diag == 'U';
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int claim_slot[2];
    Claim cl{next, claim_slot};
    for (int w = cl.first(); w < count; w = cl.advance()) {
        cl.prefetch();
        const int q = order[w];
        const int n = dims[2 * q], r = dims[2 * q + 1];
        const T* A = a[q];
        T* B = b[q];
        const long la = lda[q], lb = ldb[q];
        if (alpha != T(1))  // eight loads in flight per thread before their stores
            for (long e0 = threadIdx.x; e0 < (long)n * r; e0 += 8L * kThreads) {
                T v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long e = e0 + (long)u * kThreads;
                    v[u] = e < (long)n * r ? B[(e % n) + (e / n) * lb] : T(0);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long e = e0 + (long)u * kThreads;
                    if (e < (long)n * r) B[(e % n) + (e / n) * lb] = alpha * v[u];
                }
            }
        __syncthreads();
        const int nblk = (n + kTB - 1) / kTB;
        for (int s = 0; s < nblk; ++s) {
            const int bi = upper ? nblk - 1 - s : s;
            const int kb = bi * kTB, sz = min(kTB, n - kb);
            // D (the stored triangle of op(A)'s block, zero elsewhere, the unit diagonal set
            // below) and X (the block rows of B) by asynchronous copies, all in flight at once
            for (int e = threadIdx.x; e < kTB * kTB; e += kThreads) {
                const int rr = e % kTB, cc = e / kTB;
                const bool in = rr < sz && cc < sz && (upper ? rr <= cc : rr >= cc) && !(unit && rr == cc);
                const int ar = trans == 'N' ? kb + rr : kb + cc, ac = trans == 'N' ? kb + cc : kb + rr;
                cp_async_el(&D[rr][cc], A + ar + (long)ac * la, A, in);
            }
            for (int e = threadIdx.x; e < kTB * kMaxRhs; e += kThreads) {
                const int rr = e % kTB, cc = e / kTB;
                cp_async_el(&X[rr][cc], B + kb + rr + (long)cc * lb, B, rr < sz && cc < r);
            }
            cp_async_commit();
            // rows still to solve after this block; their first panel chunk loads
            // during the substitution
            const int u0 = upper ? 0 : kb + sz, u1 = upper ? kb : n;
            if (u0 < u1) {
                load_panel(Pn, A, la, trans, u0, min(kTB, u1 - u0), kb, sz);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (unit && threadIdx.x < sz) D[threadIdx.x][threadIdx.x] = T(1);
            if (threadIdx.x < kTB) dinv[threadIdx.x] = (unit || threadIdx.x >= sz) ? T(1) : T(1) / D[threadIdx.x][threadIdx.x];
            __syncthreads();
            // ---- substitution (each warp carries only the right-hand sides it has)
            substitute_rhs<T>(X, D, dinv, sz, upper, r);
            __syncthreads();
            for (int e = threadIdx.x; e < kTB * r; e += kThreads) {
                const int rr = e % kTB, cc = e / kTB;
                if (rr < sz) B[kb + rr + (long)cc * lb] = X[rr][cc];
            }
            // ---- rank-sz update of the rows still to solve, 64 rows at a time; the
            // panel chunks alternate between Pn and D (free after the substitution)
            // thread: rows 4 rg .. 4 rg + 3 of the chunk, right-hand sides 4 cg .. 4 cg + 3
            const int rg = threadIdx.x & 15, cg = threadIdx.x >> 4;
            for (int c0 = u0, ci = 0; c0 < u1; c0 += kTB, ++ci) {
                const int rows = min(kTB, u1 - c0);
                T(*P)[kPP] = (ci & 1) ? Pd : Pn;
                if (c0 + kTB < u1) {
                    load_panel((ci & 1) ? Pn : Pd, A, la, trans, c0 + kTB, min(kTB, u1 - c0 - kTB), kb, sz);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                if constexpr (sizeof(T) == 8) {
                    // FP64: the chunk update B[c0 .. c0 + rows) -= P^T X as 16 x 8 DMMA tiles;
                    // warp w takes row tile w % 4 and column tiles 4 (w / 4) .. +3 (those below r)
                    const int g = lane >> 2, tq = lane & 3, rt = warp & 3, ct0 = (warp >> 2) * 4;
                    const int nct = (r + 7) / 8;
                    double acc[4][4] = {}, bv[4][4];
                    if (ct0 < nct) {
                        // the B values this warp updates, in flight before the products
#pragma unroll
                        for (int u = 0; u < 4; ++u)
#pragma unroll
                            for (int v = 0; v < 4; ++v) {
                                const int row = 16 * rt + g + 8 * (v >> 1), col = 8 * (ct0 + u) + 2 * tq + (v & 1);
                                bv[u][v] = (ct0 + u < nct && row < rows && col < r) ? B[c0 + row + (long)col * lb]
                                                                                   : 0.0;
                            }
                        for (int k8 = 0; k8 < (sz + 7) / 8; ++k8) {
                            double af[4];
#pragma unroll
                            for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
                                for (int v0 = 0; v0 < 2; ++v0)
                                    af[v0 + 2 * v1] = P[8 * k8 + tq + 4 * v1][16 * rt + g + 8 * v0];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                if (ct0 + u >= nct) break;
                                double bf[2];
#pragma unroll
                                for (int v = 0; v < 2; ++v) bf[v] = X[8 * k8 + tq + 4 * v][8 * (ct0 + u) + g];
                                dmma_16x8x8(acc[u], af, bf);
                            }
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (ct0 + u >= nct) break;
#pragma unroll
                            for (int v = 0; v < 4; ++v) {
                                const int row = 16 * rt + g + 8 * (v >> 1), col = 8 * (ct0 + u) + 2 * tq + (v & 1);
                                if (row < rows && col < r) B[c0 + row + (long)col * lb] = bv[u][v] - acc[u][v];
                            }
                        }
                    }
                } else if (4 * cg < r) {
                    // the B values this thread updates, fetched before the K loop
                    T bv[4][4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int col = 4 * cg + j, row = 4 * rg + i;
                            bv[i][j] = (col < r && row < rows) ? B[c0 + row + (long)col * lb] : T(0);
                        }
                    T acc[4][4];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
                    for (int p = 0; p < sz; ++p) {
                        T av[4], xv[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) av[i] = P[p][4 * rg + i];
#pragma unroll
                        for (int j = 0; j < 4; ++j) xv[j] = X[p][4 * cg + j];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                            for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], xv[j], acc[i][j]);
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (4 * cg + j >= r) break;
                        T* bp = B + c0 + (long)(4 * cg + j) * lb;
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (4 * rg + i < rows) bp[4 * rg + i] = bv[i][j] - acc[i][j];
                    }
                }
                __syncthreads();
            }
            __syncthreads();
        }
    }
}

// FP64 left-looking solver, one CTA per problem (left side, r <= 64): for each
// 64-row block in solve order, acc = sum over the solved blocks j of
// op(A)[block, j] X_j streams 32-deep K chunks of op(A) and of the solved rows
// X (read back from B) through a two-stage cp.async ring into 16 x 8 DMMA tiles
// held in registers (warp w: row tile w % 4, column tiles 4 (w / 4) .. +3);
// then X_block = B_block - acc is solved in shared memory by a warp-synchronous
// substitution (each warp carries only the right-hand sides it has) and
// written back to B once.  The diagonal block's copy is in flight during the
// products.
constexpr int kLlK = 32;                          // K chunk
constexpr int kLlPitch = kTB + 4;                 // 68: [k][row] and [k][col] tiles
constexpr int kLlStage = 2 * kLlK * kLlPitch;     // A chunk + X chunk, in doubles
constexpr int kLlRing = 2 * kLlStage;             // two stages (also holds the 64 x 68 solve block)

__global__ void __launch_bounds__(kThreads, 2)
trsm_batched_ll_f64(const int* __restrict__ order, int count, int* __restrict__ next, const int* __restrict__ dims, char uplo, char trans,
                    char diag, double alpha, const double* const* __restrict__ a, const int* __restrict__ lda,
                    double* const* __restrict__ b, const int* __restrict__ ldb) {
    extern __shared__ __align__(16) unsigned char ll_smem[];
    double* ring = reinterpret_cast<double*>(ll_smem);
    double(*X)[kPP] = reinterpret_cast<double(*)[kPP]>(ring);  // solve block, after the products
    double(*D)[kTP] = reinterpret_cast<double(*)[kTP]>(ring + kLlRing);
    double* dinv = ring + kLlRing + kTB * kTP;
    const bool upper = (trans == 'N' && uplo == 'U') || (trans != 'N' && uplo == 'L');
    const bool unit = diag == 'U';
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31, g = lane >> 2, tq = lane & 3;
    const int rt = warp & 3, ct0 = (warp >> 2) * 4;
    __shared__ int claim_slot[2];
    Claim cl{next, claim_slot};
    for (int w = cl.first(); w < count; w = cl.advance()) {
        cl.prefetch();
        const int q = order[w];
        const int n = dims[2 * q], r = dims[2 * q + 1];
        const double* A = a[q];
        double* B = b[q];
        const long la = lda[q], lb = ldb[q];
        if (alpha != 1.0)  // eight loads in flight per thread before their stores
            for (long e0 = t; e0 < (long)n * r; e0 += 8L * kThreads) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long e = e0 + (long)u * kThreads;
                    v[u] = e < (long)n * r ? B[(e % n) + (e / n) * lb] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long e = e0 + (long)u * kThreads;
                    if (e < (long)n * r) B[(e % n) + (e / n) * lb] = alpha * v[u];
                }
            }
        __syncthreads();
        const int nblk = (n + kTB - 1) / kTB, nct = (r + 7) / 8;
        for (int s = 0; s < nblk; ++s) {
            const int bi = upper ? nblk - 1 - s : s;
            const int kb = bi * kTB, sz = min(kTB, n - kb);
            // diagonal block: stored triangle of op(A), zero elsewhere (unit diagonal set below)
            for (int e = t; e < kTB * kTB; e += kThreads) {
                const int rr = e % kTB, cc = e / kTB;
                const bool in = rr < sz && cc < sz && (upper ? rr <= cc : rr >= cc) && !(unit && rr == cc);
                const int ar = trans == 'N' ? kb + rr : kb + cc, ac = trans == 'N' ? kb + cc : kb + rr;
                cp_async_el(&D[rr][cc], A + ar + (long)ac * la, A, in);
            }
            cp_async_commit();
            // this thread's B values of the block (DMMA accumulator layout), loaded ahead
            double bv[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = 16 * rt + g + 8 * (v >> 1), col = 8 * (ct0 + u) + 2 * tq + (v & 1);
                    bv[u][v] = (row < sz && col < r) ? B[kb + row + (long)col * lb] : 0.0;
                }
            // solved rows: [0, kb) for a lower op(A), [kb + sz, n) for an upper one
            const int k0 = upper ? kb + sz : 0, k1 = upper ? n : kb;
            const int nch = (k1 - k0 + kLlK - 1) / kLlK;
            auto stage = [&](int c) {
                double(*As)[kLlPitch] = reinterpret_cast<double(*)[kLlPitch]>(ring + (c & 1) * kLlStage);
                double(*Xs)[kLlPitch] = As + kLlK;
                const int kc = k0 + c * kLlK, kw = min(kLlK, k1 - kc);
                for (int e = t; e < kTB * kLlK; e += kThreads) {  // op(A)[kb + row][kc + k] -> As[k][row]
                    int row, k;
                    if (trans == 'N') row = e % kTB, k = e / kTB;
                    else k = e % kLlK, row = e / kLlK;
                    const int ar = trans == 'N' ? kb + row : kc + k, ac = trans == 'N' ? kc + k : kb + row;
                    cp_async_el(&As[k][row], A + ar + (long)ac * la, A, row < sz && k < kw);
                }
                for (int e = t; e < kLlK * kMaxRhs; e += kThreads) {  // X[kc + k][col] = B(kc + k, col) -> Xs[k][col]
                    const int k = e % kLlK, col = e / kLlK;
                    cp_async_el(&Xs[k][col], B + (kc + k) + (long)col * lb, B, k < kw && col < r);
                }
            };
            double acc[4][4] = {};
            if (nch > 0) stage(0);
            cp_async_commit();
            for (int c = 0; c < nch; ++c) {
                if (c + 1 < nch) stage(c + 1);
                cp_async_commit();
                cp_async_wait<1>();
                __syncthreads();
                const double(*As)[kLlPitch] = reinterpret_cast<const double(*)[kLlPitch]>(ring + (c & 1) * kLlStage);
                const double(*Xs)[kLlPitch] = As + kLlK;
                if (ct0 < nct) {
#pragma unroll
                    for (int k8 = 0; k8 < kLlK / 8; ++k8) {
                        double af[4];
#pragma unroll
                        for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
                            for (int v0 = 0; v0 < 2; ++v0) af[v0 + 2 * v1] = As[8 * k8 + tq + 4 * v1][16 * rt + g + 8 * v0];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (ct0 + u >= nct) break;
                            double bf[2];
#pragma unroll
                            for (int v = 0; v < 2; ++v) bf[v] = Xs[8 * k8 + tq + 4 * v][8 * (ct0 + u) + g];
                            dmma_16x8x8(acc[u], af, bf);
                        }
                    }
                }
                __syncthreads();
            }
            cp_async_wait<0>();
            __syncthreads();
            // the block to solve: X = B_block - acc, zero outside sz x r
            for (int e = t; e < kTB * kPP; e += kThreads) X[e / kPP][e % kPP] = 0.0;
            if (unit && t < sz) D[t][t] = 1.0;
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = 16 * rt + g + 8 * (v >> 1), col = 8 * (ct0 + u) + 2 * tq + (v & 1);
                    if (ct0 + u < nct && row < sz && col < r) X[row][col] = bv[u][v] - acc[u][v];
                }
            if (t < kTB) dinv[t] = (unit || t >= sz) ? 1.0 : 1.0 / D[t][t];
            __syncthreads();
            // substitution: warp w holds right-hand sides w + 8 c for the c < cw it has
            // (cw rounded up to 1, 2, 4 or 8 slots; a warp without columns skips it)
            substitute_rhs<double>(X, D, dinv, sz, upper, r);
            __syncthreads();
            for (int e = t; e < kTB * r; e += kThreads) {
                const int rr = e % kTB, cc = e / kTB;
                if (rr < sz) B[kb + rr + (long)cc * lb] = X[rr][cc];
            }
            __syncthreads();  // the solved rows are visible to the next block's copies
        }
    }
}

}  // namespace

// ------------------------------------------------------------------ host
cudaError_t launch_gemm_batched(const BatchDevice& d, int dtype, char transa, char transb, const void* alpha,
                                const void* const* a, const int* lda, const void* const* b, const int* ldb,
                                const void* beta, void* const* c, const int* ldc, int grid, cudaStream_t st) {
    if (d.n_work == 0) return cudaSuccess;
    cudaError_t e;
    if (dtype == BATCH_F64) {
        const bool ak = transa != 'N', bk = transb == 'N';
        const double al = *static_cast<const double*>(alpha), be = *static_cast<const double*>(beta);
        auto A = reinterpret_cast<const double* const*>(a);
        auto B = reinterpret_cast<const double* const*>(b);
        auto Cp = reinterpret_cast<double* const*>(c);
        const size_t sm = dsmem_bytes();
#define ZB_DB(AKV, BKV)                                                                                         \
    if (ak == AKV && bk == BKV) {                                                                               \
        auto kern = dgemm_batched_kernel<AKV, BKV>;                                                             \
        if ((e = ensure_dynamic_smem(kern, (int)sm)) != cudaSuccess) \
            return e;                                                                                           \
        if ((e = cudaMemsetAsync(d.next, 0, sizeof(int), st)) != cudaSuccess) return e;                        \
        prof_begin(st);                                                                                         \
        kern<<<grid, kThreads, sm, st>>>(d.work, d.n_work, d.next, d.dims, A, lda, B, ldb, al, be, Cp, ldc);   \
        count_launch();                                                                                         \
        prof_end(st);                                                                                           \
        return cudaGetLastError();                                                                              \
    }
        ZB_DB(false, false) ZB_DB(false, true) ZB_DB(true, false) ZB_DB(true, true)
#undef ZB_DB
    } else {
        const bool ak = transa != 'N', bk = transb == 'N';
        const float al = *static_cast<const float*>(alpha), be = *static_cast<const float*>(beta);
        auto A = reinterpret_cast<const float* const*>(a);
        auto B = reinterpret_cast<const float* const*>(b);
        auto Cp = reinterpret_cast<float* const*>(c);
        const size_t sm = ssmem_bytes();
#define ZB_SB(AKV, BKV)                                                                                         \
    if (ak == AKV && bk == BKV) {                                                                               \
        auto kern = sgemm_batched_kernel<AKV, BKV>;                                                             \
        if ((e = ensure_dynamic_smem(kern, (int)sm)) != cudaSuccess) \
            return e;                                                                                           \
        if ((e = cudaMemsetAsync(d.next, 0, sizeof(int), st)) != cudaSuccess) return e;                        \
        prof_begin(st);                                                                                         \
        kern<<<grid, kThreads, sm, st>>>(d.work, d.n_work, d.next, d.dims, A, lda, B, ldb, al, be, Cp, ldc);   \
        count_launch();                                                                                         \
        prof_end(st);                                                                                           \
        return cudaGetLastError();                                                                              \
    }
        ZB_SB(false, false) ZB_SB(false, true) ZB_SB(true, false) ZB_SB(true, true)
#undef ZB_SB
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_trsm_batched(const int* order, int count, int* next, const int* dims, int dtype, char uplo,
                                char trans, char diag, const void* alpha, const void* const* a, const int* lda,
                                void* const* b, const int* ldb, int grid, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    const int sm = (3 * kTB * (kTB + 4) + kTB) * (dtype == BATCH_F64 ? 8 : 4);
    const int sm_ll = (kLlRing + kTB * kTP + kTB) * 8;
    cudaError_t e = dtype == BATCH_F64 ? ensure_dynamic_smem(trsm_batched_ll_f64, sm_ll)
                                       : ensure_dynamic_smem(trsm_batched_kernel<float>, sm);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(next, 0, sizeof(int), st)) != cudaSuccess) return e;
    prof_begin(st);
    if (dtype == BATCH_F64)
        trsm_batched_ll_f64<<<grid, kThreads, sm_ll, st>>>(
            order, count, next, dims, uplo, trans, diag, *static_cast<const double*>(alpha),
            reinterpret_cast<const double* const*>(a), lda, reinterpret_cast<double* const*>(b), ldb);
    else
        trsm_batched_kernel<float><<<grid, kThreads, sm, st>>>(
            order, count, next, dims, uplo, trans, diag, *static_cast<const float*>(alpha),
            reinterpret_cast<const float* const*>(a), lda, reinterpret_cast<float* const*>(b), ldb);
    count_launch();
    prof_end(st);
    return cudaGetLastError();
}

int batched_tile_n(int cfg, int dtype) {
    (void)dtype;  // TILE_CFG_128 runs as 64 x 64 (both dtypes on DMMA tiles)
    return cfg == TILE_CFG_64 || cfg == TILE_CFG_128 ? 64 : 32;
}
int batched_tile_m(int cfg, int dtype) { return batched_tile_n(cfg, dtype); }

}  // namespace zb
