// Triangular and symmetric Level-3 routines on the GEMM tiles: TRSM, SYRK,
// SYMM, TRMM and SYR2K.
//
// TRSM  B := alpha * op(A)^-1 * B  (side L)  or  B * op(A)^-1  (side R)
//   Reference: core/matrix_matrix/triangular.zig:233 trsm (alpha pre-scale
//   :51-58, one trsv per right-hand side :103-117, right side row solves :72)
//   and the blocked template structured_blocked.zig:315 tryTrsm (GEMM trailing
//   updates with alpha = -1, beta = 1 at :344/:365).
//   GPU algorithm: all 64 x 64 diagonal blocks of op(A) are inverted in one
//   launch (tri_inv_blocks, exact substitution per column in shared memory);
//   the order is halved recursively on 256-row boundaries, the halves coupled
//   by GEMMs on the native (or Ozaki) tiles (B_rest -= op(A)_rest,J X_J), and
//   each 256-row leaf is solved in place by one trsm_leaf launch (inverted
//   64-blocks and the leaf's own off-diagonal blocks applied in shared memory).
//
// SYRK  C := alpha * op(A) op(A)^T + beta * C on one triangle
//   Reference: core/matrix_matrix/symmetric.zig:237 syrk / runSyrkColumns :180
//   (one dot product per (i, j) of the triangle).  GPU algorithm: the GEMM
//   kernel in triangle mode: tiles outside the triangle are skipped and
//   elements outside it are never written.  SYR2K (symmetric.zig:366 /
//   runSyr2kColumns :301) is two such GEMMs, the second with beta = 1.
//
// SYMM  C := alpha * A * B + beta * C (side L) or alpha * B * A + beta * C,
//   A symmetric with one stored triangle (symmetric.zig:107 / runSymmColumns
//   :56, symValue access.zig:31).  GPU algorithm: the stored triangle is
//   mirrored into a dense scratch copy (one O(n^2) pass through shared-memory
//   transposes), then one GEMM on the native (or Ozaki) tiles.
//
// TRMM  B := alpha * op(A) * B (side L) or alpha * B * op(A), A triangular,
//   in place (triangular.zig:202; left side trmv + scale per column :103-110,
//   right side row products :212-229).  GPU algorithm: B is copied to a
//   scratch W; every 256 x 256 diagonal block of op(A) is written out dense
//   (zeros outside the triangle, ones on a unit diagonal) in one launch and
//   applied as B_J = alpha D_J W_J; the off-diagonal part of op(A) is added by
//   recursive halving on block boundaries, one GEMM (beta = 1) per level and
//   half.  Reading W rather than B makes every GEMM independent of the order.
#include <functional>
#include <type_traits>

#include "common.cuh"
#include "level3.h"

namespace zb {
namespace {

constexpr int kNB = 64;

inline int grid_for(long total) {
    long b = (total + 255) / 256;
    if (b > 148L * 32) b = 148L * 32;
    return b < 1 ? 1 : (int)b;
}

__host__ __device__ inline bool op_is_upper(char uplo, char trans) {
    return (trans == 'N' && uplo == 'U') || (trans != 'N' && uplo == 'L');
}

// Element (r, c) of op(A) for a triangular A (access.zig:54-64 triValue).
template <typename T>
ZB_DEVICE T op_tri(const T* a, long lda, char uplo, char trans, char diag, int r, int c) {
    const int ar = (trans == 'N') ? r : c, ac = (trans == 'N') ? c : r;
    if (ar == ac && diag == 'U') return T(1);
    if (uplo == 'U' && ar > ac) return T(0);
    if (uplo == 'L' && ar < ac) return T(0);
    return conj_if(a[ar + (long)ac * lda], trans == 'C');  // op = C conjugates (access.zig:54-63)
}

// Block b: inverse of the diagonal block op(A)[b*64 .. , b*64 ..] of size
// s <= 64, written column-major with ld 64 (zero outside s x s).  Column j of
// the inverse is solved by the four lanes of quad j % 8 of warp j / 8 (256
// threads): for each row in solve order the lanes add every fourth term of
// sum_q L[r][q] X[q][j], two shuffles combine them, and the row's reciprocal
// diagonal (computed once per block) scales the result.
template <typename T>
__global__ void __launch_bounds__(256) tri_inv_blocks(const T* __restrict__ a, long lda, char uplo, char trans,
                                                      char diag, int n, T* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char tri_smem[];  // 2 x 64 x 65 elements + 64 reciprocals
    T(*L)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(tri_smem);
    T(*X)[kNB + 1] = L + kNB;
    T* dinv = reinterpret_cast<T*>(X + kNB);
    grid_dependency_wait();  // may start during the tail of the kernel before it (which may write A)
    const int b0 = blockIdx.x * kNB;
    const int s = min(kNB, n - b0);
    const int t = threadIdx.x;
    // all sixteen loads of a thread in flight before the first shared store
    constexpr int kIt = kNB * kNB / 256;
    T pre[kIt];
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
        const int q = i * 256 + t, r = q % kNB, c = q / kNB;
        pre[i] = (r < s && c < s) ? op_tri(a, lda, uplo, trans, diag, b0 + r, b0 + c) : T(0);
    }
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
        const int q = i * 256 + t, r = q % kNB, c = q / kNB;
        L[r][c] = pre[i];
        X[r][c] = T(0);
    }
    __syncthreads();
    if (t < kNB) dinv[t] = (t < s && diag != 'U') ? T(1) / L[t][t] : T(1);
    __syncthreads();
    const bool upper = op_is_upper(uplo, trans);
    const int lane = t & 31, j = (t >> 5) * 8 + (lane >> 2), part = lane & 3;
    for (int step = 0; step < kNB; ++step) {
        const int r = upper ? kNB - 1 - step : step;
        const bool active = j < s && r < s && (upper ? r <= j : r >= j);
        T v = T(0);
        if (active) {
            if (!upper) {
                for (int q = j + part; q < r; q += 4) v = fma(L[r][q], X[q][j], v);
            } else {
                for (int q = r + 1 + part; q <= j; q += 4) v = fma(L[r][q], X[q][j], v);
            }
        }
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        if (active && part == 0) X[r][j] = ((r == j ? T(1) : T(0)) - v) * dinv[r];
        __syncwarp();
    }
    __syncthreads();
    T* o = out + (long)blockIdx.x * kNB * kNB;
    for (int q = t; q < kNB * kNB; q += 256) o[q] = X[q % kNB][q / kNB];
}

// One TRSM leaf of up to kLeaf rows (up to four diagonal 64-blocks), solved in
// place for the 16 right-hand sides of this CTA: M Y = Z, where for side L
// M = op(A)[p0.., p0..] and Z = B[p0.., c0 .. c0+15]; for side R (X op(A) = B,
// i.e. op(A)^T X^T = B^T) M = op(A)[p0.., p0..]^T and Z = B[c0 .. c0+15, p0..]^T.
// Z lives in shared memory; step by step (forward for a lower M, backward for
// an upper one) Y_s = inv(M_ss) Z_s with the inverted 64-block of op(A) (read
// transposed for side R), then Z_t -= M_ts Y_s for the later blocks t of the
// leaf.  Each thread owns 4 rows x 1 column of a 64 x 16 block.
constexpr int kLeaf = 256;
constexpr int kLeafCols = 16;

template <typename T>
__global__ void __launch_bounds__(256)
trsm_leaf(const T* __restrict__ a, long lda, int trans_n, int conj_a, int left, int fwd, const T* __restrict__ inv,
          int p0, int len, T* __restrict__ b, long ldb, int ncols) {
    extern __shared__ __align__(16) unsigned char leaf_smem[];
    T(*Z)[kLeafCols + 1] = reinterpret_cast<T(*)[kLeafCols + 1]>(leaf_smem);
    T(*W)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(leaf_smem + sizeof(T) * kLeaf * (kLeafCols + 1));
    const int t = threadIdx.x;
    const int c0 = blockIdx.x * kLeafCols;
    const int nc = min(kLeafCols, ncols - c0);
    // Z(r, c): side L b[(p0 + r) + (c0 + c) ldb], side R b[(c0 + c) + (p0 + r) ldb]
    for (int idx = t; idx < kLeaf * kLeafCols; idx += 256) {
        const int r = left ? idx % kLeaf : idx / kLeafCols, c = left ? idx / kLeaf : idx % kLeafCols;
        T v = T(0);
        if (r < len && c < nc)
            v = left ? b[(p0 + r) + (long)(c0 + c) * ldb] : b[(c0 + c) + (long)(p0 + r) * ldb];
        Z[r][c] = v;
    }
    // M(i, j) = op(A)(p0 + i, p0 + j) (side L) or op(A)(p0 + j, p0 + i) (side R); op(A)(r, c) is
    // a[r + c lda] for trans N, a[c + r lda] otherwise; the storage row is contiguous
    const bool i_contig = (left != 0) == (trans_n != 0);
    auto load_m = [&](int bt, int bs) {  // W = M[bt*64 .., bs*64 ..], zero outside the leaf
        for (int idx = t; idx < kNB * kNB; idx += 256) {
            const int i = i_contig ? idx % kNB : idx / kNB, j = i_contig ? idx / kNB : idx % kNB;
            const int gi = bt * kNB + i, gj = bs * kNB + j;
            T v = T(0);
            if (gi < len && gj < len) {
                const int r = left ? p0 + gi : p0 + gj, c = left ? p0 + gj : p0 + gi;
                v = conj_if(trans_n ? a[r + (long)c * lda] : a[c + (long)r * lda], conj_a != 0);
            }
            W[i][j] = v;
        }
    };
    const int nsb = (len + kNB - 1) / kNB;
    const int c = t & (kLeafCols - 1), rg = (t >> 4) * 4;  // 4 rows rg .. rg+3 of a 64-block, column c
    for (int step = 0; step < nsb; ++step) {
        const int sb = fwd ? step : nsb - 1 - step;
        const T* ib = inv + (long)(p0 / kNB + sb) * kNB * kNB;
        __syncthreads();
        for (int idx = t; idx < kNB * kNB; idx += 256) {  // W = inv(M_ss): inv block, transposed for side R
            const int i = idx % kNB, j = idx / kNB;
            W[i][j] = left ? ib[i + j * kNB] : ib[j + i * kNB];
        }
        __syncthreads();
        T y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) y[u] = T(0);
        for (int q = 0; q < kNB; ++q) {
            const T z = Z[sb * kNB + q][c];
#pragma unroll
            for (int u = 0; u < 4; ++u) y[u] = fma(W[rg + u][q], z, y[u]);
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) Z[sb * kNB + rg + u][c] = y[u];
        for (int o = 1; o < nsb; ++o) {  // the later blocks of the solve order
            const int tb = fwd ? sb + o : sb - o;
            if (tb < 0 || tb >= nsb) break;
            __syncthreads();
            load_m(tb, sb);
            __syncthreads();
            T acc[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] = Z[tb * kNB + rg + u][c];
            for (int q = 0; q < kNB; ++q) {
                const T z = Z[sb * kNB + q][c];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(-W[rg + u][q], z, acc[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) Z[tb * kNB + rg + u][c] = acc[u];
        }
    }
    __syncthreads();
    for (int idx = t; idx < kLeaf * kLeafCols; idx += 256) {
        const int r = left ? idx % kLeaf : idx / kLeafCols, cc = left ? idx / kLeaf : idx % kLeafCols;
        if (r < len && cc < nc) {
            if (left)
                b[(p0 + r) + (long)(c0 + cc) * ldb] = Z[r][cc];
            else
                b[(c0 + cc) + (long)(p0 + r) * ldb] = Z[r][cc];
        }
    }
}

// FP64 TRSM leaves through their inverses.  tri_inv_leaf turns the inverted
// 64-blocks into the full inverse of every kLeaf-row diagonal block of op(A)
// (one launch for all leaves, off the solve's critical chain); each leaf of
// the solve is then one trsm_leaf_apply launch, Y = inv(M) Z, a single pass
// of DMMA tiles with no dependent phases.
constexpr int kStagePitch = kNB + 2;  // 66 doubles: 16-byte aligned shared rows

// Stage the 64 x 64 block whose element (r, c) sits at base[r * sr + c * sc],
// exactly one of sr / sc being 1, into W with the contiguous index innermost
// (W[c][r] when sr == 1, W[r][c] otherwise) by 16-byte cp.async; elements with
// r >= rlim or c >= clim are zero.  Needs base, the other stride and the
// shared rows 16-byte aligned.
ZB_DEVICE void stage_block(double (*W)[kStagePitch], const double* base, long sr, long sc, int rlim, int clim,
                           const double* dummy) {
    const bool rfast = sr == 1;
    const long ld = rfast ? sc : sr;
    const int lim_in = rfast ? rlim : clim, lim_out = rfast ? clim : rlim;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        const int q = it * 256 + threadIdx.x;
        const int inner = (q & 31) * 2, outer = q >> 5;
        const int valid = outer < lim_out ? max(0, min(2, lim_in - inner)) : 0;
        const double* src = valid ? base + inner + (long)outer * ld : dummy;
        cp_async_16(smem_u32(&W[outer][inner]), src, valid * 8);
    }
}

// element (r, c) of a block staged by stage_block
ZB_DEVICE double staged(const double (*W)[kStagePitch], bool rfast, int r, int c) {
    return rfast ? W[c][r] : W[r][c];
}

// acc[u] += A (64 x 64, staged) * B (64 x 64 in X[k][c]) for this warp's tiles:
// row tile rt = warp / 2, column tiles 4 (warp % 2) + u.
ZB_DEVICE void mma_64(double (&acc)[4][4], const double (*A)[kStagePitch], bool arfast, const double (*B)[kNB + 1]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3, rt = warp >> 1, ct0 = (warp & 1) * 4;
#pragma unroll
    for (int kb = 0; kb < kNB / 8; ++kb) {
        double af[4];
#pragma unroll
        for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
            for (int v0 = 0; v0 < 2; ++v0)
                af[v0 + 2 * v1] = staged(A, arfast, 16 * rt + g + 8 * v0, 8 * kb + tq + 4 * v1);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            double bf[2];
#pragma unroll
            for (int v = 0; v < 2; ++v) bf[v] = B[8 * kb + tq + 4 * v][8 * (ct0 + u) + g];
            dmma_16x8x8(acc[u], af, bf);
        }
    }
}

// Block (leaf, j): column block j of the inverse of the diagonal kLeaf-block
// `leaf` of op(A), written to inv_leaf + leaf kLeaf^2 (column-major, ld kLeaf;
// zero outside the triangle and the leaf).  Lower op(A): X_jj = inv(A_jj),
// X_ij = -inv(A_ii) sum_{k=j}^{i-1} A_ik X_kj for i = j+1, ...; upper op(A):
// the same for i = j-1, ..., 0 with k = i+1 .. j.  The 64-blocks this takes
// (inv(A_jj), then per row block i its A_ik and inv(A_ii)) are known up front:
// they are staged through two shared buffers, the next one loading while the
// current one is used (a load-then-use sequence waited out one L2 or DRAM
// round trip per block).
__global__ void __launch_bounds__(256)
tri_inv_leaf(const double* __restrict__ a, long lda, int trans_n, int upper, int na, const double* __restrict__ inv64,
             double* __restrict__ inv_leaf) {
    extern __shared__ __align__(16) unsigned char til_smem[];
    double(*X)[kNB][kNB + 1] = reinterpret_cast<double(*)[kNB][kNB + 1]>(til_smem);
    double(*S0)[kStagePitch] =
        reinterpret_cast<double(*)[kStagePitch]>(til_smem + sizeof(double) * 4 * kNB * (kNB + 1));
    double(*S1)[kStagePitch] = S0 + kNB;
    grid_dependency_wait();  // launched during the tail of tri_inv_blocks
    const int leaf = blockIdx.x, j = blockIdx.y, t = threadIdx.x;
    const int P = leaf * kLeaf, len = min(kLeaf, na - P), nsb = (len + kNB - 1) / kNB;
    double* out = inv_leaf + (long)leaf * kLeaf * kLeaf;
    bool have[4] = {false, false, false, false};
    if (j < nsb) {
        // op(A)(r, c) = a[r + c lda] (trans N) or a[c + r lda]; block (bi, bk) of the leaf
        const long sr = trans_n ? 1 : lda, sc = trans_n ? lda : 1;
        auto ablock = [&](int bi, int bk) { return a + (long)(P + bi * kNB) * sr + (long)(P + bk * kNB) * sc; };
        auto iblock = [&](int bi) { return inv64 + (long)(P / kNB + bi) * kNB * kNB; };
        // steps: 0 = inv(A_jj); then for o = 1, 2, ..: A_ik for k = k0(i) .. k1(i) (o blocks), inv(A_ii)
        const int nrows = upper ? j : nsb - 1 - j;  // row blocks i below (above) j
        const int nsteps = 1 + nrows * (nrows + 3) / 2;
        auto info = [&](int s, bool& inv_step, int& i, int& k) {
            inv_step = true;
            i = j;
            k = 0;
            int rest = s - 1;
            for (int o = 1; s > 0; ++o) {
                const int ii = upper ? j - o : j + o;
                i = ii;
                if (rest < o) {
                    inv_step = false;
                    k = (upper ? ii + 1 : j) + rest;
                    return;
                }
                if (rest == o) return;
                rest -= o + 1;
            }
        };
        auto issue = [&](int s) {
            bool inv_step;
            int i, k;
            info(s, inv_step, i, k);
            double(*Sb)[kStagePitch] = (s & 1) ? S1 : S0;
            if (inv_step)
                stage_block(Sb, iblock(i), 1, kNB, kNB, kNB, inv64);
            else
                stage_block(Sb, ablock(i, k), sr, sc, len - i * kNB, len - k * kNB, a);
            cp_async_commit();
        };
        const int lane = t & 31, warp = t >> 5, g = lane >> 2, tq = lane & 3, rt = warp >> 1, ct0 = (warp & 1) * 4;
        double acc[4][4] = {};
        issue(0);
        for (int s = 0; s < nsteps; ++s) {
            if (s + 1 < nsteps) {
                issue(s + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const double(*Sb)[kStagePitch] = (s & 1) ? S1 : S0;
            bool inv_step;
            int i, k;
            info(s, inv_step, i, k);
            if (s == 0) {  // X_jj = inv(A_jj)
                for (int q = t; q < kNB * kNB; q += 256) X[j][q % kNB][q / kNB] = staged(Sb, true, q % kNB, q / kNB);
                have[j] = true;
            } else if (!inv_step) {  // acc += A_ik X_kj; after the last k the sum goes to X[i]
                const int k0 = upper ? i + 1 : j, k1 = upper ? j : i - 1;
                if (k == k0) {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
                }
                mma_64(acc, Sb, sr == 1, X[k]);
                if (k == k1) {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            X[i][16 * rt + g + 8 * (v >> 1)][8 * (ct0 + u) + 2 * tq + (v & 1)] = acc[u][v];
                }
            } else {  // X_ij = -inv(A_ii) * sum
                double y[4][4] = {};
                mma_64(y, Sb, true, X[i]);
                __syncthreads();
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        X[i][16 * rt + g + 8 * (v >> 1)][8 * (ct0 + u) + 2 * tq + (v & 1)] = -y[u][v];
                have[i] = true;
            }
            __syncthreads();  // the buffer of step s is refilled by the issue of step s + 2
        }
    }
    // column block j of the leaf inverse: rows of computed blocks, zeros elsewhere
    for (int q = t; q < kLeaf * kNB; q += 256) {
        const int r = q % kLeaf, c = q / kLeaf, bi = r / kNB;
        out[r + (long)(j * kNB + c) * kLeaf] = (j < nsb && have[bi]) ? X[bi][r % kNB][c] : 0.0;
    }
}

// One leaf of the solve in place: Y = inv(M) Z, inv(M) = the leaf inverse
// (side L) or its transpose (side R), Z = B[p0.., c..] (side L) or
// B[c.., p0..]^T (side R).  A cluster of four CTAs takes 16 right-hand sides;
// CTA r of the cluster computes output rows 64 r .. 64 r + 63 over the nonzero
// K range of the triangular inverse.  Every CTA loads all of Z (the leaf's
// rows are read by all four) and the cluster barrier orders those reads
// before any CTA writes its rows back.  Warp w: row tile w / 2, column tile
// w % 2, two accumulators.
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(256)
trsm_leaf_apply(const double* __restrict__ inv_leaf, int left, int inv_t, int fwd, int p0, int len,
                double* __restrict__ b, long ldb, int ncols, int wait_first) {
    extern __shared__ __align__(16) unsigned char ap_smem[];
    double(*Z)[kLeafCols + 1] = reinterpret_cast<double(*)[kLeafCols + 1]>(ap_smem);
    double* A = reinterpret_cast<double*>(ap_smem + sizeof(double) * kLeaf * (kLeafCols + 1));
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, g = lane >> 2, tq = lane & 3;
    const int rb = (int)cluster_ctarank();
    const int c0 = (blockIdx.x / 4) * kLeafCols, nc = min(kLeafCols, ncols - c0);
    // nonzero K range of rows 64 rb .. of the (lower when fwd) inverse, within the leaf
    const int kbeg = fwd ? 0 : kNB * rb, kend = min(len, fwd ? kNB * (rb + 1) : kLeaf);
    const int klen = max(0, kend - kbeg);
    const int klen8 = (klen + 7) & ~7;
    // rows 64 rb + i, columns kbeg + kk of inv(M): stored as is (inv_t = 0) inv[i' + k' kLeaf] (runs
    // along i, staged [kk][i], pitch 66); stored transposed (inv_t = 1: side R, or an inverse of A
    // serving op(A) = A^T) inv[k' + i' kLeaf] (runs along kk, staged [i][kk], pitch kLeaf + 2)
    if (wait_first) grid_dependency_wait();  // the kernel before this one wrote the inverses
    if (64 * rb < len && klen > 0) {
        if (!inv_t) {
            for (int q = t; q < klen8 * (kNB / 2); q += 256) {
                const int kk = q / (kNB / 2), i = (q % (kNB / 2)) * 2;
                const bool ok = kk < klen;
                cp_async_16(smem_u32(A + kk * kStagePitch + i),
                            ok ? inv_leaf + (kNB * rb + i) + (long)(kbeg + kk) * kLeaf : inv_leaf, ok ? 16 : 0);
            }
        } else {
            for (int q = t; q < kNB * (klen8 / 2); q += 256) {
                const int i = q / (klen8 / 2), kk = (q % (klen8 / 2)) * 2;
                const bool ok = kk < klen;
                cp_async_16(smem_u32(A + i * (kLeaf + 2) + kk),
                            ok ? inv_leaf + (kbeg + kk) + (long)(kNB * rb + i) * kLeaf : inv_leaf, ok ? 16 : 0);
            }
        }
    }
    cp_async_commit();
    // The inverse is not written by the kernel before this one (a coupling
    // product or its reduction): its copies above may overlap that kernel's
    // tail; the rows of B it updates are read after it has finished.
    grid_dependency_wait();
    // all sixteen loads of a thread in flight before the first shared store (a
    // load-store loop waited out one L2 round trip per element)
    constexpr int kZIt = kLeaf * kLeafCols / 256;
    double zv[kZIt];
#pragma unroll
    for (int i = 0; i < kZIt; ++i) {
        const int idx = i * 256 + t;
        const int r = left ? idx % kLeaf : idx / kLeafCols, c = left ? idx / kLeaf : idx % kLeafCols;
        zv[i] = 0.0;
        if (r < len && c < nc)
            zv[i] = left ? b[(p0 + r) + (long)(c0 + c) * ldb] : b[(c0 + c) + (long)(p0 + r) * ldb];
    }
#pragma unroll
    for (int i = 0; i < kZIt; ++i) {
        const int idx = i * 256 + t;
        Z[left ? idx % kLeaf : idx / kLeafCols][left ? idx / kLeaf : idx % kLeafCols] = zv[i];
    }
    cluster_sync();  // every CTA of the cluster has read its Z from B
    cp_async_wait<0>();
    __syncthreads();
    if (64 * rb >= len) return;
    const int rt = warp >> 1, ct = warp & 1;
    double acc0[4] = {0.0, 0.0, 0.0, 0.0}, acc1[4] = {0.0, 0.0, 0.0, 0.0};
    for (int kb = 0; kb < klen8 / 8; ++kb) {
        double af[4], bf[2];
#pragma unroll
        for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
            for (int v0 = 0; v0 < 2; ++v0) {
                const int i = 16 * rt + g + 8 * v0, kk = 8 * kb + tq + 4 * v1;
                af[v0 + 2 * v1] = !inv_t ? A[kk * kStagePitch + i] : A[i * (kLeaf + 2) + kk];
            }
#pragma unroll
        for (int v = 0; v < 2; ++v) bf[v] = Z[kbeg + 8 * kb + tq + 4 * v][8 * ct + g];
        if (kb & 1)
            dmma_16x8x8(acc1, af, bf);
        else
            dmma_16x8x8(acc0, af, bf);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const int r = kNB * rb + 16 * rt + g + 8 * (v >> 1), cc = 8 * ct + 2 * tq + (v & 1);
        if (r < len && cc < nc) {
            const double y = acc0[v] + acc1[v];
            if (left)
                b[(p0 + r) + (long)(c0 + cc) * ldb] = y;
            else
                b[(c0 + cc) + (long)(p0 + r) * ldb] = y;
        }
    }
}

// B := alpha B on the m x n window (plain product, like the reference's
// scaleDenseColumns: NaN * 0 stays NaN).
template <typename T>
__global__ void scale_plain(int m, int n, T alpha, T* __restrict__ b, long ldb) {
    const long total = (long)m * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        T* p = b + (q % m) + (q / m) * ldb;
        *p = alpha * *p;
    }
}

// C := beta C on one triangle (beta == 0 writes zeros).
template <typename T>
__global__ void scale_triangle(int n, int tri, T beta, T* __restrict__ c, long ldc) {
    const long total = (long)n * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int i = (int)(q % n), j = (int)(q / n);
        if (tri == 1 ? i > j : i < j) continue;
        T* p = c + i + (long)j * ldc;
        *p = (beta == T(0)) ? T(0) : beta * *p;
    }
}

// Copy the stored triangle of an n x n matrix onto the other one.
template <typename T>
__global__ void symmetrize(int n, int from_upper, T* __restrict__ c, long ldc) {
    const long total = (long)n * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int i = (int)(q % n), j = (int)(q / n);
        if (from_upper ? (i > j) : (i < j)) c[i + (long)j * ldc] = c[j + (long)i * ldc];
    }
}

// Dense symmetric S (n x n, ld lds) from the uplo triangle of A; Hermitian
// when herm (mirrored elements conjugated, diagonal real: symValue,
// access.zig:31-42).  A 32 x 32 output tile takes its stored elements straight
// from A and its mirrored elements from a shared-memory transpose of the
// opposite tile, so global reads and writes are all coalesced.  Block (32, 8).
template <typename T>
__global__ void sym_expand(int n, int from_upper, int herm, const T* __restrict__ a, long lda, T* __restrict__ s,
                           long lds) {
    __shared__ T t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // does the tile hold any element of the unstored triangle?
    const bool mirror = from_upper ? (r0 + 31 > c0) : (r0 < c0 + 31);
    if (mirror) {  // t[y][x] = A(c0 + x, r0 + y)
        for (int y = ty; y < 32; y += 8) {
            const int ar = c0 + tx, ac = r0 + y;
            t[y][tx] = (ar < n && ac < n) ? a[ar + (long)ac * lda] : T(0);
        }
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
        const int i = r0 + tx, j = c0 + y;
        if (i >= n || j >= n) continue;
        const bool stored = from_upper ? i <= j : i >= j;
        T v = stored ? a[i + (long)j * lda] : conj_if(t[tx][y], herm != 0);
        s[i + (long)j * lds] = i == j ? herm_diag(v, herm != 0) : v;
    }
}

// Block (x, y): the dense diagonal block y of op(A), rows / columns y*nb ..
// (size s <= nb), column-major with ld nb; zeros outside the triangle and
// outside s x s, ones on a unit diagonal.
template <typename T>
__global__ void tri_dense_blocks(const T* __restrict__ a, long lda, char uplo, char trans, char diag, int n, int nb,
                                 T* __restrict__ out) {
    const int b0 = blockIdx.y * nb;
    const int s = min(nb, n - b0);
    T* o = out + (long)blockIdx.y * nb * nb;
    const long total = (long)nb * nb;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int r = (int)(q % nb), c = (int)(q / nb);
        o[q] = (r < s && c < s) ? op_tri(a, lda, uplo, trans, diag, b0 + r, b0 + c) : T(0);
    }
}

constexpr int kTrmmNB = 256;

// C := alpha (W + W^T) + beta C (two) or alpha W + beta C on the uplo
// triangle, W n x n with ld ldw, conj(W) in place of W when conj_w.  herm:
// C := alpha W + alpha2 W^H + beta C (two, Hermitian rank 2k) and the diagonal
// is made real.
// beta == 0 writes without reading C; alpha == 0 reads no W.  32 x 32 tiles,
// W^T through a shared-memory transpose; tiles outside the triangle return at
// once.  Block (32, 8).
template <typename T>
__global__ void tri_update(int n, int upper, int two, int conj_w, int herm, T alpha, T alpha2, const T* __restrict__ w,
                           long ldw, T beta, T* __restrict__ c, long ldc) {
    __shared__ T t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    if (upper ? r0 > c0 + 31 : r0 + 31 < c0) return;  // the whole block: no element of the triangle
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (two) {  // t[y][x] = W(c0 + x, r0 + y)
        for (int y = ty; y < 32; y += 8) {
            const int wr = c0 + tx, wc = r0 + y;
            t[y][tx] = (wr < n && wc < n) ? w[wr + (long)wc * ldw] : T(0);
        }
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
        const int i = r0 + tx, j = c0 + y;
        if (i >= n || j >= n || (upper ? i > j : i < j)) continue;
        T out = T(0);
        if (alpha != T(0)) {  // alpha = 0: W is not read (a scale-only call passes w = c)
            const T v = conj_if(w[i + (long)j * ldw], conj_w != 0);
            if (!two) {
                out = alpha * v;
            } else {
                const T u = conj_if(t[tx][y], conj_w != 0);  // W(j, i)
                // symmetric rank 2k: alpha (W + W^T); Hermitian: alpha W + alpha2 W^H
                out = herm ? alpha * v + alpha2 * conj_if(u, true) : alpha * (v + u);
            }
        }
        T* cp = c + i + (long)j * ldc;
        out = beta == T(0) ? out : fma(beta, *cp, out);
        *cp = i == j ? herm_diag(out, herm != 0) : out;
    }
}

}  // namespace

template <typename T>
cudaError_t triangle_update_h(char uplo, bool two, bool herm, int n, T alpha, T alpha2, const T* w, long ldw, T beta,
                              T* c, long ldc, cudaStream_t st, bool conj_w) {
    if (n <= 0) return cudaSuccess;
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    tri_update<T><<<grid, dim3(32, 8), 0, st>>>(n, uplo == 'U' ? 1 : 0, two ? 1 : 0, conj_w ? 1 : 0, herm ? 1 : 0,
                                                alpha, alpha2, w, ldw, beta, c, ldc);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t triangle_update(char uplo, bool two, int n, T alpha, const T* w, long ldw, T beta, T* c, long ldc,
                            cudaStream_t st, bool conj_w) {
    return triangle_update_h<T>(uplo, two, false, n, alpha, alpha, w, ldw, beta, c, ldc, st, conj_w);
}
template cudaError_t triangle_update<double>(char, bool, int, double, const double*, long, double, double*, long,
                                             cudaStream_t, bool);
template cudaError_t triangle_update<float>(char, bool, int, float, const float*, long, float, float*, long,
                                            cudaStream_t, bool);
template cudaError_t triangle_update<cnum<double>>(char, bool, int, cnum<double>, const cnum<double>*, long,
                                                   cnum<double>, cnum<double>*, long, cudaStream_t, bool);
template cudaError_t triangle_update<cnum<float>>(char, bool, int, cnum<float>, const cnum<float>*, long, cnum<float>,
                                                  cnum<float>*, long, cudaStream_t, bool);
template cudaError_t triangle_update_h<cnum<double>>(char, bool, bool, int, cnum<double>, cnum<double>,
                                                     const cnum<double>*, long, cnum<double>, cnum<double>*, long,
                                                     cudaStream_t, bool);
template cudaError_t triangle_update_h<cnum<float>>(char, bool, bool, int, cnum<float>, cnum<float>,
                                                    const cnum<float>*, long, cnum<float>, cnum<float>*, long,
                                                    cudaStream_t, bool);

template <typename T>
size_t symm_plane_bytes(char side, int m, int n) {
    const long na = (side == 'L') ? m : n;
    return ((size_t)(na * na) * sizeof(T) + 1023) & ~size_t(1023);
}

template <typename T>
cudaError_t symm(char side, char uplo, int m, int n, T alpha, const T* a, long lda, const T* b, long ldb, T beta,
                 T* c, long ldc, void* planes, const GemmFn<T>& gemm, cudaStream_t st, bool herm) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    const int na = (side == 'L') ? m : n;
    T* S = static_cast<T*>(planes);
    dim3 grid((na + 31) / 32, (na + 31) / 32);
    sym_expand<T><<<grid, dim3(32, 8), 0, st>>>(na, uplo == 'U' ? 1 : 0, herm ? 1 : 0, a, lda, S, na);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (side == 'L') return gemm({'N', 'N', m, n, m, alpha, S, na, b, ldb, beta, c, ldc});
    return gemm({'N', 'N', m, n, n, alpha, b, ldb, S, na, beta, c, ldc});
}

template <typename T>
size_t trmm_plane_bytes(char side, int m, int n) {
    const long na = (side == 'L') ? m : n;
    const long nblk = (na + kTrmmNB - 1) / kTrmmNB;
    const size_t d = ((size_t)(nblk * kTrmmNB * kTrmmNB) * sizeof(T) + 1023) & ~size_t(1023);
    return d + (((size_t)m * n * sizeof(T) + 1023) & ~size_t(1023));
}

template <typename T>
cudaError_t trmm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st) {
    const int m = t.m, n = t.n;
    if (m <= 0 || n <= 0) return cudaSuccess;
    const bool left = t.side == 'L';
    const int na = left ? m : n;
    const int nblk = (na + kTrmmNB - 1) / kTrmmNB;
    T* D = static_cast<T*>(planes);
    T* W = reinterpret_cast<T*>(static_cast<char*>(planes) +
                                (((size_t)nblk * kTrmmNB * kTrmmNB * sizeof(T) + 1023) & ~size_t(1023)));
    cudaError_t e = cudaMemcpy2DAsync(W, (size_t)m * sizeof(T), t.b, (size_t)t.ldb * sizeof(T), (size_t)m * sizeof(T),
                                      n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    tri_dense_blocks<T><<<dim3(64, nblk), 256, 0, st>>>(t.a, t.lda, t.uplo, t.trans, t.diag, na, kTrmmNB, D);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const long ldb = t.ldb, lda = t.lda;
    // diagonal blocks: B_J := alpha D_J W_J (left) or alpha W_J D_J (right)
    for (int J = 0; J < nblk; ++J) {
        const int p0 = J * kTrmmNB, len = std::min(kTrmmNB, na - p0);
        const T* dj = D + (long)J * kTrmmNB * kTrmmNB;
        if (left)
            e = gemm({'N', 'N', len, n, len, t.alpha, dj, kTrmmNB, W + p0, m, T(0), t.b + p0, ldb});
        else
            e = gemm({'N', 'N', m, len, len, t.alpha, W + (long)p0 * m, m, dj, kTrmmNB, T(0), t.b + (long)p0 * ldb,
                      ldb});
        if (e != cudaSuccess) return e;
    }
    const bool upper = op_is_upper(t.uplo, t.trans);
    // op = C keeps its conjugation in the couplings of a complex A
    const char ta = (t.trans == 'N') ? 'N' : (is_cnum<T>::value ? t.trans : 'T');
    auto opa = [&](int r0, int c0) -> const T* {
        return (ta == 'N') ? t.a + r0 + (long)c0 * lda : t.a + c0 + (long)r0 * lda;
    };
    // off-diagonal blocks of op(A), halved on block boundaries: B += alpha op(A)_off W
    std::function<cudaError_t(int, int)> add_off = [&](int p0, int p1) -> cudaError_t {
        const int len = p1 - p0;
        if (len <= kTrmmNB) return cudaSuccess;
        const int mid = p0 + ((len / 2 + kTrmmNB - 1) / kTrmmNB) * kTrmmNB;
        const int h1 = mid - p0, h2 = p1 - mid;
        cudaError_t err;
        if (left) {
            if (!upper)  // rows mid..p1 gain op(A)[mid:p1, p0:mid] W[p0:mid]
                err = gemm({ta, 'N', h2, n, h1, t.alpha, opa(mid, p0), lda, W + p0, m, T(1), t.b + mid, ldb});
            else  // rows p0..mid gain op(A)[p0:mid, mid:p1] W[mid:p1]
                err = gemm({ta, 'N', h1, n, h2, t.alpha, opa(p0, mid), lda, W + mid, m, T(1), t.b + p0, ldb});
        } else {
            if (upper)  // columns mid..p1 gain W[:, p0:mid] op(A)[p0:mid, mid:p1]
                err = gemm({'N', ta, m, h2, h1, t.alpha, W + (long)p0 * m, m, opa(p0, mid), lda, T(1),
                            t.b + (long)mid * ldb, ldb});
            else  // columns p0..mid gain W[:, mid:p1] op(A)[mid:p1, p0:mid]
                err = gemm({'N', ta, m, h1, h2, t.alpha, W + (long)mid * m, m, opa(mid, p0), lda, T(1),
                            t.b + (long)p0 * ldb, ldb});
        }
        if (err != cudaSuccess) return err;
        if ((err = add_off(p0, mid)) != cudaSuccess) return err;
        return add_off(mid, p1);
    };
    if ((e = add_off(0, na)) != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T>
cudaError_t symmetrize_matrix(char uplo, int n, T* c, long ldc, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    symmetrize<T><<<grid_for((long)n * n), 256, 0, st>>>(n, uplo == 'U' ? 1 : 0, c, ldc);
    count_launch();
    return cudaGetLastError();
}
template cudaError_t symmetrize_matrix<double>(char, int, double*, long, cudaStream_t);
template cudaError_t symmetrize_matrix<float>(char, int, float*, long, cudaStream_t);

// inverted 64-blocks, then (FP64) the kLeaf-block inverses
template <typename T>
size_t inv_plane_bytes(int na) {
    const long nblk = (na + kNB - 1) / kNB;
    return ((size_t)(nblk * kNB * kNB) * sizeof(T) + 1023) & ~size_t(1023);
}

// Wider right-hand-side sets apply each leaf inverse as a GEMM from a copy of
// the leaf's rows (columns for side R) instead of the cluster kernel.
constexpr int kApplyMaxCols = 1024;

template <typename T>
size_t leaf_plane_bytes(int na) {
    const long nleaf = (na + kLeaf - 1) / kLeaf;
    return std::is_same<T, double>::value ? (((size_t)nleaf * kLeaf * kLeaf * sizeof(T) + 1023) & ~size_t(1023)) : 0;
}

template <typename T>
size_t trsm_plane_bytes(char side, int m, int n) {
    const int na = (side == 'L') ? m : n, ncols = (side == 'L') ? n : m;
    const size_t copy = (std::is_same<T, double>::value && ncols > kApplyMaxCols) ? (size_t)kLeaf * ncols * sizeof(T) : 0;
    return inv_plane_bytes<T>(na) + leaf_plane_bytes<T>(na) + copy;
}

template <typename T>
cudaError_t trsm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st,
                 const TrsmInverses* given) {
    const int m = t.m, n = t.n;
    if (m <= 0 || n <= 0) return cudaSuccess;
    cudaError_t e;
    if (t.alpha != T(1)) {
        scale_plain<T><<<grid_for((long)m * n), 256, 0, st>>>(m, n, t.alpha, t.b, t.ldb);
        count_launch();
    }
    const bool left = t.side == 'L';
    const int na = left ? m : n;
    const int nblk = (na + kNB - 1) / kNB;
    T* inv = static_cast<T*>(planes);
    // inverses of the diagonal blocks given by the caller (FP64): none are formed here
    const bool have_given = given != nullptr && std::is_same<T, double>::value;
    const bool given_t = have_given && given->transposed;
    if (!have_given) {
        const int tri_smem = (2 * kNB * (kNB + 1) + kNB) * (int)sizeof(T);
        if ((e = ensure_dynamic_smem(tri_inv_blocks<T>, tri_smem)) != cudaSuccess) return e;
        if ((e = launch_dependent(tri_inv_blocks<T>, dim3(nblk), dim3(256), (size_t)tri_smem, st, t.a, t.lda, t.uplo,
                                  t.trans, t.diag, na, inv)) != cudaSuccess)
            return e;
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    const bool upper = op_is_upper(t.uplo, t.trans);
    // the GEMM operand op(A): complex keeps C (conjugate transpose), real reads C as T
    const char ta = (t.trans == 'N') ? 'N' : (is_cnum<T>::value ? t.trans : 'T');
    const long lda = t.lda, ldb = t.ldb;
    // op(A)[r0:r1, c0:c1] as a GEMM operand (pointer, transpose flag)
    auto opa = [&](int r0, int c0) -> const T* {
        return (ta == 'N') ? t.a + r0 + (long)c0 * lda : t.a + c0 + (long)r0 * lda;
    };
    // Recursive halving on kLeaf-aligned boundaries: the two halves are solved
    // recursively and coupled by one GEMM whose K is half the range, so most of
    // the work runs as large GEMMs; each leaf of up to kLeaf rows is one launch
    // over the right-hand sides, in place.  FP64 with a 16-byte aligned A and an
    // even lda (16-byte operand copies) applies precomputed leaf inverses on
    // the tensor pipe; otherwise trsm_leaf solves phase by phase.
    const bool inv_leaves = have_given || (std::is_same<T, double>::value &&
                                           reinterpret_cast<uintptr_t>(t.a) % 16 == 0 && t.lda % 2 == 0);
    const int ncols = left ? n : m;
    const int fwd = left ? !upper : upper;
    // the leaf's M is op(A)'s block (side L) or its transpose (side R); inverses of
    // op(A) are stored as is, given inverses of A serving op(A) = A^T transposed
    const int inv_t = left ? (int)given_t : (int)!given_t;
    int leaf_smem;
    const double* inv_leaf = nullptr;
    if (inv_leaves && have_given) {
        inv_leaf = given->leaf;
        constexpr int kRows = kLeaf * kStagePitch > kNB * (kLeaf + 2) ? kLeaf * kStagePitch : kNB * (kLeaf + 2);
        leaf_smem = (int)sizeof(double) * (kLeaf * (kLeafCols + 1) + kRows);
        e = ensure_dynamic_smem(trsm_leaf_apply, leaf_smem);
    } else if (inv_leaves) {
        const int nleaf = (na + kLeaf - 1) / kLeaf;
        double* built = reinterpret_cast<double*>(static_cast<char*>(planes) + inv_plane_bytes<T>(na));
        inv_leaf = built;
        const int til_smem = (int)sizeof(double) * (4 * kNB * (kNB + 1) + 2 * kNB * kStagePitch);
        if ((e = ensure_dynamic_smem(tri_inv_leaf, til_smem)) != cudaSuccess) return e;
        if ((e = launch_dependent(tri_inv_leaf, dim3(nleaf, kLeaf / kNB), dim3(256), (size_t)til_smem, st,
                                  reinterpret_cast<const double*>(t.a), lda, (int)(ta == 'N'), (int)upper, na,
                                  reinterpret_cast<const double*>(inv), built)) != cudaSuccess)
            return e;
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        // Z plus 64 rows of the inverse over up to kLeaf columns (either staging layout)
        constexpr int kRows = kLeaf * kStagePitch > kNB * (kLeaf + 2) ? kLeaf * kStagePitch : kNB * (kLeaf + 2);
        leaf_smem = (int)sizeof(double) * (kLeaf * (kLeafCols + 1) + kRows);
        e = ensure_dynamic_smem(trsm_leaf_apply, leaf_smem);
    } else {
        leaf_smem = (int)sizeof(T) * (kLeaf * (kLeafCols + 1) + kNB * (kNB + 1));
        e = ensure_dynamic_smem(trsm_leaf<T>, leaf_smem);
    }
    if (e != cudaSuccess) return e;
    bool first_leaf = true;
    std::function<cudaError_t(int, int)> solve = [&](int p0, int p1) -> cudaError_t {
        cudaError_t err = cudaSuccess;
        const int len = p1 - p0;
        if (len <= kLeaf) {
            const int grid = (ncols + kLeafCols - 1) / kLeafCols;
            if (inv_leaves && ncols > kApplyMaxCols) {  // copy of the leaf's rows / columns, then one GEMM
                const T* il = reinterpret_cast<const T*>(inv_leaf + (long)(p0 / kLeaf) * kLeaf * kLeaf);
                const char il_t = given_t ? 'T' : 'N';  // the leaf inverse of op(A) is the given one transposed
                T* W = reinterpret_cast<T*>(static_cast<char*>(planes) + inv_plane_bytes<T>(na) +
                                            leaf_plane_bytes<T>(na));
                if (left) {
                    if ((err = cudaMemcpy2DAsync(W, (size_t)len * sizeof(T), t.b + p0, ldb * sizeof(T),
                                                 (size_t)len * sizeof(T), n, cudaMemcpyDeviceToDevice, st)) !=
                        cudaSuccess)
                        return err;
                    return gemm({il_t, 'N', len, n, len, T(1), il, kLeaf, W, len, T(0), t.b + p0, ldb});
                }
                if ((err = cudaMemcpy2DAsync(W, (size_t)m * sizeof(T), t.b + (long)p0 * ldb, ldb * sizeof(T),
                                             (size_t)m * sizeof(T), len, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
                    return err;
                return gemm({'N', il_t, m, len, len, T(1), W, m, il, kLeaf, T(0), t.b + (long)p0 * ldb, ldb});
            }
            if (inv_leaves) {  // clusters of four CTAs per 16 right-hand sides
                const double* il = inv_leaf + (long)(p0 / kLeaf) * kLeaf * kLeaf;
                double* bd = reinterpret_cast<double*>(t.b);
                // every leaf after the first follows a coupling product (or its reduction),
                // which does not write the inverses: it stages them during that kernel's
                // tail; the first follows tri_inv_leaf and waits before staging
                err = launch_dependent(trsm_leaf_apply, dim3(4 * grid), dim3(256), (size_t)leaf_smem, st, il, left, inv_t,
                                       fwd, p0, len, bd, ldb, ncols, (int)first_leaf);
                first_leaf = false;
                count_launch();
                if (err != cudaSuccess) return err;
                return cudaGetLastError();
            } else
                trsm_leaf<T><<<grid, 256, leaf_smem, st>>>(t.a, lda, ta == 'N', is_cnum<T>::value && t.trans == 'C',
                                                           left, fwd, inv, p0, len, t.b, ldb, ncols);
            count_launch();
            return cudaGetLastError();
        }
        const int mid = p0 + ((len / 2 + kLeaf - 1) / kLeaf) * kLeaf;
        const int h1 = mid - p0, h2 = p1 - mid;
        if (left) {
            if (!upper) {  // rows p0..mid first, then update mid..p1
                if ((err = solve(p0, mid)) != cudaSuccess) return err;
                if ((err = gemm({ta, 'N', h2, n, h1, T(-1), opa(mid, p0), lda, t.b + p0, ldb, T(1), t.b + mid,
                                 ldb})) != cudaSuccess)
                    return err;
                return solve(mid, p1);
            }
            if ((err = solve(mid, p1)) != cudaSuccess) return err;
            if ((err = gemm({ta, 'N', h1, n, h2, T(-1), opa(p0, mid), lda, t.b + mid, ldb, T(1), t.b + p0, ldb})) !=
                cudaSuccess)
                return err;
            return solve(p0, mid);
        }
        // right side: X op(A) = B over column ranges
        if (upper) {
            if ((err = solve(p0, mid)) != cudaSuccess) return err;
            if ((err = gemm({'N', ta, m, h2, h1, T(-1), t.b + (long)p0 * ldb, ldb, opa(p0, mid), lda, T(1),
                             t.b + (long)mid * ldb, ldb})) != cudaSuccess)
                return err;
            return solve(mid, p1);
        }
        if ((err = solve(mid, p1)) != cudaSuccess) return err;
        if ((err = gemm({'N', ta, m, h1, h2, T(-1), t.b + (long)mid * ldb, ldb, opa(mid, p0), lda, T(1),
                         t.b + (long)p0 * ldb, ldb})) != cudaSuccess)
            return err;
        return solve(p0, mid);
    };
    if ((e = solve(0, na)) != cudaSuccess) return e;
    return cudaGetLastError();
}

size_t trsm_leaf_inverse_bytes(int n) { return n > 0 ? leaf_plane_bytes<double>(n) : 0; }
size_t trsm_leaf_inverse_scratch_bytes(int n) { return n > 0 ? inv_plane_bytes<double>(n) : 0; }

cudaError_t trsm_leaf_inverses(char uplo, char diag, int n, const double* a, long lda, void* scratch, double* leaf,
                               cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (reinterpret_cast<uintptr_t>(a) % 16 != 0 || lda % 2 != 0) return cudaErrorInvalidValue;
    cudaError_t e;
    double* inv = static_cast<double*>(scratch);
    const int nblk = (n + kNB - 1) / kNB, nleaf = (n + kLeaf - 1) / kLeaf;
    const int tri_smem = (2 * kNB * (kNB + 1) + kNB) * (int)sizeof(double);
    if ((e = ensure_dynamic_smem(tri_inv_blocks<double>, tri_smem)) != cudaSuccess) return e;
    if ((e = launch_dependent(tri_inv_blocks<double>, dim3(nblk), dim3(256), (size_t)tri_smem, st, a, lda, uplo, 'N',
                              diag, n, inv)) != cudaSuccess)
        return e;
    count_launch();
    const int til_smem = (int)sizeof(double) * (4 * kNB * (kNB + 1) + 2 * kNB * kStagePitch);
    if ((e = ensure_dynamic_smem(tri_inv_leaf, til_smem)) != cudaSuccess) return e;
    if ((e = launch_dependent(tri_inv_leaf, dim3(nleaf, kLeaf / kNB), dim3(256), (size_t)til_smem, st, a, lda, 1,
                              (int)(uplo == 'U'), n, (const double*)inv, leaf)) != cudaSuccess)
        return e;
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t syrk_scale_only(int n, char uplo, T beta, T* c, long ldc, cudaStream_t st) {
    scale_triangle<T><<<grid_for((long)n * n), 256, 0, st>>>(n, uplo == 'U' ? 1 : 2, beta, c, ldc);
    count_launch();
    return cudaGetLastError();
}

template size_t trsm_plane_bytes<double>(char, int, int);
template size_t trsm_plane_bytes<float>(char, int, int);
template cudaError_t trsm<double>(const TrsmArgs<double>&, void*, const GemmFn<double>&, cudaStream_t,
                                  const TrsmInverses*);
template cudaError_t trsm<float>(const TrsmArgs<float>&, void*, const GemmFn<float>&, cudaStream_t,
                                 const TrsmInverses*);
template size_t trsm_plane_bytes<cnum<double>>(char, int, int);
template size_t trsm_plane_bytes<cnum<float>>(char, int, int);
template cudaError_t trsm<cnum<double>>(const TrsmArgs<cnum<double>>&, void*, const GemmFn<cnum<double>>&,
                                        cudaStream_t, const TrsmInverses*);
template cudaError_t trsm<cnum<float>>(const TrsmArgs<cnum<float>>&, void*, const GemmFn<cnum<float>>&,
                                       cudaStream_t, const TrsmInverses*);
template cudaError_t syrk_scale_only<cnum<double>>(int, char, cnum<double>, cnum<double>*, long, cudaStream_t);
template cudaError_t syrk_scale_only<cnum<float>>(int, char, cnum<float>, cnum<float>*, long, cudaStream_t);
template cudaError_t syrk_scale_only<double>(int, char, double, double*, long, cudaStream_t);
template cudaError_t syrk_scale_only<float>(int, char, float, float*, long, cudaStream_t);
template size_t symm_plane_bytes<double>(char, int, int);
template size_t symm_plane_bytes<float>(char, int, int);
template cudaError_t symm<double>(char, char, int, int, double, const double*, long, const double*, long, double,
                                  double*, long, void*, const GemmFn<double>&, cudaStream_t, bool);
template cudaError_t symm<float>(char, char, int, int, float, const float*, long, const float*, long, float, float*,
                                 long, void*, const GemmFn<float>&, cudaStream_t, bool);
template size_t trmm_plane_bytes<double>(char, int, int);
template size_t trmm_plane_bytes<float>(char, int, int);
template cudaError_t trmm<double>(const TrsmArgs<double>&, void*, const GemmFn<double>&, cudaStream_t);
template cudaError_t trmm<float>(const TrsmArgs<float>&, void*, const GemmFn<float>&, cudaStream_t);
template size_t symm_plane_bytes<cnum<double>>(char, int, int);
template size_t symm_plane_bytes<cnum<float>>(char, int, int);
template cudaError_t symm<cnum<double>>(char, char, int, int, cnum<double>, const cnum<double>*, long,
                                        const cnum<double>*, long, cnum<double>, cnum<double>*, long, void*,
                                        const GemmFn<cnum<double>>&, cudaStream_t, bool);
template cudaError_t symm<cnum<float>>(char, char, int, int, cnum<float>, const cnum<float>*, long, const cnum<float>*,
                                       long, cnum<float>, cnum<float>*, long, void*, const GemmFn<cnum<float>>&,
                                       cudaStream_t, bool);
template size_t trmm_plane_bytes<cnum<double>>(char, int, int);
template size_t trmm_plane_bytes<cnum<float>>(char, int, int);
template cudaError_t trmm<cnum<double>>(const TrsmArgs<cnum<double>>&, void*, const GemmFn<cnum<double>>&,
                                        cudaStream_t);
template cudaError_t trmm<cnum<float>>(const TrsmArgs<cnum<float>>&, void*, const GemmFn<cnum<float>>&,
                                       cudaStream_t);

}  // namespace zb
