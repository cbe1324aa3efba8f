// TRSM and SYRK on the GEMM tiles.
//
// TRSM  B := alpha * op(A)^-1 * B  (side L)  or  B * op(A)^-1  (side R)
//   Reference: core/matrix_matrix/triangular.zig:233 trsm (alpha pre-scale
//   :51-58, one trsv per right-hand side :103-117, right side row solves :72)
//   and the blocked template structured_blocked.zig:315 tryTrsm (GEMM trailing
//   updates with alpha = -1, beta = 1 at :344/:365).
//   GPU algorithm: all 64 x 64 diagonal blocks of op(A) are inverted in one
//   launch (tri_inv_blocks, exact substitution per column in shared memory);
//   then, block by block in solve order, X_J = inv(A_JJ) B_J and the trailing
//   update B_rest -= op(A)_rest,J X_J are GEMMs on the native (or Ozaki) tiles.
//
// SYRK  C := alpha * op(A) op(A)^T + beta * C on one triangle
//   Reference: core/matrix_matrix/symmetric.zig:237 syrk / runSyrkColumns :180
//   (one dot product per (i, j) of the triangle).  GPU algorithm: the GEMM
//   kernel in triangle mode: tiles outside the triangle are skipped and
//   elements outside it are never written.
#include "common.cuh"
#include "trsm_syrk.h"

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
    return a[ar + (long)ac * lda];
}

// Block b: inverse of the diagonal block op(A)[b*64 .. , b*64 ..] of size
// s <= 64, written column-major with ld 64 (zero outside s x s).  Thread j
// solves op(A)_bb x = e_j by substitution.
template <typename T>
__global__ void __launch_bounds__(kNB) tri_inv_blocks(const T* __restrict__ a, long lda, char uplo, char trans,
                                                      char diag, int n, T* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char tri_smem[];  // 2 x 64 x 65 elements
    T(*L)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(tri_smem);
    T(*X)[kNB + 1] = L + kNB;
    const int b0 = blockIdx.x * kNB;
    const int s = min(kNB, n - b0);
    const int j = threadIdx.x;
    for (int r = 0; r < kNB; ++r) {
        L[r][j] = (r < s && j < s) ? op_tri(a, lda, uplo, trans, diag, b0 + r, b0 + j) : T(0);
        X[r][j] = T(0);
    }
    __syncthreads();
    const bool upper = op_is_upper(uplo, trans);
    if (j < s) {
        if (!upper) {
            for (int r = j; r < s; ++r) {
                T v = (r == j) ? T(1) : T(0);
                for (int q = j; q < r; ++q) v -= L[r][q] * X[q][j];
                X[r][j] = (diag == 'U') ? v : v / L[r][r];
            }
        } else {
            for (int r = j; r >= 0; --r) {
                T v = (r == j) ? T(1) : T(0);
                for (int q = r + 1; q <= j; ++q) v -= L[r][q] * X[q][j];
                X[r][j] = (diag == 'U') ? v : v / L[r][r];
            }
        }
    }
    __syncthreads();
    T* o = out + (long)blockIdx.x * kNB * kNB;
    for (int r = 0; r < kNB; ++r) o[r + (long)j * kNB] = X[r][j];
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

}  // namespace

template <typename T>
size_t trsm_plane_bytes(char side, int m, int n) {
    const int na = (side == 'L') ? m : n;
    const long nblk = (na + kNB - 1) / kNB;
    const long w = (side == 'L') ? (long)kNB * n : (long)m * kNB;
    return ((size_t)(nblk * kNB * kNB + w) * sizeof(T) + 1023) & ~size_t(1023);
}

template <typename T>
cudaError_t trsm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st) {
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
    T* W = inv + (long)nblk * kNB * kNB;
    const int tri_smem = 2 * kNB * (kNB + 1) * (int)sizeof(T);
    if ((e = cudaFuncSetAttribute(tri_inv_blocks<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem)) !=
        cudaSuccess)
        return e;
    tri_inv_blocks<T><<<nblk, kNB, tri_smem, st>>>(t.a, t.lda, t.uplo, t.trans, t.diag, na, inv);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const bool upper = op_is_upper(t.uplo, t.trans);
    const char ta = (t.trans == 'N') ? 'N' : 'T';
    const long lda = t.lda, ldb = t.ldb;
    // Left: lower -> blocks top-down; upper -> bottom-up.
    // Right (X op(A) = B): upper -> column blocks left to right; lower -> right to left.
    const bool forward = left ? !upper : upper;
    for (int q = 0; q < nblk; ++q) {
        const int bi = forward ? q : nblk - 1 - q;
        const int kb = bi * kNB, s = std::min(kNB, na - kb);
        const T* invb = inv + (long)bi * kNB * kNB;
        if (left) {
            // X_J = inv_J * B[kb:kb+s, :]  (s x n) -> W, then back into B
            if ((e = gemm({'N', 'N', s, n, s, T(1), invb, kNB, t.b + kb, ldb, T(0), W, s})) != cudaSuccess) return e;
            if ((e = cudaMemcpy2DAsync(t.b + kb, ldb * sizeof(T), W, (size_t)s * sizeof(T), (size_t)s * sizeof(T), n,
                                       cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
                return e;
            if (!upper && kb + s < m) {
                const int r0 = kb + s;
                const T* asub = (ta == 'N') ? t.a + r0 + (long)kb * lda : t.a + kb + (long)r0 * lda;
                if ((e = gemm({ta, 'N', m - r0, n, s, T(-1), asub, lda, t.b + kb, ldb, T(1), t.b + r0, ldb})) !=
                    cudaSuccess)
                    return e;
            }
            if (upper && kb > 0) {
                const T* asub = (ta == 'N') ? t.a + (long)kb * lda : t.a + kb;
                if ((e = gemm({ta, 'N', kb, n, s, T(-1), asub, lda, t.b + kb, ldb, T(1), t.b, ldb})) != cudaSuccess)
                    return e;
            }
        } else {
            // X_J = B[:, kb:kb+s] * inv_J  (m x s) -> W, then back into B
            T* bj = t.b + (long)kb * ldb;
            if ((e = gemm({'N', 'N', m, s, s, T(1), bj, ldb, invb, kNB, T(0), W, m})) != cudaSuccess) return e;
            if ((e = cudaMemcpy2DAsync(bj, ldb * sizeof(T), W, (size_t)m * sizeof(T), (size_t)m * sizeof(T), s,
                                       cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
                return e;
            if (upper && kb + s < n) {
                const int c0 = kb + s;
                const T* asub = (ta == 'N') ? t.a + kb + (long)c0 * lda : t.a + c0 + (long)kb * lda;
                if ((e = gemm({'N', ta, m, n - c0, s, T(-1), bj, ldb, asub, lda, T(1), t.b + (long)c0 * ldb, ldb})) !=
                    cudaSuccess)
                    return e;
            }
            if (!upper && kb > 0) {
                const T* asub = (ta == 'N') ? t.a + kb : t.a + (long)kb * lda;
                if ((e = gemm({'N', ta, m, kb, s, T(-1), bj, ldb, asub, lda, T(1), t.b, ldb})) != cudaSuccess) return e;
            }
        }
    }
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
template cudaError_t trsm<double>(const TrsmArgs<double>&, void*, const GemmFn<double>&, cudaStream_t);
template cudaError_t trsm<float>(const TrsmArgs<float>&, void*, const GemmFn<float>&, cudaStream_t);
template cudaError_t syrk_scale_only<double>(int, char, double, double*, long, cudaStream_t);
template cudaError_t syrk_scale_only<float>(int, char, float, float*, long, cudaStream_t);

}  // namespace zb
