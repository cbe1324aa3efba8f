// TRSM, SYRK, SYMM, TRMM and SYR2K built on the GEMM tiles.
#pragma once

#include <algorithm>
#include <cstddef>
#include <functional>

#include <cuda_runtime.h>

#include "kernels.h"
#include "cnum.cuh"

namespace zb {

template <typename T>
struct TrsmArgs {
    char side, uplo, trans, diag;  // upper-case, validated
    int m, n;
    T alpha;
    const T* a;
    long lda;
    T* b;
    long ldb;
};

// One real GEMM on device pointers (the caller's method and scratch).
template <typename T>
using GemmFn = std::function<cudaError_t(const GemmArgs<T>&)>;

// Device scratch TRSM needs besides its GEMMs' own scratch.
template <typename T>
size_t trsm_plane_bytes(char side, int m, int n);

// Inverses of the 256-row diagonal blocks of an FP64 triangular A (op = N),
// computed once for several solves with the same A (trsm_leaf_inverses); a
// solve with op(A) = A^T reads them transposed.
struct TrsmInverses {
    const double* leaf;  // leaf b at leaf + b 256^2, column-major, ld 256, zero outside the triangle
    bool transposed;     // the solve's op(A) is A^T
};

// given: precomputed inverses (FP64 only); the diagonal blocks are then not inverted again.
template <typename T>
cudaError_t trsm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st,
                 const TrsmInverses* given = nullptr);

// Bytes of the inverses of an n x n triangular matrix's 256-row diagonal blocks,
// and the scratch (the 64-block inverses) forming them takes.
size_t trsm_leaf_inverse_bytes(int n);
size_t trsm_leaf_inverse_scratch_bytes(int n);
// leaf := the inverses of the 256-row diagonal blocks of A (uplo, diag; op = N)
// for trsm's `given`; A 16-byte aligned with an even lda.
cudaError_t trsm_leaf_inverses(char uplo, char diag, int n, const double* a, long lda, void* scratch, double* leaf,
                               cudaStream_t st);

// Device scratch SYMM needs besides its GEMM's scratch: the dense symmetric copy of A.
template <typename T>
size_t symm_plane_bytes(char side, int m, int n);

// C := alpha A B + beta C (side L) or alpha B A + beta C (side R), A symmetric
// (Hermitian when herm: conjugate mirror, real diagonal) with its uplo triangle
// stored; arguments validated, device pointers.
template <typename T>
cudaError_t symm(char side, char uplo, int m, int n, T alpha, const T* a, long lda, const T* b, long ldb, T beta,
                 T* c, long ldc, void* planes, const GemmFn<T>& gemm, cudaStream_t st, bool herm = false);

// Device scratch TRMM needs besides its GEMMs' scratch: dense diagonal blocks and a copy of B.
template <typename T>
size_t trmm_plane_bytes(char side, int m, int n);

// B := alpha op(A) B (side L) or alpha B op(A) (side R), A triangular (TrsmArgs fields).
template <typename T>
cudaError_t trmm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st);

// C := alpha (W + W^T) + beta C (two) or alpha W + beta C on the uplo triangle
// of the n x n C (SYRK / SYR2K from a full product W, conj(W) in place of W
// when conj_w; beta == 0 writes zeros over NaN).
template <typename T>
cudaError_t triangle_update(char uplo, bool two, int n, T alpha, const T* w, long ldw, T beta, T* c, long ldc,
                            cudaStream_t st, bool conj_w = false);

// The general form: with herm, C := alpha W + alpha2 W^H + beta C (two, HER2K)
// or alpha W + beta C (HERK) with the diagonal made real; without, as
// triangle_update (alpha2 unused).  alpha == 0 reads no W.
template <typename T>
cudaError_t triangle_update_h(char uplo, bool two, bool herm, int n, T alpha, T alpha2, const T* w, long ldw, T beta,
                              T* c, long ldc, cudaStream_t st, bool conj_w = false);

// Copy the uplo triangle of the n x n matrix c onto the other triangle.
template <typename T>
cudaError_t symmetrize_matrix(char uplo, int n, T* c, long ldc, cudaStream_t st);

// SYRK with k == 0: C := beta C on the triangle.
template <typename T>
cudaError_t syrk_scale_only(int n, char uplo, T beta, T* c, long ldc, cudaStream_t st);

}  // namespace zb
