// TRSM and SYRK built on the GEMM tiles.
#pragma once

#include <algorithm>
#include <cstddef>
#include <functional>

#include <cuda_runtime.h>

#include "kernels.h"

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

template <typename T>
cudaError_t trsm(const TrsmArgs<T>& t, void* planes, const GemmFn<T>& gemm, cudaStream_t st);

// Copy the uplo triangle of the n x n matrix c onto the other triangle.
template <typename T>
cudaError_t symmetrize_matrix(char uplo, int n, T* c, long ldc, cudaStream_t st);

// SYRK with k == 0: C := beta C on the triangle.
template <typename T>
cudaError_t syrk_scale_only(int n, char uplo, T beta, T* c, long ldc, cudaStream_t st);

}  // namespace zb
