// Complex GEMM through real GEMMs (expanded-real 4M form and the 3M form).
#pragma once

#include <cstddef>
#include <functional>

#include <cuda_runtime.h>

#include "kernels.h"

namespace zb {

enum ComplexMethod : int { COMPLEX_4M = 0, COMPLEX_3M = 1 };

// Interleaved complex operands; alpha / beta are host (re, im) pairs.
template <typename T>
struct ComplexArgs {
    char transa, transb;  // 'N', 'T' or 'C'
    int m, n, k;
    T alpha[2];
    const T* a;
    long lda;
    const T* b;
    long ldb;
    T beta[2];
    T* c;
    long ldc;
    // m == n only: 0 = all of C; 1 = only the upper triangle (row <= col), 2 =
    // only the lower one (row >= col) is computed and written (rank-k updates)
    int tri = 0;
};

// C (m x n, ldc) = A (m x k, lda) * B (k x n, ldb), real, alpha = 1, beta = 0;
// tri as in GemmArgs (tiles outside the triangle are skipped, C there is left alone).
template <typename T>
using RealGemm = std::function<cudaError_t(int m, int n, int k, const T* a, long lda, const T* b, long ldb, T* c,
                                           long ldc, int tri)>;

// Device scratch the complex route needs for its planes (the real GEMMs'
// own scratch comes on top of it).
template <typename T>
size_t complex_plane_bytes(int method, int m, int n, int k);

// Arguments validated, m, n > 0, k > 0, alpha != 0.
template <typename T>
cudaError_t complex_gemm(const ComplexArgs<T>& g, int method, void* planes, const RealGemm<T>& real_gemm,
                         cudaStream_t st);

}  // namespace zb
