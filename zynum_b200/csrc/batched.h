// Variable-size batched GEMM / TRSM: persistent kernels, plans and autotuner.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "kernels.h"

namespace zb {

enum BatchDtype : int { BATCH_F64 = 0, BATCH_F32 = 1 };
enum TileCfg : int { TILE_CFG_32 = 0, TILE_CFG_64 = 1, TILE_CFG_128 = 2 };

// One output tile of one problem (prob < 0: padding, skipped).
struct BatchWork {
    int prob, m0, n0, cfg;
};

// Device side of a GEMM batch plan.
struct BatchDevice {
    const BatchWork* work;
    int n_work;
    const int* dims;  // m, n, k per problem
};

int batched_tile_edge(int cfg);

// a, b, c, lda, ldb, ldc: DEVICE arrays with one entry per problem.
cudaError_t launch_gemm_batched(const BatchDevice& d, int dtype, char transa, char transb, const void* alpha,
                                const void* const* a, const int* lda, const void* const* b, const int* ldb,
                                const void* beta, void* const* c, const int* ldc, int grid, cudaStream_t st);

// order: per-CTA interleaved problem order (-1 = padding); dims: n, nrhs per problem.
cudaError_t launch_trsm_batched(const int* order, int count, const int* dims, int dtype, char uplo, char trans,
                                char diag, const void* alpha, const void* const* a, const int* lda, void* const* b,
                                const int* ldb, int grid, cudaStream_t st);

}  // namespace zb
