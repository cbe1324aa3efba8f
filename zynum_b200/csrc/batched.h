// Variable-size batched GEMM / TRSM: persistent kernels, plans and autotuner.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "kernels.h"

namespace zb {

enum BatchDtype : int { BATCH_F64 = 0, BATCH_F32 = 1 };
enum TileCfg : int { TILE_CFG_32 = 0, TILE_CFG_64 = 1, TILE_CFG_128 = 2 };

// A chunk of `count` consecutive output tiles t0.. of one problem.  Tile t covers rows (t % mt) TM.. and columns (t / mt) TN..
// with TM x TN = batched_tile_m x batched_tile_n and mt = ceil(m / TM).
struct BatchWork {
    int prob, t0, count, cfg;
};

// Device side of a GEMM batch plan.
struct BatchDevice {
    const BatchWork* work;  // longest first; CTAs claim items in this order
    int n_work;
    const int* dims;  // m, n, k per problem
    int* next;        // claim counter, zeroed by each launch
};

// Output tile of a config: rows x columns (square; TILE_CFG_128 is 128 x 128
// for FP32 and runs as 64 x 64 for FP64).
int batched_tile_m(int cfg, int dtype);
int batched_tile_n(int cfg, int dtype);

// a, b, c, lda, ldb, ldc: DEVICE arrays with one entry per problem.
cudaError_t launch_gemm_batched(const BatchDevice& d, int dtype, char transa, char transb, const void* alpha,
                                const void* const* a, const int* lda, const void* const* b, const int* ldb,
                                const void* beta, void* const* c, const int* ldc, int grid, cudaStream_t st);

// order: problems longest first (CTAs claim them through the counter `next`, zeroed
// by the launch); dims: n, nrhs per problem.
cudaError_t launch_trsm_batched(const int* order, int count, int* next, const int* dims, int dtype, char uplo,
                                char trans, char diag, const void* alpha, const void* const* a, const int* lda,
                                void* const* b, const int* ldb, int grid, cudaStream_t st);

}  // namespace zb
