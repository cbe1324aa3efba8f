// Internal interface between the C-ABI layer, the planner and the kernels.
// Nothing here is exported from the shared library; the public surface is
// include/zynum_blas_gpu.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace zb {

// Column-major GEMM operands, BLAS conventions: op(X) = X for 'N', X^T for
// 'T' (and for 'C' on real types).  Leading dimensions are in elements.
template <typename T>
struct GemmArgs {
    char transa, transb;
    int m, n, k;
    T alpha;
    const T* a;
    long lda;
    const T* b;
    long ldb;
    T beta;
    T* c;
    long ldc;
    // 0: full C; 1: only the upper triangle (row <= col); 2: only the lower
    // triangle (row >= col).  Tiles entirely outside are skipped (SYRK).
    int tri = 0;
};
using GemmArgsF64 = GemmArgs<double>;
using GemmArgsF32 = GemmArgs<float>;

// TILE_GEMV: n == 1 or m == 1, served by the matrix-vector kernels (splits =
// K splits of the GEMV partials, workspace splits * m * n elements as for split-K).
// TILE_NARROW_N / TILE_NARROW_M: n <= 16 / m <= 16 (the other side >= 512):
// FP64 128 x 16 / 16 x 128 DMMA tiles, FP32 the narrow FFMA kernel (HBM-bound;
// a 64- or 128-wide tile would be compute-bound on padding).
// TILE_64x64: FP64 products whose 128 x 128 tiles would leave most SMs idle.
enum TileShape : int {
    TILE_128x128 = 0,
    TILE_128x64 = 1,
    TILE_GEMV = 2,
    TILE_NARROW_N = 3,
    TILE_NARROW_M = 4,
    TILE_64x64 = 5
};

// What the planner decided for one native GEMM call.
struct GemmPlan {
    int tile = TILE_128x128;
    int splits = 1;  // > 1: split-K over `splits` K ranges, needs a workspace
};

// Workspace (in elements of T) a plan needs.
inline size_t splitk_workspace_elems(int m, int n, int splits) {
    return splits > 1 ? (size_t)splits * (size_t)m * (size_t)n : 0;
}

// ---------------------------------------------------------------- kernels
cudaError_t dgemm_native(const GemmArgsF64& g, const GemmPlan& plan, double* workspace, cudaStream_t st);
// TMA-fed, warp-specialised 128 x 128 DGEMM tiles (gemm_f64_tma.cu): for
// 16-byte aligned operands with even leading dimensions.  K is split into
// ranges of dgemm_tma_k_chunk(k, splits) (a multiple of the 32-deep slice);
// with more than one range the raw sums go to `workspace` (range z at
// z * m * n, ld m) and the caller reduces them.
bool dgemm_tma_applies(const GemmArgsF64& g);
int dgemm_tma_k_chunk(int k, int splits);
cudaError_t dgemm_tma(const GemmArgsF64& g, int splits, double* workspace, cudaStream_t st);
// K ranges dgemm_native will actually use for this plan (1: no workspace); the
// route (GEMV, tall-skinny, tiles) and the rounding of K slices can only lower
// it below plan.splits.
int dgemm_native_used_splits(const GemmArgsF64& g, const GemmPlan& plan);
cudaError_t sgemm_native(const GemmArgsF32& g, const GemmPlan& plan, float* workspace, cudaStream_t st);
// Workspace of sgemm_native in bytes: split-K partials plus, for large
// products, an MN-contiguous copy of each K-contiguous operand.  The bound
// covers every FP32 product of shape up to m x n x k and any transposes.
size_t sgemm_native_workspace_bytes(char transa, char transb, int m, int n, int k, const GemmPlan& plan);
// Tall-skinny route (n <= 64, k <= 64, m >= 2048, no triangle mode): op(B)
// staged once per persistent CTA, op(A) streamed in 128-row blocks.
bool skinny_gemm_applies(int m, int n, int k, int tri);
cudaError_t dgemm_skinny(const GemmArgsF64& g, cudaStream_t st);
// FP64 tall-skinny route on TMA-fed op(A) row blocks (gemm_skinny_tma.cu): for a
// 16-byte aligned op(A) with an even leading dimension.
bool dgemm_skinny_tma_applies(const GemmArgsF64& g);
cudaError_t dgemm_skinny_tma(const GemmArgsF64& g, cudaStream_t st);
// FP32 tall-skinny route on TMA-fed op(A) row blocks: 16-byte aligned op(A), lda a multiple of 4.
bool sgemm_skinny_tma_applies(const GemmArgsF32& g);
cudaError_t sgemm_skinny_tma(const GemmArgsF32& g, cudaStream_t st);
cudaError_t sgemm_skinny(const GemmArgsF32& g, cudaStream_t st);
size_t sgemm_native_workspace_bound(int m, int n, int k, int sm_count);
// Vector-edge route (n == 1 or m == 1, no triangle mode): HBM-bound
// matrix-vector kernels; `splits` > 1 needs splits * max(m, n) elements of workspace.
bool gemv_applies(int m, int n, int k, int tri);
constexpr long kGemvSplitTarget = 1L << 20;   // outputs x K splits the planner aims for
constexpr long kGemvMaxPartials = 2L << 20;   // bound on splits * outputs (workspace elements)
int gemv_split_count(int rows, int k);
// K splits the GEMV kernels use when asked for `splits` (K slices are rounded up).
int gemv_used_splits(int k, int splits);
cudaError_t dgemv_route(const GemmArgsF64& g, int splits, double* ws, cudaStream_t st);
cudaError_t sgemv_route(const GemmArgsF32& g, int splits, float* ws, cudaStream_t st);
// Narrow route (n <= 16 with m >= 512, or m <= 16 with n >= 512; n, m > 1):
// K split count for 128-output tiles, and the FP32 kernel (splits * m * n
// elements of workspace when splits > 1).
bool narrow_gemm_applies(int m, int n, int tri);
int narrow_split_count(int m, int n, int k, int sm_count);
cudaError_t sgemm_narrow(const GemmArgsF32& g, int splits, float* workspace, cudaStream_t st);

// C = beta * C on the m x n window (beta == 0 writes exact zeros, clearing NaNs),
// the reference's k == 0 / alpha == 0 quick return (gemm.zig:1407-1414).
cudaError_t scale_matrix_f64(int m, int n, double beta, double* c, long ldc, cudaStream_t st);
cudaError_t scale_matrix_f32(int m, int n, float beta, float* c, long ldc, cudaStream_t st);
// Complex (interleaved) scale by a complex beta.
cudaError_t scale_matrix_z(int m, int n, const double* beta, double* c, long ldc, cudaStream_t st);
cudaError_t scale_matrix_c(int m, int n, const float* beta, float* c, long ldc, cudaStream_t st);

// ------------------------------------------------------------ profiling
// When enabled (zynum_blas_gpu_profile), CUDA events are recorded on the
// launching stream around the dominant kernel of each call; the host reads
// the per-launch durations afterwards.  Disabled: no cost beyond a branch.
void prof_begin(cudaStream_t st);
// Every kernel launch of the library is counted (reported by
// zynum_blas_gpu_launch_count) so a caller can see the GPU work it caused.
void count_launch();
// cudaFuncSetAttribute(func, MaxDynamicSharedMemorySize, bytes) once per
// function, device and size (the attribute persists; repeating it per launch
// costs a driver call on every small GEMM).
cudaError_t ensure_dynamic_smem(const void* func, int bytes);
template <typename F>
cudaError_t ensure_dynamic_smem(F* func, int bytes) {
    return ensure_dynamic_smem(reinterpret_cast<const void*>(func), bytes);
}
void prof_end(cudaStream_t st);

// Fortran GEMM argument check (fortran.zig:88-102 gemmError): 0 or the index
// of the first illegal argument.  trans characters must already be upper case.
int gemm_arg_error(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc);

// cuTensorMapEncodeTiled from the driver (nullptr if unavailable), looked up once.
void* tensor_map_encoder();

// ---------------------------------------------------------------- planner
GemmPlan plan_native_gemm(int m, int n, int k, int elem_bytes, int sm_count);

}  // namespace zb
