// Ozaki-scheme DGEMM (INT8 tcgen05 slices) and 3xBF16 SGEMM.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "kernels.h"

namespace zb {

constexpr int kOzakiMaxSlices = 12;
// The automatic slice count never exceeds this (its workspace is sized for it).
constexpr int kOzakiAutoMaxSlices = 10;

struct OzakiPlan {
    int slices = 0;   // INT8 slices per operand (7 bits each); 0 = chosen from the data
    int m_pad = 0;    // rows of A padded to the 128-row UMMA tile
    int n_pad = 0;    // columns of B padded to the 256-column UMMA tile
    int k_pad = 0;    // K padded to the 128-byte TMA box
    bool pair = false;  // CTA-pair (cta_group::2, M = 256) slice-product kernel; m_pad is then a multiple of 256
};

// Whether the automatic method should prefer Ozaki for this shape.
bool ozaki_preferred(int m, int n, int k);
// slices == 0 leaves the count to dgemm_ozaki, which derives it from the
// dynamic range of the operands (and synchronises the stream to read it).
OzakiPlan plan_ozaki(int m, int n, int k, int slices);
int ozaki_auto_slices(float spread_a, float spread_b);
// Slice count of the most recent Ozaki call.
int ozaki_last_slices();
size_t ozaki_workspace_bytes(const OzakiPlan& p);
// C = alpha op(A) op(B) + beta C through INT8 slice products; `ws` holds
// ozaki_workspace_bytes(p) bytes of device scratch.
cudaError_t dgemm_ozaki(const GemmArgsF64& g, const OzakiPlan& p, void* ws, cudaStream_t st);

size_t bf16x3_workspace_bytes(int m, int n, int k);
// C = alpha op(A) op(B) + beta C as a 3xBF16 split product with FP32 accumulation.
cudaError_t sgemm_bf16x3(const GemmArgsF32& g, void* ws, cudaStream_t st);

}  // namespace zb
