// Ozaki-scheme DGEMM and SGEMM (INT8 tcgen05 slices / CRT residues) and 3xBF16 SGEMM.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "kernels.h"

namespace zb {

constexpr int kOzakiMaxSlices = 12;
// The automatic slice count never exceeds this (its workspace is sized for it).
constexpr int kOzakiAutoMaxSlices = 10;

// Scheme II (CRT): products of int8 residues modulo up to 16 pairwise coprime
// moduli <= 256; K is bounded so that a modular product cannot overflow INT32.
constexpr int kCrtMaxModuli = 16;
constexpr int kCrtDefaultModuli = 16;
constexpr int kCrtMaxK = 130816;  // 1022 x 128: k_pad * 128^2 < 2^31 - 2^21

enum OzakiScheme : int { OZAKI_AUTO = 0, OZAKI_SLICES = 1, OZAKI_CRT = 2 };

struct OzakiPlan {
    int scheme = OZAKI_SLICES;  // OZAKI_SLICES or OZAKI_CRT after planning
    int moduli = 0;   // CRT: number of moduli (products)
    int slices = 0;   // INT8 slices per operand (7 bits each); 0 = chosen from the data
    int m_pad = 0;    // rows of A padded to the 128-row UMMA tile
    int n_pad = 0;    // columns of B padded to the 256-column UMMA tile
    int k_pad = 0;    // K padded to the 128-byte TMA box
    bool pair = false;  // CTA-pair (cta_group::2, M = 256) slice-product kernel; m_pad is then a multiple of 256
    bool hold = false;  // test-only: the product kernel's MMA issuer waits on a barrier nothing arrives on
};

// Bounded waits of the tensor-core product kernels: every mbarrier wait gives
// up after a time limit, records its site in the device's report word and
// leaves C untouched (CRT scheme; the slice scheme's fused epilogue may have
// updated part of C).  Reads and clears the current device's report word
// after synchronising `stream`: 0 if no wait ran out since the last read, else
// the site (1 .. 7); *err receives a CUDA error of the read itself.
int ozaki_take_wait_report(cudaStream_t stream, cudaError_t* err);
// Device address of the current device's report word, for other kernels with
// bounded waits (looked up once per device; marks the word as worth reading).
cudaError_t wait_report_word(int** out);

// Whether the automatic method should prefer Ozaki for this shape.
bool ozaki_preferred(int m, int n, int k);
// The same model against a native route that does native_fraction of the full
// product's flops (0.5: triangle-mode tiles), the emulated route ozaki_fraction
// of its products and reconstruction (0.5: triangle tiles) and extra_bytes more
// through HBM.
bool ozaki_preferred_scaled(int m, int n, int k, double native_fraction, double ozaki_fraction, double extra_bytes);
// Scheme choice: OZAKI_AUTO takes the slice scheme when `slices` > 0 and the
// CRT scheme otherwise (K <= kCrtMaxK); OZAKI_CRT falls back to slices beyond
// kCrtMaxK.  slices == 0 leaves the slice count to dgemm_ozaki, which derives
// it from the dynamic range of the operands (and synchronises the stream to
// read it); moduli == 0 takes kCrtDefaultModuli.
OzakiPlan plan_ozaki(int m, int n, int k, int slices, int scheme = OZAKI_AUTO, int moduli = 0);
// Row / column scaling bits of the CRT scheme with `moduli` moduli: every
// scaled row of op(A) and column of op(B) has 2-norm <= 2^P.
int ozaki_crt_bits(int moduli);
// Modulus count of the most recent CRT-scheme call.
int ozaki_last_moduli();
int ozaki_auto_slices(float spread_a, float spread_b);
// Slice count of the most recent Ozaki call.
int ozaki_last_slices();
size_t ozaki_workspace_bytes(const OzakiPlan& p);
// C = alpha op(A) op(B) + beta C through INT8 slice or residue products; `ws` holds
// ozaki_workspace_bytes(p) bytes of device scratch.  a_ready (CRT scheme only):
// op(A)'s row statistics, exponents and residue planes are already in `ws` from an
// earlier call on the same op(A), plan and workspace (column panels of one product);
// they are reused, not recomputed.  The plan may cover more columns than g.n.
cudaError_t dgemm_ozaki(const GemmArgsF64& g, const OzakiPlan& p, void* ws, cudaStream_t st, bool a_ready = false);

// FP32 GEMM through the CRT scheme: FP32 operands are scaled per row of op(A) /
// column of op(B) to integers (exact FP64 widening first), multiplied modulo
// sgemm_crt_moduli(k) int8 moduli with exact INT32 accumulation, reconstructed
// in FP64 and rounded once to FP32 (alpha x + beta C in FP64).  Rows / columns
// holding Inf or NaN get IEEE results from a plain dot-product patch.
// The plan comes from plan_ozaki(m, n, k, 0, OZAKI_CRT, moduli), k <= kCrtMaxK.
int sgemm_crt_moduli(int k);
cudaError_t sgemm_ozaki(const GemmArgsF32& g, const OzakiPlan& p, void* ws, cudaStream_t st);

size_t bf16x3_workspace_bytes(int m, int n, int k);
// C = alpha op(A) op(B) + beta C as a 3xBF16 split product with FP32 accumulation.
cudaError_t sgemm_bf16x3(const GemmArgsF32& g, void* ws, cudaStream_t st);

}  // namespace zb
