// placeholder, replaced by the Ozaki implementation
#include "ozaki.h"
namespace zb {
bool ozaki_preferred(int, int, int) { return false; }
OzakiPlan plan_ozaki(int, int, int, int) { return OzakiPlan{}; }
size_t ozaki_workspace_bytes(const OzakiPlan&) { return 0; }
cudaError_t dgemm_ozaki(const GemmArgsF64&, const OzakiPlan&, void*, cudaStream_t) { return cudaErrorNotSupported; }
size_t bf16x3_workspace_bytes(int, int, int) { return 0; }
cudaError_t sgemm_bf16x3(const GemmArgsF32&, void*, cudaStream_t) { return cudaErrorNotSupported; }
}
