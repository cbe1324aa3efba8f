// Allocation-free split-K DGEMM entry point.
//
// Some callers cannot have the library call cudaMalloc: applications whose
// device memory is owned by their own pool allocator (a framework's caching
// allocator, a solver that reserves all memory at start-up), where a second
// allocator fails or fragments the pool; and latency-critical loops, where
// cudaMalloc / cudaFree stall because they synchronise the device.  For them
// this file offers one DGEMM entry point that never allocates: its split-K
// partial sums live in a fixed file-scope device array instead of a
// grow-on-demand buffer.
#include <mutex>

#include "../../include/zynum_blas_gpu.h"
#include "kernels.h"
#include "runtime.h"

namespace zb {
namespace {

// 32 MiB of FP64 partial sums.  Every GPU that loads this library holds it
// until the process exits.
constexpr size_t kStaticScratchDoubles = size_t(4) << 20;
static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];

// Host code must not use g_static_scratch directly: on the host that name is a
// stand-in, not a device address.  The device address is looked up once per
// device, with that device current, and cached here.
constexpr int kMaxDevices = 64;
struct DeviceScratch {
    std::once_flag once;
    double* ptr = nullptr;
    cudaError_t err = cudaSuccess;
};
DeviceScratch g_scratch[kMaxDevices];

cudaError_t static_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    DeviceScratch& s = g_scratch[dev];
    std::call_once(s.once, [&s] {
        void* p = nullptr;
        s.err = cudaGetSymbolAddress(&p, g_static_scratch);
        s.ptr = static_cast<double*>(p);
    });
    if (s.err != cudaSuccess) return s.err;
    *out = s.ptr;
    return cudaSuccess;
}

}  // namespace
}  // namespace zb

using namespace zb;

extern "C" int zynum_blas_gpu_dgemm_noalloc_device(char transa, char transb, int m, int n, int k, double alpha,
                                                   const double* a, int lda, const double* b, int ldb, double beta,
                                                   double* c, int ldc, int splits, void* stream) {
    const char ta = (char)((transa >= 'a' && transa <= 'z') ? transa - 32 : transa);
    const char tb = (char)((transb >= 'a' && transb <= 'z') ? transb - 32 : transb);
    const int info = gemm_arg_error(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (k == 0 || alpha == 0.0) {
        e = scale_matrix_f64(m, n, beta, c, ldc, st);
        if (e != cudaSuccess) set_last_error(std::string("dgemm_noalloc_device: ") + cudaGetErrorString(e));
        return e == cudaSuccess ? 0 : -(int)e;
    }
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        set_last_error(std::string("dgemm_noalloc_device: ") + cudaGetErrorString(e));
        return -(int)e;
    }
    GemmPlan plan = plan_native_gemm(m, n, k, 8, sms);
    if (splits > 0) plan.splits = splits;
    const size_t need = splitk_workspace_elems(m, n, plan.splits);
    if (need > kStaticScratchDoubles) {
        set_last_error("dgemm_noalloc_device: splits * m * n = " + std::to_string(need) +
                       " partial sums exceed the fixed scratch of " + std::to_string(kStaticScratchDoubles) +
                       " doubles (32 MiB); use fewer splits or zynum_blas_gpu_dgemm_device");
        return -(int)cudaErrorInvalidValue;
    }
    double* scratch = nullptr;
    if (need && (e = static_scratch(&scratch)) != cudaSuccess) {
        set_last_error(std::string("dgemm_noalloc_device: scratch address lookup failed: ") + cudaGetErrorString(e));
        return -(int)e;
    }
    GemmArgsF64 g{ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    e = dgemm_native(g, plan, scratch, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("dgemm_noalloc_device: ") + cudaGetErrorString(e));
        return -(int)e;
    }
    return 0;
}
