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

// 32 MiB of FP64 partial sums.  The device memory behind it is committed when
// this file's module is loaded on a GPU: at library load with eager module
// loading, or at the first call on that GPU under lazy loading (the CUDA 12
// default), and it stays until the process exits.  Callers that reserve their
// whole memory pool at start-up make one call per GPU before reserving.
constexpr size_t kStaticScratchDoubles = size_t(4) << 20;
static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];
// Forced split counts are capped like the planner's own choices.
constexpr int kMaxForcedSplits = 64;

// Host code must not use g_static_scratch directly: on the host that name is a
// stand-in, not a device address.  The device address is looked up once per
// device, with that device current, and cached here, together with the check
// that the device is an sm_100 GPU.
constexpr int kMaxDevices = 64;
struct DeviceScratch {
    std::once_flag once;
    double* ptr = nullptr;
    cudaError_t err = cudaSuccess;
    bool wrong_arch = false;
};
DeviceScratch g_scratch[kMaxDevices];

cudaError_t device_setup(DeviceScratch** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    DeviceScratch& s = g_scratch[dev];
    std::call_once(s.once, [&s, dev] {
        int major = 0;
        s.err = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        if (s.err == cudaSuccess && major != 10) {
            s.wrong_arch = true;
            s.err = cudaErrorNoKernelImageForDevice;
            return;
        }
        void* p = nullptr;
        if (s.err == cudaSuccess) s.err = cudaGetSymbolAddress(&p, g_static_scratch);
        s.ptr = static_cast<double*>(p);
    });
    *out = &s;
    return s.err;
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
    DeviceScratch* ds = nullptr;
    if ((e = device_setup(&ds)) != cudaSuccess) {
        set_last_error(ds && ds->wrong_arch ? "dgemm_noalloc_device: this library runs on sm_100 (B200) GPUs only"
                                            : std::string("dgemm_noalloc_device: device set-up failed: ") +
                                                  cudaGetErrorString(e));
        return -(int)e;
    }
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
    if (splits > 0) plan.splits = splits < kMaxForcedSplits ? splits : kMaxForcedSplits;
    GemmArgsF64 g{ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    // scratch only for the partial sums of the K ranges the route really uses
    // (the tall-skinny route uses none; K slices are rounded up, which can
    // only lower the count)
    const int used = dgemm_native_used_splits(g, plan);
    const size_t need = splitk_workspace_elems(m, n, used);
    if (need > kStaticScratchDoubles) {
        set_last_error("dgemm_noalloc_device: splits * m * n = " + std::to_string(need) +
                       " partial sums exceed the fixed scratch of " + std::to_string(kStaticScratchDoubles) +
                       " doubles (32 MiB); use fewer splits or zynum_blas_gpu_dgemm_device");
        return -(int)cudaErrorInvalidValue;
    }
    double* scratch = need ? ds->ptr : nullptr;
    e = dgemm_native(g, plan, scratch, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("dgemm_noalloc_device: ") + cudaGetErrorString(e));
        return -(int)e;
    }
    return 0;
}
