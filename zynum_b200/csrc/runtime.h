// Per-process GPU context of the shim: device, host-ABI stream, staging and
// workspace buffers, method switches and the last-error string.
//
// Replaces the reference's CPU runtime/thread pool (runtime.zig:54 maxThreads,
// execution/thread_pool.zig:247-264) for the GPU product: the "pool" here is
// one CUDA stream per host-ABI context plus grow-on-demand device buffers.
// Ownership follows the reference's rule that internal workspace is acquired
// before any write to caller memory (gemm.zig:48-53): every host entry point
// reserves all of its device memory first and returns with C untouched if that
// fails.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>

#include <cuda_runtime.h>

namespace zb {

enum DgemmMethod : int { METHOD_NATIVE = 0, METHOD_OZAKI = 1, METHOD_AUTO = 2 };
enum SgemmMethod : int { SMETHOD_NATIVE = 0, SMETHOD_BF16X3 = 1, SMETHOD_OZAKI = 2 };

// A device buffer that only grows.  Growing synchronises `stream` first so the
// old allocation is no longer in use.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t need, cudaStream_t stream);
    void release();
};

// Host-side fault injection used by the tests (no GPU fault is ever made):
// the next reservation fails with cudaErrorMemoryAllocation, the next stream
// synchronisation reports the given error, or the next tensor-core product
// kernels run with a hold (their MMA issuer first waits on a barrier that
// nothing arrives on, with a 1 ms limit, so the kernel's bounded-wait abort
// path runs and the call reports it).
struct InjectedFaults {
    int fail_next_reservations = 0;
    int fail_next_sync = 0;  // cudaError_t code
    std::atomic<int> hold_next_products{0};
    // True (and one fewer left) if the next product kernel is to run with the hold.
    bool take_hold() {
        int v = hold_next_products.load();
        while (v > 0 && !hold_next_products.compare_exchange_weak(v, v - 1)) {
        }
        return v > 0;
    }
};

struct Context {
    int device = -1;
    int sm_count = 148;
    cudaStream_t stream = nullptr;  // stream of the host (Fortran / CBLAS) entry points
    // Upload / download streams of the column-panel pipeline of large host GEMMs.
    cudaStream_t stream_in = nullptr, stream_out = nullptr;
    std::recursive_mutex mutex;     // host entry points are callable from any thread
    DeviceBuffer stage_a, stage_b, stage_c;
    DeviceBuffer work;  // scratch of the host entry points (split-K partials, slices)
    // Scratch of the device entry points, one per caller stream so that calls
    // on different streams never share scratch memory.
    std::unordered_map<cudaStream_t, DeviceBuffer> stream_work;
    int dgemm_method = METHOD_NATIVE;
    int sgemm_method = SMETHOD_NATIVE;
    int ozaki_slices = 0;  // 0 = automatic
    int ozaki_scheme = 0;  // 0 = automatic, 1 = INT8 slices, 2 = CRT residues
    int ozaki_moduli = 0;  // CRT moduli, 0 = default
    int complex_method = 0;  // 0 = expanded-real 4M, 1 = 3M
    InjectedFaults faults;
    bool initialised = false;
    cudaError_t init();
    void shutdown();
    // Scratch for a device entry point running on `stream`.
    cudaError_t stream_scratch(cudaStream_t stream, size_t bytes, void** out);
    cudaError_t reserve(DeviceBuffer& buf, size_t bytes, cudaStream_t stream);
    // Synchronise `stream`; afterwards a bounded wait that ran out in a
    // product kernel (the device's report word) is returned as
    // cudaErrorLaunchTimeout with its site in the last-error text.
    cudaError_t sync(cudaStream_t stream);
    // Host wait for an event; reports an injected synchronisation error like sync().
    cudaError_t wait_event(cudaEvent_t ev);
};

Context& context();

// Read (and clear) the device's bounded-wait report after `s` was
// synchronised: cudaErrorLaunchTimeout if a product kernel's wait ran out
// (its site is kept for take_wait_site), else cudaSuccess or the read's error.
cudaError_t check_wait_report(cudaStream_t s);
// Site recorded by the last check_wait_report on this thread that found one (0: none); clears it.
int take_wait_site();

void set_last_error(const std::string& msg);
const char* last_error();

// Dominant-kernel timing (see prof_begin / prof_end in kernels.h).
int profile_control(int enable);
int profile_read(double* ms, int max);
long long launch_count();

// Reference-style error report (fortran.zig:277 reportError -> xerbla_ :20).
void report_xerbla(const char* routine, int info);

}  // namespace zb
