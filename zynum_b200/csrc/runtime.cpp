#include "runtime.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <mutex>
#include <tuple>
#include <set>
#include <atomic>

#include "kernels.h"
#include "ozaki.h"

namespace zb {

namespace {
thread_local std::string g_last_error;

int parse_method_env() {
    const char* v = std::getenv("ZYNUM_GPU_DGEMM_METHOD");
    if (!v) return METHOD_NATIVE;
    if (!std::strcmp(v, "ozaki")) return METHOD_OZAKI;
    if (!std::strcmp(v, "auto")) return METHOD_AUTO;
    return METHOD_NATIVE;
}
int parse_smethod_env() {
    const char* v = std::getenv("ZYNUM_GPU_SGEMM_METHOD");
    if (v && !std::strcmp(v, "bf16x3")) return SMETHOD_BF16X3;
    if (v && !std::strcmp(v, "ozaki")) return SMETHOD_OZAKI;
    return SMETHOD_NATIVE;
}
int parse_complex_env() {
    const char* v = std::getenv("ZYNUM_GPU_COMPLEX_METHOD");
    return (v && !std::strcmp(v, "3m")) ? 1 : 0;
}
int parse_scheme_env() {
    const char* v = std::getenv("ZYNUM_GPU_OZAKI_SCHEME");
    if (v && !std::strcmp(v, "slices")) return 1;
    if (v && !std::strcmp(v, "crt")) return 2;
    return 0;
}
int parse_moduli_env() {
    const char* v = std::getenv("ZYNUM_GPU_OZAKI_MODULI");
    if (!v) return 0;
    int s = std::atoi(v);
    return (s >= 2 && s <= 16) ? s : 0;
}
int parse_slices_env() {
    const char* v = std::getenv("ZYNUM_GPU_OZAKI_SLICES");
    if (!v || !std::strcmp(v, "auto")) return 0;
    int s = std::atoi(v);
    return (s >= 2 && s <= 12) ? s : 0;
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

void report_xerbla(const char* routine, int info) {
    // Same text as the reference (fortran.zig:34-39); routine names are trimmed.
    char name[16] = {0};
    size_t n = 0;
    while (n < 6 && routine[n] && routine[n] != ' ') {
        name[n] = routine[n];
        ++n;
    }
    std::fprintf(stderr, " ** On entry to %s parameter number %d had an illegal value\n", n ? name : "UNKNOWN", info);
}

cudaError_t DeviceBuffer::reserve(size_t need, cudaStream_t stream) {
    if (need <= bytes) return cudaSuccess;
    if (ptr) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    size_t cap = need + need / 4;
    cap = (cap + 4095) & ~size_t(4095);
    cudaError_t e = cudaMalloc(&ptr, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        // retry at the exact size before giving up
        e = cudaMalloc(&ptr, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            return e;
        }
        cap = need;
    }
    bytes = cap;
    return cudaSuccess;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

cudaError_t Context::init() {
    if (initialised) return cudaSuccess;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    if (prop.major != 10) {
        set_last_error("zynum_blas_gpu: this library runs on sm_100 (B200) GPUs only");
        return cudaErrorNoKernelImageForDevice;
    }
    sm_count = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream_out, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    dgemm_method = parse_method_env();
    sgemm_method = parse_smethod_env();
    ozaki_slices = parse_slices_env();
    ozaki_scheme = parse_scheme_env();
    ozaki_moduli = parse_moduli_env();
    complex_method = parse_complex_env();
    initialised = true;
    return cudaSuccess;
}

void Context::shutdown() {
    std::lock_guard<std::recursive_mutex> lock(mutex);
    if (!initialised) return;
    cudaStreamSynchronize(stream);
    stage_a.release();
    stage_b.release();
    stage_c.release();
    work.release();
    for (auto& kv : stream_work) {
        cudaStreamSynchronize(kv.first);
        kv.second.release();
    }
    stream_work.clear();
    cudaStreamSynchronize(stream_in);
    cudaStreamSynchronize(stream_out);
    cudaStreamDestroy(stream);
    cudaStreamDestroy(stream_in);
    cudaStreamDestroy(stream_out);
    stream = stream_in = stream_out = nullptr;
    initialised = false;
}

cudaError_t Context::reserve(DeviceBuffer& buf, size_t bytes, cudaStream_t s) {
    if (faults.fail_next_reservations > 0) {
        --faults.fail_next_reservations;
        return cudaErrorMemoryAllocation;
    }
    return buf.reserve(bytes, s);
}

cudaError_t Context::stream_scratch(cudaStream_t s, size_t bytes, void** out) {
    std::lock_guard<std::recursive_mutex> lock(mutex);
    DeviceBuffer& b = stream_work[s];
    if (bytes > b.bytes) {
        // growing means cudaMalloc, which a stream under CUDA-graph capture does not allow
        // (it would invalidate the capture): refuse with a message instead
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            set_last_error("the stream is under graph capture and its workspace must grow to " +
                           std::to_string(bytes) + " bytes: make the same call (or a larger one) once on this "
                           "stream before capturing");
            *out = nullptr;
            return cudaErrorStreamCaptureUnsupported;
        }
    }
    cudaError_t e = reserve(b, bytes, s);
    *out = b.ptr;
    return e;
}

namespace {
thread_local int g_wait_site = 0;  // site of the last bounded wait seen to run out on this thread
}

cudaError_t check_wait_report(cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    const int site = ozaki_take_wait_report(s, &err);
    if (err != cudaSuccess) return err;
    if (site) {
        g_wait_site = site;
        return cudaErrorLaunchTimeout;
    }
    return cudaSuccess;
}

int take_wait_site() {
    const int v = g_wait_site;
    g_wait_site = 0;
    return v;
}

cudaError_t Context::sync(cudaStream_t s) {
    if (faults.fail_next_sync) {
        cudaError_t e = static_cast<cudaError_t>(faults.fail_next_sync);
        faults.fail_next_sync = 0;
        cudaStreamSynchronize(s);
        return e;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? check_wait_report(s) : e;
}

cudaError_t Context::wait_event(cudaEvent_t ev) {
    if (faults.fail_next_sync) {
        cudaError_t e = static_cast<cudaError_t>(faults.fail_next_sync);
        faults.fail_next_sync = 0;
        cudaEventSynchronize(ev);
        return e;
    }
    cudaError_t e = cudaEventSynchronize(ev);
    // the report is read on the download stream, which is idle or copying finished panels
    return e == cudaSuccess ? check_wait_report(stream_out) : e;
}

namespace {
struct Profiler {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> events;  // begin/end pairs
    size_t used = 0;
};
Profiler& profiler() {
    static Profiler* p = new Profiler();
    return *p;
}
cudaEvent_t next_event(Profiler& p) {
    if (p.used == p.events.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        p.events.push_back(e);
    }
    return p.events[p.used++];
}
}  // namespace

void prof_begin(cudaStream_t st) {
    Profiler& p = profiler();
    if (!p.on) return;
    std::lock_guard<std::mutex> lock(p.mu);
    if (p.used % 2) return;  // unmatched begin: ignore
    if (cudaEvent_t e = next_event(p)) cudaEventRecord(e, st);
}
void prof_end(cudaStream_t st) {
    Profiler& p = profiler();
    if (!p.on) return;
    std::lock_guard<std::mutex> lock(p.mu);
    if (p.used % 2 == 0) return;
    if (cudaEvent_t e = next_event(p)) cudaEventRecord(e, st);
}

namespace {
std::atomic<long long> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

cudaError_t ensure_dynamic_smem(const void* func, int bytes) {
    static std::mutex mu;
    static std::set<std::tuple<int, const void*, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const auto key = std::make_tuple(dev, func, bytes);
    std::lock_guard<std::mutex> lock(mu);
    if (done.count(key)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.insert(key);
    return e;
}
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

int profile_control(int enable) {
    Profiler& p = profiler();
    std::lock_guard<std::mutex> lock(p.mu);
    int old = p.on ? 1 : 0;
    p.on = enable != 0;
    p.used = 0;
    return old;
}

int profile_read(double* ms, int max) {
    Profiler& p = profiler();
    std::lock_guard<std::mutex> lock(p.mu);
    int n = 0;
    for (size_t q = 0; q + 1 < p.used && n < max; q += 2) {
        if (cudaEventSynchronize(p.events[q + 1]) != cudaSuccess) return -1;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, p.events[q], p.events[q + 1]) != cudaSuccess) return -1;
        ms[n++] = t;
    }
    return n;
}

void* tensor_map_encoder() {
    static void* fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = p;
    });
    return fn;
}

Context& context() {
    static Context* c = new Context();  // never destroyed: CUDA may be torn down first at exit
    return *c;
}

}  // namespace zb
