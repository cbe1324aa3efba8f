// Raw issue-rate probes of the two pipes the library's hot kernels run on,
// measured on the GPU at hand so that roofline fractions use a measured
// denominator:
//   * FP64 tensor pipe: a register-only loop of independent DMMA
//     (mma.sync m16n8k8 .f64) per warp, 8 warps per CTA, two CTAs per SM;
//   * INT8 tcgen05 pipe: one thread per CTA pair issuing a chain of
//     tcgen05.mma.cta_group::2.kind::i8 M = 256, N = 256, K = 32 on operands
//     resident in shared memory (pseudo-random bytes, 128-byte swizzle layout),
//     one pair per two SMs, accumulating in TMEM.
// Neither touches global memory beyond one result word per thread (DMMA) or
// nothing at all (tcgen05); the host times them with CUDA events.
#include <cstdint>

#include "../../include/zynum_blas_gpu.h"
#include "bounded_wait.cuh"
#include "common.cuh"
#include "kernels.h"
#include "ozaki.h"
#include "runtime.h"

namespace zb {
namespace {

constexpr int kDmmaWarps = 8, kDmmaChain = 8;

__global__ void __launch_bounds__(kDmmaWarps * 32) dmma_rate_probe(double* out, int iters) {
    double acc[kDmmaChain][4];
#pragma unroll
    for (int i = 0; i < kDmmaChain; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[i][v] = 0.0;
    const double a[4] = {1.0 + threadIdx.x * 1e-9, 0.5, 0.25, 0.125}, b[2] = {1.0, 0.5};
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kDmmaChain; ++i) dmma_16x8x8(acc[i], a, b);
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kDmmaChain; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) s += acc[i][v];
    out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;  // out holds gridDim.x * blockDim.x doubles
}

constexpr int kUmmaProbeThreads = 128;
constexpr int kUmmaTile = 128 * 128;  // 128 rows x 128 bytes per operand and CTA
constexpr size_t kUmmaProbeSmem = 1024 + 2 * kUmmaTile + 64;

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kUmmaProbeThreads, 1)
umma_i8_rate_probe(int iters, int* report, unsigned long long wait_ns) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + kUmmaTile;
    uint64_t* done = reinterpret_cast<uint64_t*>(smem + 2 * kUmmaTile);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t rank = cluster_ctarank();
    // pseudo-random operand bytes (the pipe's rate depends on the data's toggling)
    for (int i = threadIdx.x; i < 2 * kUmmaTile / 4; i += kUmmaProbeThreads) {
        uint32_t x = (uint32_t)(i + 1) * 2654435761u ^ (blockIdx.x * 40503u);
        x ^= x >> 13;
        x *= 0x5bd1e995u;
        x ^= x >> 15;
        reinterpret_cast<uint32_t*>(smem)[i] = x;
    }
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    fence_proxy_async();  // the generic-proxy operand writes are visible to the tensor cores
    if (threadIdx.x < 32) {
        tmem_alloc_2sm(tmem_slot, 256);
        tmem_relinquish_2sm();
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (rank == 0 && threadIdx.x == 0) {
        const uint32_t idesc = umma_idesc(2, 1, 256, 256);
        const uint64_t ad = umma_desc_sw128(smem_u32(sA)), bd = umma_desc_sw128(smem_u32(sB));
        for (int it = 0; it < iters; ++it) {
            umma_i8_2sm(tmem, ad, bd, idesc, it > 0 ? 1u : 0u);
            umma_i8_2sm(tmem, ad + 2, bd + 2, idesc, 1u);
            umma_i8_2sm(tmem, ad + 4, bd + 4, idesc, 1u);
            umma_i8_2sm(tmem, ad + 6, bd + 6, idesc, 1u);
        }
        umma_commit_2sm(done, 0x3);  // arrives in both CTAs once every MMA completed
    }
    if (threadIdx.x == 0) {
        const WaitCtl W{abort_flag, nullptr, report, wait_ns};
        wait_phase(done, 0, W, WAIT_MMA_FULL_A);
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    tc_fence_after();
    if (threadIdx.x < 32) tmem_dealloc_2sm(tmem, 256);
}

}  // namespace
}  // namespace zb

using namespace zb;

extern "C" int zynum_blas_gpu_measure_pipe_rate(int pipe, double* rate, void* stream) {
    if (!rate || (pipe != 0 && pipe != 1)) return 1;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    double work = 0.0;
    float ms = 0.f;
    if (e == cudaSuccess && pipe == 0) {
        const int blocks = 2 * cx.sm_count, threads = kDmmaWarps * 32, iters = 20000;
        double* out = nullptr;
        e = cudaMallocAsync(reinterpret_cast<void**>(&out), sizeof(double) * blocks * threads, st);
        for (int rep = 0; e == cudaSuccess && rep < 3; ++rep) {  // the last of three runs is timed
            if ((e = cudaEventRecord(e0, st)) != cudaSuccess) break;
            dmma_rate_probe<<<blocks, threads, 0, st>>>(out, iters);
            count_launch();
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            e = cudaEventRecord(e1, st);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (out) cudaFreeAsync(out, st);
        work = (double)blocks * kDmmaWarps * iters * kDmmaChain * 2048.0;  // 2 x 16 x 8 x 8 flop per DMMA
    } else if (e == cudaSuccess) {
        const int pairs = cx.sm_count / 2, iters = 100000;
        int* report = nullptr;
        e = wait_report_word(&report);
        if (e == cudaSuccess) e = ensure_dynamic_smem(umma_i8_rate_probe, (int)kUmmaProbeSmem);
        for (int rep = 0; e == cudaSuccess && rep < 3; ++rep) {
            if ((e = cudaEventRecord(e0, st)) != cudaSuccess) break;
            umma_i8_rate_probe<<<2 * pairs, kUmmaProbeThreads, kUmmaProbeSmem, st>>>(iters, report, 4000000000ull);
            count_launch();
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            e = cudaEventRecord(e1, st);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = check_wait_report(st);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        work = (double)pairs * iters * 4 * (2.0 * 256 * 256 * 32);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        set_last_error(std::string("measure_pipe_rate: ") + cudaGetErrorString(e));
        return -(int)e;
    }
    *rate = work / (ms * 1e-3) / 1e12;
    return 0;
}
