// Fortran / CBLAS ABI of the GPU backend and the device-pointer entry points.
//
// Mirrors, symbol for symbol, the reference's exports in
// src/blas/abi/fortran.zig and src/blas/abi/cblas.zig:
//   * argument validation and parameter numbering of gemmError (fortran.zig:88-102),
//   * xerbla_ reporting (fortran.zig:20, :277) with C left untouched,
//   * CBLAS enum validation with silent return and the row-major -> column-major
//     swap (cblas.zig:1415-1465),
//   * quick returns: m <= 0 or n <= 0 does nothing; k == 0 or alpha == 0 gives
//     C = beta * C with beta == 0 writing exact zeros (gemm.zig:1392-1414).
// The compute always runs on the GPU; there is no CPU fallback.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/zynum_blas_gpu.h"
#include "kernels.h"
#include "complex.h"
#include "ozaki.h"
#include "level3.h"
#include "runtime.h"

using namespace zb;

namespace {

inline char up(const char* p) { return (char)std::toupper((unsigned char)p[0]); }
inline bool valid_trans(char c) { return c == 'N' || c == 'T' || c == 'C'; }
inline int max1(int x) { return x > 1 ? x : 1; }

// fortran.zig:88-102 gemmError
int gemm_error(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc) {
    if (!valid_trans(ta)) return 1;
    if (!valid_trans(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    const int nrowa = (ta == 'N') ? m : k;
    const int nrowb = (tb == 'N') ? k : n;
    if (lda < max1(nrowa)) return 8;
    if (ldb < max1(nrowb)) return 10;
    if (ldc < max1(m)) return 13;
    return 0;
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    const int site = e == cudaErrorLaunchTimeout ? take_wait_site() : 0;
    if (site)
        set_last_error(std::string(what) + ": a bounded wait in a tensor-core product kernel ran out (site " +
                       std::to_string(site) + "); the product was abandoned and C was not written");
    else if (e == cudaErrorStreamCaptureUnsupported)  // keep the workspace message of stream_scratch
        set_last_error(std::string(what) + ": " + last_error());
    else
        set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return -(int)e;
}

void report_gpu_failure(const char* routine) {
    std::fprintf(stderr, " ** zynum_blas_gpu: %s did not run on the GPU (%s); C is unchanged\n", routine,
                 last_error());
}

// Scratch providers: the host ABI uses the context's own buffer on its stream;
// the device entry points use a per-caller-stream buffer.
struct HostScratch {
    Context* cx;
    cudaError_t operator()(size_t bytes, cudaStream_t st, void** out) {
        cudaError_t e = cx->reserve(cx->work, bytes, st);
        *out = cx->work.ptr;
        return e;
    }
};
struct StreamScratch {
    Context* cx;
    cudaError_t operator()(size_t bytes, cudaStream_t st, void** out) { return cx->stream_scratch(st, bytes, out); }
};

template <typename T>
cudaError_t scale_matrix(int m, int n, T beta, T* c, long ldc, cudaStream_t st);
template <>
cudaError_t scale_matrix<double>(int m, int n, double beta, double* c, long ldc, cudaStream_t st) {
    return scale_matrix_f64(m, n, beta, c, ldc, st);
}
template <>
cudaError_t scale_matrix<float>(int m, int n, float beta, float* c, long ldc, cudaStream_t st) {
    return scale_matrix_f32(m, n, beta, c, ldc, st);
}

// Device-pointer real GEMM on `st`; arguments already validated, m, n > 0.
template <typename Scratch>
cudaError_t run_dgemm(const GemmArgsF64& g, cudaStream_t st, Scratch scratch) {
    Context& cx = context();
    if (g.k == 0 || g.alpha == 0.0) return scale_matrix<double>(g.m, g.n, g.beta, g.c, g.ldc, st);
    int method = cx.dgemm_method;
    if (method == METHOD_AUTO) method = ozaki_preferred(g.m, g.n, g.k) ? METHOD_OZAKI : METHOD_NATIVE;
    if (method == METHOD_OZAKI) {
        OzakiPlan op = plan_ozaki(g.m, g.n, g.k, cx.ozaki_slices, cx.ozaki_scheme, cx.ozaki_moduli);
        op.hold = cx.faults.take_hold();
        void* ws = nullptr;
        cudaError_t e = scratch(ozaki_workspace_bytes(op), st, &ws);
        if (e != cudaSuccess) return e;
        return dgemm_ozaki(g, op, ws, st);
    }
    GemmPlan p = plan_native_gemm(g.m, g.n, g.k, 8, cx.sm_count);
    void* ws = nullptr;
    size_t need = splitk_workspace_elems(g.m, g.n, p.splits) * sizeof(double);
    if (need) {
        cudaError_t e = scratch(need, st, &ws);
        if (e != cudaSuccess) return e;
    }
    return dgemm_native(g, p, static_cast<double*>(ws), st);
}

template <typename Scratch>
cudaError_t run_sgemm(const GemmArgsF32& g, cudaStream_t st, Scratch scratch) {
    Context& cx = context();
    if (g.k == 0 || g.alpha == 0.0f) return scale_matrix<float>(g.m, g.n, g.beta, g.c, g.ldc, st);
    if (cx.sgemm_method == SMETHOD_BF16X3) {
        void* ws = nullptr;
        cudaError_t e = scratch(bf16x3_workspace_bytes(g.m, g.n, g.k), st, &ws);
        if (e != cudaSuccess) return e;
        return sgemm_bf16x3(g, ws, st);
    }
    if (cx.sgemm_method == SMETHOD_OZAKI) {
        // K beyond the INT32 bound of one modular product: K panels, each added to C
        const int kp = std::min(g.k, kCrtMaxK);
        const OzakiPlan op = plan_ozaki(g.m, g.n, kp, 0, OZAKI_CRT, sgemm_crt_moduli(kp));
        void* ws = nullptr;
        cudaError_t e = scratch(ozaki_workspace_bytes(op), st, &ws);
        for (int k0 = 0; e == cudaSuccess && k0 < g.k; k0 += kp) {
            GemmArgsF32 p = g;
            p.k = std::min(kp, g.k - k0);
            p.a = g.a + (g.transa == 'N' ? (long)k0 * g.lda : k0);
            p.b = g.b + (g.transb == 'N' ? k0 : (long)k0 * g.ldb);
            if (k0 > 0) p.beta = 1.0f;
            e = sgemm_ozaki(p, op, ws, st);
        }
        return e;
    }
    GemmPlan p = plan_native_gemm(g.m, g.n, g.k, 4, cx.sm_count);
    void* ws = nullptr;
    size_t need = sgemm_native_workspace_bytes(g.transa, g.transb, g.m, g.n, g.k, p);
    if (need) {
        cudaError_t e = scratch(need, st, &ws);
        if (e != cudaSuccess) return e;
    }
    return sgemm_native(g, p, static_cast<float*>(ws), st);
}

cudaError_t run_gemm(const GemmArgsF64& g, cudaStream_t st, HostScratch s) { return run_dgemm(g, st, s); }
cudaError_t run_gemm(const GemmArgsF32& g, cudaStream_t st, HostScratch s) { return run_sgemm(g, st, s); }

// Large host GEMMs run as column panels of C over three streams: the upload
// stream copies A and then, panel by panel, B (and C when beta != 0); the
// compute stream runs a panel's GEMM once its inputs are in; each C panel is
// downloaded on the download stream as soon as the host has seen its GEMM
// finish without error.  Uploads, products and downloads of different panels
// overlap (the link is full duplex).  Every device buffer is reserved before
// the first copy; a GPU error in panel j leaves panels 0 .. j-1 of C holding
// their final values and the rest of C untouched.
constexpr double kPanelMinFlops = 8.0e9;  // 2 m n k

size_t real_scratch_bytes(int m, int n, int k, double*);
size_t real_scratch_bytes(int m, int n, int k, float*);

int host_panel_count(int m, int n, int k) {
    if (n < 2048 || 2.0 * m * (double)n * k < kPanelMinFlops) return 1;
    // ZYNUM_GPU_HOST_PANELS: most panels per call (2..32, default 16; DGEMM 8192^3 through
    // dgemm_ measured 23.2 / 22.8 / 24.4 ms per call with 8 / 16 / 32 panels)
    static const int cap = [] {
        const char* v = std::getenv("ZYNUM_GPU_HOST_PANELS");
        const int x = v ? std::atoi(v) : 16;
        return (x >= 2 && x <= 32) ? x : 16;
    }();
    return std::min(cap, std::max(2, n / 1024 * cap / 8));
}

template <typename T>
void host_gemm_panels(const char* routine, Context& cx, int panels, char ta, char tb, int m, int n, int k, T alpha,
                      const T* a, int lda, const T* b, int ldb, T beta, T* c, int ldc, T* da, T* db, T* dc) {
    const cudaStream_t st = cx.stream, up = cx.stream_in, down = cx.stream_out;
    const int ra = (ta == 'N') ? m : k, ca = (ta == 'N') ? k : m;
    const int rb = (tb == 'N') ? k : n;
    const size_t es = sizeof(T);
    const int nb = ((n + panels - 1) / panels + 255) / 256 * 256;
    panels = (n + nb - 1) / nb;
    cudaError_t e = cx.reserve(cx.work, real_scratch_bytes(m, nb, k, (T*)nullptr), st);
    if (e != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    std::vector<cudaEvent_t> ev(2 * panels, nullptr);
    auto release = [&]() {
        cudaStreamSynchronize(up);
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(down);
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    };
    for (auto& x : ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    // uploads: A, then per panel op(B)[:, j0:j1] (and C[:, j0:j1]); in_j after panel j
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice,
                              up);
    for (int j = 0; j < panels && e == cudaSuccess; ++j) {
        const int j0 = j * nb, w = std::min(nb, n - j0);
        if (tb == 'N')  // B is k x n: columns j0 .. j0 + w
            e = cudaMemcpy2DAsync(db + (long)j0 * rb, (size_t)rb * es, b + (long)j0 * ldb, (size_t)ldb * es,
                                  (size_t)rb * es, w, cudaMemcpyHostToDevice, up);
        else  // B is n x k: rows j0 .. j0 + w
            e = cudaMemcpy2DAsync(db + j0, (size_t)rb * es, b + j0, (size_t)ldb * es, (size_t)w * es, k,
                                  cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess && beta != T(0))
            e = cudaMemcpy2DAsync(dc + (long)j0 * m, (size_t)m * es, c + (long)j0 * ldc, (size_t)ldc * es,
                                  (size_t)m * es, w, cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * j], up);
    }
    // products.  FP64 through the CRT Ozaki scheme: one plan for the full panel width,
    // op(A)'s residues computed by the first panel and reused by the others (its row
    // scaling depends on op(A) alone, each column of op(B) is scaled independently, so
    // the result equals the unpanelled product's)
    bool crt = false;
    OzakiPlan op{};
    if constexpr (std::is_same<T, double>::value) {
        int method = cx.dgemm_method;
        if (method == METHOD_AUTO) method = ozaki_preferred(m, nb, k) ? METHOD_OZAKI : METHOD_NATIVE;
        if (method == METHOD_OZAKI && k > 0 && alpha != 0.0) {
            op = plan_ozaki(m, nb, k, cx.ozaki_slices, cx.ozaki_scheme, cx.ozaki_moduli);
            op.hold = cx.faults.take_hold();
            crt = op.scheme == OZAKI_CRT;
        }
    }
    void* ows = nullptr;
    if (crt && e == cudaSuccess) e = HostScratch{&cx}(ozaki_workspace_bytes(op), st, &ows);
    for (int j = 0; j < panels && e == cudaSuccess; ++j) {
        const int j0 = j * nb, w = std::min(nb, n - j0);
        e = cudaStreamWaitEvent(st, ev[2 * j], 0);
        if (e != cudaSuccess) break;
        const T* bj = (tb == 'N') ? db + (long)j0 * rb : db + j0;
        GemmArgs<T> g{ta, tb, m, w, k, alpha, da, ra, bj, rb, beta, dc + (long)j0 * m, m};
        if constexpr (std::is_same<T, double>::value) {
            e = crt ? dgemm_ozaki(g, op, ows, st, j > 0) : run_gemm(g, st, HostScratch{&cx});
        } else {
            e = run_gemm(g, st, HostScratch{&cx});
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * j + 1], st);
    }
    if (e != cudaSuccess) {  // nothing of C was written yet
        release();
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    // downloads, each after its panel is known to have finished without error
    for (int j = 0; j < panels; ++j) {
        const int j0 = j * nb, w = std::min(nb, n - j0);
        if ((e = cx.wait_event(ev[2 * j + 1])) != cudaSuccess) {
            release();
            cuda_status(e, "GPU execution");
            report_gpu_failure(routine);
            return;
        }
        e = cudaMemcpy2DAsync(c + (long)j0 * ldc, (size_t)ldc * es, dc + (long)j0 * m, (size_t)m * es,
                              (size_t)m * es, w, cudaMemcpyDeviceToHost, down);
        if (e != cudaSuccess) break;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(down);
    release();
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

// Host-pointer GEMM: stage -> compute -> copy the C window back.
template <typename T>
void host_gemm(const char* routine, char ta, char tb, int m, int n, int k, T alpha, const T* a, int lda, const T* b,
               int ldb, T beta, T* c, int ldc) {
    if (m <= 0 || n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const bool quick = (k == 0 || alpha == T(0));
    const int ra = (ta == 'N') ? m : k, ca = (ta == 'N') ? k : m;
    const int rb = (tb == 'N') ? k : n, cb = (tb == 'N') ? n : k;
    const size_t es = sizeof(T);
    // Acquire every device buffer before touching C (failure before write).
    if (!quick) {
        if ((e = cx.reserve(cx.stage_a, (size_t)ra * ca * es, st)) != cudaSuccess ||
            (e = cx.reserve(cx.stage_b, (size_t)rb * cb * es, st)) != cudaSuccess) {
            cuda_status(e, "staging reservation");
            report_gpu_failure(routine);
            return;
        }
    }
    if ((e = cx.reserve(cx.stage_c, (size_t)m * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* db = static_cast<T*>(cx.stage_b.ptr);
    T* dc = static_cast<T*>(cx.stage_c.ptr);
    const int panels = quick ? 1 : host_panel_count(m, n, k);
    if (panels > 1) {
        host_gemm_panels<T>(routine, cx, panels, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, da, db, dc);
        return;
    }
    if (!quick) {
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(db, (size_t)rb * es, b, (size_t)ldb * es, (size_t)rb * es, cb, cudaMemcpyHostToDevice,
                                  st);
    }
    if (e == cudaSuccess && beta != T(0))
        e = cudaMemcpy2DAsync(dc, (size_t)m * es, c, (size_t)ldc * es, (size_t)m * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        GemmArgs<T> g{ta, tb, m, n, k, alpha, da, ra, db, rb, beta, dc, m};
        e = run_gemm(g, st, HostScratch{&cx});
    }
    if (e == cudaSuccess) e = cx.sync(st);  // compute finished without error before C is written
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)m * es, (size_t)m * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

// ---------------------------------------------------------------- complex
// Scratch the real GEMM of run_dgemm / run_sgemm would request for this shape.
size_t real_scratch_bytes(int m, int n, int k, double*) {
    Context& cx = context();
    int method = cx.dgemm_method;
    if (method == METHOD_AUTO) method = ozaki_preferred(m, n, k) ? METHOD_OZAKI : METHOD_NATIVE;
    if (method == METHOD_OZAKI) {
        size_t b = ozaki_workspace_bytes(plan_ozaki(m, n, k, cx.ozaki_slices, cx.ozaki_scheme, cx.ozaki_moduli));
        // a smaller-K product of the same call (TRSM updates) may take the CRT scheme
        if (cx.ozaki_scheme != OZAKI_SLICES && cx.ozaki_slices == 0)
            b = std::max(b, ozaki_workspace_bytes(plan_ozaki(m, n, std::min(k, kCrtMaxK), 0, OZAKI_CRT,
                                                              cx.ozaki_moduli)));
        return b;
    }
    GemmPlan p = plan_native_gemm(m, n, k, 8, cx.sm_count);
    return splitk_workspace_elems(m, n, p.splits) * sizeof(double);
}
size_t real_scratch_bytes(int m, int n, int k, float*) {
    Context& cx = context();
    if (cx.sgemm_method == SMETHOD_BF16X3) return bf16x3_workspace_bytes(m, n, k);
    if (cx.sgemm_method == SMETHOD_OZAKI) {
        const int kp = std::min(k, kCrtMaxK);
        return ozaki_workspace_bytes(plan_ozaki(m, n, kp, 0, OZAKI_CRT, sgemm_crt_moduli(kp)));
    }
    GemmPlan p = plan_native_gemm(m, n, k, 4, cx.sm_count);
    return sgemm_native_workspace_bytes('T', 'N', m, n, k, p);  // both operand copies, if any
}

// Scratch that covers every GEMM of shape up to m x n x k (TRSM's recursive
// updates): split-K partials never exceed sm_count x 128 x 128 elements
// (splits <= sm_count / tiles and tiles >= m n / 128^2) and matrix-vector
// partials kGemvMaxPartials, FP32 products may add
// an MN-contiguous copy of each operand, and the Ozaki planes grow with every
// dimension.
template <typename T>
size_t real_scratch_bound(int m, int n, int k) {
    Context& cx = context();
    const long partials = std::max<long>((long)cx.sm_count * 128 * 128, kGemvMaxPartials);
    const size_t splitk = sizeof(T) == 4 ? sgemm_native_workspace_bound(m, n, k, cx.sm_count)
                                         : (size_t)partials * sizeof(T) + 4096;
    return std::max(splitk, real_scratch_bytes(m, n, k, (T*)nullptr));
}

// A fixed region handed to the real GEMMs of a complex call.
struct FixedScratch {
    void* base;
    size_t cap;
    cudaError_t operator()(size_t bytes, cudaStream_t, void** out) {
        if (bytes > cap) return cudaErrorInvalidValue;
        *out = base;
        return cudaSuccess;
    }
};

cudaError_t run_real(const GemmArgsF64& g, cudaStream_t st, FixedScratch s) { return run_dgemm(g, st, s); }
cudaError_t run_real(const GemmArgsF32& g, cudaStream_t st, FixedScratch s) { return run_sgemm(g, st, s); }

cudaError_t scale_complex(int m, int n, const double* beta, double* c, long ldc, cudaStream_t st) {
    return scale_matrix_z(m, n, beta, c, ldc, st);
}
cudaError_t scale_complex(int m, int n, const float* beta, float* c, long ldc, cudaStream_t st) {
    return scale_matrix_c(m, n, beta, c, ldc, st);
}

// Device-pointer complex GEMM on `st`; arguments validated, m, n > 0.
template <typename T, typename Scratch>
cudaError_t run_complex(const ComplexArgs<T>& g, cudaStream_t st, Scratch scratch) {
    Context& cx = context();
    if (g.k == 0 || (g.alpha[0] == T(0) && g.alpha[1] == T(0)))
        return scale_complex(g.m, g.n, g.beta, g.c, g.ldc, st);
    const int method = cx.complex_method;
    const size_t planes = complex_plane_bytes<T>(method, g.m, g.n, g.k);
    const size_t real = (method == COMPLEX_3M) ? real_scratch_bytes(g.m, g.n, g.k, (T*)nullptr)
                                               : real_scratch_bytes(2 * g.m, g.n, 2 * g.k, (T*)nullptr);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    RealGemm<T> rg = [&](int m, int n, int k, const T* a, long lda, const T* b, long ldb, T* c, long ldc, int tri) {
        GemmArgs<T> rgs{'N', 'N', m, n, k, T(1), a, lda, b, ldb, T(0), c, ldc};
        rgs.tri = tri;
        return run_real(rgs, st, fs);
    };
    return complex_gemm<T>(g, method, ws, rg, st);
}

// Host-pointer complex GEMM: stage -> compute -> copy the C window back.
template <typename T>
void host_complex_gemm(const char* routine, char ta, char tb, int m, int n, int k, const T* alpha, const T* a,
                       int lda, const T* b, int ldb, const T* beta, T* c, int ldc) {
    if (m <= 0 || n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const bool quick = (k == 0 || (alpha[0] == T(0) && alpha[1] == T(0)));
    const bool beta0 = (beta[0] == T(0) && beta[1] == T(0));
    const int ra = (ta == 'N') ? m : k, ca = (ta == 'N') ? k : m;
    const int rb = (tb == 'N') ? k : n, cb = (tb == 'N') ? n : k;
    const size_t es = 2 * sizeof(T);
    if (!quick) {
        if ((e = cx.reserve(cx.stage_a, (size_t)ra * ca * es, st)) != cudaSuccess ||
            (e = cx.reserve(cx.stage_b, (size_t)rb * cb * es, st)) != cudaSuccess) {
            cuda_status(e, "staging reservation");
            report_gpu_failure(routine);
            return;
        }
    }
    if ((e = cx.reserve(cx.stage_c, (size_t)m * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* db = static_cast<T*>(cx.stage_b.ptr);
    T* dc = static_cast<T*>(cx.stage_c.ptr);
    if (!quick) {
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(db, (size_t)rb * es, b, (size_t)ldb * es, (size_t)rb * es, cb, cudaMemcpyHostToDevice,
                                  st);
    }
    if (e == cudaSuccess && !beta0)
        e = cudaMemcpy2DAsync(dc, (size_t)m * es, c, (size_t)ldc * es, (size_t)m * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        ComplexArgs<T> g{ta, tb, m, n, k, {alpha[0], alpha[1]}, da, ra, db, rb, {beta[0], beta[1]}, dc, m};
        e = run_complex(g, st, HostScratch{&cx});
    }
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)m * es, (size_t)m * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

template <typename T>
int device_complex_gemm(const char* what, char transa, char transb, int m, int n, int k, const T* alpha, const T* a,
                        int lda, const T* b, int ldb, const T* beta, T* c, int ldc, void* stream) {
    const char ta = up(&transa), tb = up(&transb);
    int info = gemm_error(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    ComplexArgs<T> g{ta, tb, m, n, k, {alpha[0], alpha[1]}, a, lda, b, ldb, {beta[0], beta[1]}, c, ldc};
    return cuda_status(run_complex(g, static_cast<cudaStream_t>(stream), StreamScratch{&cx}), what);
}

// ------------------------------------------------------------ TRSM / SYRK
inline bool valid_uplo(char c) { return c == 'U' || c == 'L'; }
inline bool valid_diag(char c) { return c == 'N' || c == 'U'; }
inline bool valid_side(char c) { return c == 'L' || c == 'R'; }

// fortran.zig:105-118 triangularMatrixError
int trsm_error(char side, char uplo, char trans, char diag, int m, int n, int lda, int ldb) {
    if (!valid_side(side)) return 1;
    if (!valid_uplo(uplo)) return 2;
    if (!valid_trans(trans)) return 3;
    if (!valid_diag(diag)) return 4;
    if (m < 0) return 5;
    if (n < 0) return 6;
    const int nrowa = (side == 'L') ? m : n;
    if (lda < max1(nrowa)) return 9;
    if (ldb < max1(m)) return 11;
    return 0;
}

// fortran.zig:252-263 rankKMatrixError
int syrk_error(char uplo, char trans, int n, int k, int lda, int ldc) {
    if (!valid_uplo(uplo)) return 1;
    if (!valid_trans(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    const int nrowa = (trans == 'N') ? n : k;
    if (lda < max1(nrowa)) return 7;
    if (ldc < max1(n)) return 10;
    return 0;
}

// fortran.zig:239-250 symmetricMatrixError
int symm_error(char side, char uplo, int m, int n, int lda, int ldb, int ldc) {
    if (!valid_side(side)) return 1;
    if (!valid_uplo(uplo)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    const int nrowa = (side == 'L') ? m : n;
    if (lda < max1(nrowa)) return 7;
    if (ldb < max1(m)) return 9;
    if (ldc < max1(m)) return 12;
    return 0;
}

// fortran.zig:264-275 rank2KMatrixError
int syr2k_error(char uplo, char trans, int n, int k, int lda, int ldb, int ldc) {
    if (!valid_uplo(uplo)) return 1;
    if (!valid_trans(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    const int nrow = (trans == 'N') ? n : k;
    if (lda < max1(nrow)) return 7;
    if (ldb < max1(nrow)) return 9;
    if (ldc < max1(n)) return 12;
    return 0;
}

// GEMMs inside TRSM: the real GEMM route with a fixed scratch region.
template <typename T>
GemmFn<T> gemm_fn(cudaStream_t st, FixedScratch* fs) {
    return [st, fs](const GemmArgs<T>& g) -> cudaError_t {
        if (g.m <= 0 || g.n <= 0) return cudaSuccess;
        return run_real(g, st, *fs);
    };
}

template <typename T, typename Scratch>
cudaError_t run_trsm(const TrsmArgs<T>& t, cudaStream_t st, Scratch scratch, const TrsmInverses* given = nullptr) {
    if (t.m <= 0 || t.n <= 0) return cudaSuccess;
    const size_t planes = trsm_plane_bytes<T>(t.side, t.m, t.n);
    // the GEMMs of the recursive solve are at most m x n x (order of A)
    const int na = (t.side == 'L') ? t.m : t.n;
    const size_t real = real_scratch_bound<T>(t.m, t.n, na);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return trsm<T>(t, ws, gemm_fn<T>(st, &fs), st, given);
}

// SYRK / SYR2K in FP64 take the emulated product when the DGEMM method is
// Ozaki, or automatic and the model prefers it (plus the triangle pass over W)
// to the native route.  SYRK: native triangle-mode tiles against emulated
// products on the triangle's tiles, each half a full product; SYR2K: two
// native triangle-mode GEMMs against one full emulated W.
inline bool rank_k_uses_ozaki(int n, int k, bool two) {
    const int method = context().dgemm_method;
    if (method == METHOD_OZAKI) return true;
    const double half = two ? 1.0 : 0.5;
    return method == METHOD_AUTO && ozaki_preferred_scaled(n, n, k, half, half, 24.0 * n * (double)n);
}

// W = op(A) op(B)^T as one emulated DGEMM into scratch, then
// C := alpha (W [+ W^T]) + beta C on the triangle (op(B) op(A)^T = W^T).  SYRK
// (one term) needs only W's stored triangle: the product runs in triangle mode
// and, op(B)^T being op(A), splits op(A) once.
template <typename Scratch>
cudaError_t run_rank_k_ozaki(char uplo, char trans, bool two, int n, int k, double alpha, const double* a, long lda,
                             const double* b, long ldb, double beta, double* c, long ldc, cudaStream_t st,
                             Scratch scratch) {
    Context& cx = context();
    const OzakiPlan op = plan_ozaki(n, n, k, cx.ozaki_slices, cx.ozaki_scheme, cx.ozaki_moduli);
    const size_t wbytes = ((size_t)n * n * sizeof(double) + 1023) & ~size_t(1023);
    void* ws = nullptr;
    cudaError_t e = scratch(wbytes + ozaki_workspace_bytes(op), st, &ws);
    if (e != cudaSuccess) return e;
    double* W = static_cast<double*>(ws);
    const char t1 = trans == 'N' ? 'N' : 'T', t2 = trans == 'N' ? 'T' : 'N';
    GemmArgsF64 g{t1, t2, n, n, k, 1.0, a, lda, b, ldb, 0.0, W, n};
    if (!two) g.tri = uplo == 'U' ? 1 : 2;
    if ((e = dgemm_ozaki(g, op, static_cast<char*>(ws) + wbytes, st)) != cudaSuccess) return e;
    return triangle_update<double>(uplo, two, n, alpha, W, n, beta, c, ldc, st);
}

template <typename T, typename Scratch>
cudaError_t run_syrk(char uplo, char trans, int n, int k, T alpha, const T* a, long lda, T beta, T* c, long ldc,
                     cudaStream_t st, Scratch scratch) {
    if (n <= 0) return cudaSuccess;
    if (k == 0) return syrk_scale_only<T>(n, uplo, beta, c, ldc, st);
    if constexpr (sizeof(T) == 8) {
        if (rank_k_uses_ozaki(n, k, false))
            return run_rank_k_ozaki(uplo, trans, false, n, k, alpha, a, lda, a, lda, beta, c, ldc, st, scratch);
    }
    Context& cx = context();
    GemmArgs<T> g{trans == 'N' ? 'N' : 'T', trans == 'N' ? 'T' : 'N', n, n, k, alpha, a, lda, a, lda, beta, c, ldc};
    g.tri = (uplo == 'U') ? 1 : 2;
    GemmPlan p = plan_native_gemm(n, n, k, sizeof(T), cx.sm_count);
    void* ws = nullptr;
    const size_t need = sizeof(T) == 4 ? sgemm_native_workspace_bytes(g.transa, g.transb, n, n, k, p)
                                       : splitk_workspace_elems(n, n, p.splits) * sizeof(T);
    if (need) {
        cudaError_t e = scratch(need, st, &ws);
        if (e != cudaSuccess) return e;
    }
    if constexpr (sizeof(T) == 8)
        return dgemm_native(g, p, static_cast<double*>(ws), st);
    else
        return sgemm_native(g, p, static_cast<float*>(ws), st);
}

template <typename T, typename Scratch>
cudaError_t run_trmm(const TrsmArgs<T>& t, cudaStream_t st, Scratch scratch) {
    if (t.m <= 0 || t.n <= 0) return cudaSuccess;
    const size_t planes = trmm_plane_bytes<T>(t.side, t.m, t.n);
    const int na = (t.side == 'L') ? t.m : t.n;
    const size_t real = real_scratch_bound<T>(t.m, t.n, na);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return trmm<T>(t, ws, gemm_fn<T>(st, &fs), st);
}

template <typename T, typename Scratch>
cudaError_t run_symm(char side, char uplo, int m, int n, T alpha, const T* a, long lda, const T* b, long ldb, T beta,
                     T* c, long ldc, cudaStream_t st, Scratch scratch) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    if (alpha == T(0)) return scale_matrix<T>(m, n, beta, c, ldc, st);
    const size_t planes = symm_plane_bytes<T>(side, m, n);
    const int na = (side == 'L') ? m : n;
    const size_t real = real_scratch_bytes(m, n, na, (T*)nullptr);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return symm<T>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, ws, gemm_fn<T>(st, &fs), st);
}

// SYR2K: two triangle-mode GEMMs, alpha op(A) op(B)^T + beta C, then
// alpha op(B) op(A)^T added with beta = 1.
template <typename T, typename Scratch>
cudaError_t run_syr2k(char uplo, char trans, int n, int k, T alpha, const T* a, long lda, const T* b, long ldb,
                      T beta, T* c, long ldc, cudaStream_t st, Scratch scratch) {
    if (n <= 0) return cudaSuccess;
    if (k == 0) return syrk_scale_only<T>(n, uplo, beta, c, ldc, st);
    if constexpr (sizeof(T) == 8) {
        if (rank_k_uses_ozaki(n, k, true))
            return run_rank_k_ozaki(uplo, trans, true, n, k, alpha, a, lda, b, ldb, beta, c, ldc, st, scratch);
    }
    Context& cx = context();
    const char t1 = trans == 'N' ? 'N' : 'T', t2 = trans == 'N' ? 'T' : 'N';
    GemmArgs<T> g1{t1, t2, n, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    GemmArgs<T> g2{t1, t2, n, n, k, alpha, b, ldb, a, lda, T(1), c, ldc};
    g1.tri = g2.tri = (uplo == 'U') ? 1 : 2;
    GemmPlan p = plan_native_gemm(n, n, k, sizeof(T), cx.sm_count);
    void* ws = nullptr;
    const size_t need = sizeof(T) == 4 ? sgemm_native_workspace_bytes(t1, t2, n, n, k, p)
                                       : splitk_workspace_elems(n, n, p.splits) * sizeof(T);
    if (need) {
        cudaError_t e = scratch(need, st, &ws);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e;
    if constexpr (sizeof(T) == 8) {
        if ((e = dgemm_native(g1, p, static_cast<double*>(ws), st)) != cudaSuccess) return e;
        return dgemm_native(g2, p, static_cast<double*>(ws), st);
    } else {
        if ((e = sgemm_native(g1, p, static_cast<float*>(ws), st)) != cudaSuccess) return e;
        return sgemm_native(g2, p, static_cast<float*>(ws), st);
    }
}

// Scratch that covers every complex GEMM of shape up to m x n x k under either
// complex method (the plane buffers plus the real GEMMs they run).
template <typename R>
size_t complex_scratch_bound(int m, int n, int k) {
    const size_t m4 = complex_plane_bytes<R>(COMPLEX_4M, m, n, k) + real_scratch_bound<R>(2 * m, n, 2 * k);
    const size_t m3 = complex_plane_bytes<R>(COMPLEX_3M, m, n, k) + real_scratch_bound<R>(m, n, k);
    return std::max(m4, m3) + 4096;
}

// GEMMs inside a complex TRSM: the complex GEMM route with a fixed scratch region.
template <typename R>
GemmFn<cnum<R>> gemm_fn_c(cudaStream_t st, FixedScratch* fs) {
    return [st, fs](const GemmArgs<cnum<R>>& g) -> cudaError_t {
        if (g.m <= 0 || g.n <= 0) return cudaSuccess;
        ComplexArgs<R> cg{g.transa, g.transb, g.m, g.n, g.k, {g.alpha.re, g.alpha.im},
                          reinterpret_cast<const R*>(g.a), g.lda, reinterpret_cast<const R*>(g.b), g.ldb,
                          {g.beta.re, g.beta.im}, reinterpret_cast<R*>(g.c), g.ldc};
        return run_complex(cg, st, *fs);
    };
}

// Complex TRSM (ztrsm_ / ctrsm_): the recursive solve with complex GEMM couplings.
template <typename R, typename Scratch>
cudaError_t run_trsm(const TrsmArgs<cnum<R>>& t, cudaStream_t st, Scratch scratch) {
    if (t.m <= 0 || t.n <= 0) return cudaSuccess;
    const size_t planes = trsm_plane_bytes<cnum<R>>(t.side, t.m, t.n);
    const int na = (t.side == 'L') ? t.m : t.n;
    const size_t real = complex_scratch_bound<R>(t.m, t.n, na);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return trsm<cnum<R>>(t, ws, gemm_fn_c<R>(st, &fs), st);
}

// Complex SYRK (zsyrk_ / csyrk_, symmetric.zig:180-199 with herm = false): one
// complex GEMM W = op(A) op(A)^T into scratch, then C := alpha W + beta C on
// the triangle.  trans = C takes op(A) = A^H, so op(A) op(A)^T = conj(A^T A).
template <typename R, typename Scratch>
cudaError_t run_syrk_c(char uplo, char trans, int n, int k, cnum<R> alpha, const cnum<R>* a, long lda, cnum<R> beta,
                       cnum<R>* c, long ldc, cudaStream_t st, Scratch scratch) {
    if (n <= 0) return cudaSuccess;
    if (k == 0 || alpha == cnum<R>(0)) return syrk_scale_only<cnum<R>>(n, uplo, beta, c, ldc, st);
    const size_t wbytes = ((size_t)n * n * sizeof(cnum<R>) + 1023) & ~size_t(1023);
    const size_t cb = complex_scratch_bound<R>(n, n, k);
    void* ws = nullptr;
    cudaError_t e = scratch(wbytes + cb, st, &ws);
    if (e != cudaSuccess) return e;
    cnum<R>* W = static_cast<cnum<R>*>(ws);
    const char t1 = trans == 'N' ? 'N' : 'T', t2 = trans == 'N' ? 'T' : 'N';
    ComplexArgs<R> cg{t1, t2, n, n, k, {R(1), R(0)}, reinterpret_cast<const R*>(a), lda, reinterpret_cast<const R*>(a),
                      lda, {R(0), R(0)}, reinterpret_cast<R*>(W), n};
    cg.tri = uplo == 'U' ? 1 : 2;  // the update reads only the stored triangle of W
    if ((e = run_complex(cg, st, FixedScratch{static_cast<char*>(ws) + wbytes, cb})) != cudaSuccess) return e;
    return triangle_update<cnum<R>>(uplo, false, n, alpha, W, n, beta, c, ldc, st, trans == 'C');
}

// Complex TRMM (ztrmm_ / ctrmm_): dense diagonal blocks + complex GEMM couplings.
template <typename R, typename Scratch>
cudaError_t run_trmm(const TrsmArgs<cnum<R>>& t, cudaStream_t st, Scratch scratch) {
    if (t.m <= 0 || t.n <= 0) return cudaSuccess;
    const size_t planes = trmm_plane_bytes<cnum<R>>(t.side, t.m, t.n);
    const int na = (t.side == 'L') ? t.m : t.n;
    const size_t real = complex_scratch_bound<R>(t.m, t.n, na);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return trmm<cnum<R>>(t, ws, gemm_fn_c<R>(st, &fs), st);
}

// Complex SYMM / HEMM (zsymm_ / zhemm_, symmetric.zig:107 with herm): the
// stored triangle mirrored (conjugated for HEMM) into scratch, one complex GEMM.
template <typename R, typename Scratch>
cudaError_t run_symm(char side, char uplo, int m, int n, cnum<R> alpha, const cnum<R>* a, long lda, const cnum<R>* b,
                     long ldb, cnum<R> beta, cnum<R>* c, long ldc, cudaStream_t st, Scratch scratch, bool herm) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    if (alpha == cnum<R>(0)) {
        const R be[2] = {beta.re, beta.im};
        return scale_complex(m, n, be, reinterpret_cast<R*>(c), ldc, st);
    }
    const size_t planes = symm_plane_bytes<cnum<R>>(side, m, n);
    const int na = (side == 'L') ? m : n;
    const size_t real = complex_scratch_bound<R>(m, n, na);
    void* ws = nullptr;
    cudaError_t e = scratch(planes + real, st, &ws);
    if (e != cudaSuccess) return e;
    FixedScratch fs{static_cast<char*>(ws) + planes, real};
    return symm<cnum<R>>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, ws, gemm_fn_c<R>(st, &fs), st, herm);
}

// Complex rank-k / rank-2k updates through one complex GEMM W into scratch and a
// triangle update (symmetric.zig:180-199 / :301-329):
//   SYR2K (herm false, two): W = op(A) op(B)^T, C := alpha (W + W^T) + beta C;
//   HER2K (herm, two):       W = op(A) op(B)^H, C := alpha W + conj(alpha) W^H + beta C;
//   HERK (herm, b == a, not two): W = op(A) op(A)^H, C := alpha W + beta C (alpha, beta real).
// op = C on a symmetric update conjugates W; op = T on a Hermitian one takes the
// conjugate of op = C's W.
template <typename R, typename Scratch>
cudaError_t run_rank2k_c(char uplo, char trans, bool herm, bool two, int n, int k, cnum<R> alpha, const cnum<R>* a,
                         long lda, const cnum<R>* b, long ldb, cnum<R> beta, cnum<R>* c, long ldc, cudaStream_t st,
                         Scratch scratch) {
    if (n <= 0) return cudaSuccess;
    if (k == 0 || alpha == cnum<R>(0)) {
        if (!herm) return syrk_scale_only<cnum<R>>(n, uplo, beta, c, ldc, st);
        // Hermitian: beta C with the diagonal made real (alpha = 0 reads no W)
        return triangle_update_h<cnum<R>>(uplo, false, true, n, cnum<R>(0), cnum<R>(0), c, ldc, beta, c, ldc, st,
                                          false);
    }
    const size_t wbytes = ((size_t)n * n * sizeof(cnum<R>) + 1023) & ~size_t(1023);
    const size_t cb = complex_scratch_bound<R>(n, n, k);
    void* ws = nullptr;
    cudaError_t e = scratch(wbytes + cb, st, &ws);
    if (e != cudaSuccess) return e;
    cnum<R>* W = static_cast<cnum<R>*>(ws);
    char t1, t2;
    bool conj_w;
    if (!herm) {
        t1 = trans == 'N' ? 'N' : 'T', t2 = trans == 'N' ? 'T' : 'N', conj_w = trans == 'C';
    } else {
        t1 = trans == 'N' ? 'N' : 'C', t2 = trans == 'N' ? 'C' : 'N', conj_w = trans == 'T';
    }
    ComplexArgs<R> cg{t1, t2, n, n, k, {R(1), R(0)}, reinterpret_cast<const R*>(a), lda, reinterpret_cast<const R*>(b),
                      ldb, {R(0), R(0)}, reinterpret_cast<R*>(W), n};
    // HERK reads only the stored triangle of W; SYR2K / HER2K also read its transpose
    if (!two) cg.tri = uplo == 'U' ? 1 : 2;
    if ((e = run_complex(cg, st, FixedScratch{static_cast<char*>(ws) + wbytes, cb})) != cudaSuccess) return e;
    const cnum<R> alpha2 = herm ? cnum<R>(alpha.re, -alpha.im) : alpha;
    return triangle_update_h<cnum<R>>(uplo, two, herm, n, alpha, alpha2, W, n, beta, c, ldc, st, conj_w);
}

template <typename T>
void host_trsm(const char* routine, char side, char uplo, char trans, char diag, int m, int n, T alpha, const T* a,
               int lda, T* b, int ldb, bool multiply = false) {
    if (m <= 0 || n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const int na = (side == 'L') ? m : n;
    const size_t es = sizeof(T);
    if ((e = cx.reserve(cx.stage_a, (size_t)na * na * es, st)) != cudaSuccess ||
        (e = cx.reserve(cx.stage_b, (size_t)m * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* db = static_cast<T*>(cx.stage_b.ptr);
    e = cudaMemcpy2DAsync(da, (size_t)na * es, a, (size_t)lda * es, (size_t)na * es, na, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(db, (size_t)m * es, b, (size_t)ldb * es, (size_t)m * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const TrsmArgs<T> t{side, uplo, trans, diag, m, n, alpha, da, na, db, m};
        e = multiply ? run_trmm(t, st, HostScratch{&cx}) : run_trsm(t, st, HostScratch{&cx});
    }
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(b, (size_t)ldb * es, db, (size_t)m * es, (size_t)m * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

template <typename T>
void host_syrk(const char* routine, char uplo, char trans, int n, int k, T alpha, const T* a, int lda, T beta, T* c,
               int ldc) {
    if (n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const int ra = (trans == 'N') ? n : k, ca = (trans == 'N') ? k : n;
    const size_t es = sizeof(T);
    if ((k > 0 && (e = cx.reserve(cx.stage_a, (size_t)ra * ca * es, st)) != cudaSuccess) ||
        (e = cx.reserve(cx.stage_c, (size_t)n * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* dc = static_cast<T*>(cx.stage_c.ptr);
    e = cudaSuccess;
    if (k > 0)
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice,
                              st);
    // C is copied in whole so the other triangle comes back bit-identical
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dc, (size_t)n * es, c, (size_t)ldc * es, (size_t)n * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = run_syrk<T>(uplo, trans, n, k, alpha, da, ra, beta, dc, n, st, HostScratch{&cx});
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)n * es, (size_t)n * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

// SYMM on host arrays: A's na x na window, B and C staged; only C's m x n window comes back.
template <typename T>
void host_symm(const char* routine, char side, char uplo, int m, int n, T alpha, const T* a, int lda, const T* b,
               int ldb, T beta, T* c, int ldc, bool herm = false) {
    if (m <= 0 || n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const int na = (side == 'L') ? m : n;
    const size_t es = sizeof(T);
    if ((e = cx.reserve(cx.stage_a, (size_t)na * na * es, st)) != cudaSuccess ||
        (e = cx.reserve(cx.stage_b, (size_t)m * n * es, st)) != cudaSuccess ||
        (e = cx.reserve(cx.stage_c, (size_t)m * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* db = static_cast<T*>(cx.stage_b.ptr);
    T* dc = static_cast<T*>(cx.stage_c.ptr);
    e = cudaSuccess;
    if (alpha != T(0)) {
        e = cudaMemcpy2DAsync(da, (size_t)na * es, a, (size_t)lda * es, (size_t)na * es, na, cudaMemcpyHostToDevice,
                              st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(db, (size_t)m * es, b, (size_t)ldb * es, (size_t)m * es, n, cudaMemcpyHostToDevice,
                                  st);
    }
    if (e == cudaSuccess && beta != T(0))
        e = cudaMemcpy2DAsync(dc, (size_t)m * es, c, (size_t)ldc * es, (size_t)m * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if constexpr (is_cnum<T>::value)
            e = run_symm(side, uplo, m, n, alpha, da, na, db, m, beta, dc, m, st, HostScratch{&cx}, herm);
        else
            e = run_symm<T>(side, uplo, m, n, alpha, da, na, db, m, beta, dc, m, st, HostScratch{&cx});
    }
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)m * es, (size_t)m * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

// SYR2K on host arrays: C is staged whole so the other triangle comes back bit-identical.
template <typename T>
void host_syr2k(const char* routine, char uplo, char trans, int n, int k, T alpha, const T* a, int lda, const T* b,
                int ldb, T beta, T* c, int ldc, bool herm = false) {
    if (n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const int ra = (trans == 'N') ? n : k, ca = (trans == 'N') ? k : n;
    const size_t es = sizeof(T);
    if ((k > 0 && ((e = cx.reserve(cx.stage_a, (size_t)ra * ca * es, st)) != cudaSuccess ||
                   (e = cx.reserve(cx.stage_b, (size_t)ra * ca * es, st)) != cudaSuccess)) ||
        (e = cx.reserve(cx.stage_c, (size_t)n * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    T* da = static_cast<T*>(cx.stage_a.ptr);
    T* db = static_cast<T*>(cx.stage_b.ptr);
    T* dc = static_cast<T*>(cx.stage_c.ptr);
    e = cudaSuccess;
    if (k > 0) {
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice,
                              st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(db, (size_t)ra * es, b, (size_t)ldb * es, (size_t)ra * es, ca,
                                  cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dc, (size_t)n * es, c, (size_t)ldc * es, (size_t)n * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if constexpr (is_cnum<T>::value)
            e = run_rank2k_c(uplo, trans, herm, true, n, k, alpha, da, ra, db, ra, beta, dc, n, st, HostScratch{&cx});
        else
            e = run_syr2k<T>(uplo, trans, n, k, alpha, da, ra, db, ra, beta, dc, n, st, HostScratch{&cx});
    }
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)n * es, (size_t)n * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

// Complex SYRK on host arrays: C staged whole so the other triangle comes back bit-identical.
template <typename R>
void host_syrk_c(const char* routine, char uplo, char trans, int n, int k, cnum<R> alpha, const cnum<R>* a, int lda,
                 cnum<R> beta, cnum<R>* c, int ldc, bool herm = false) {
    if (n <= 0) return;
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cudaError_t e = cx.init();
    if (e != cudaSuccess) {
        cuda_status(e, "initialisation");
        report_gpu_failure(routine);
        return;
    }
    cudaStream_t st = cx.stream;
    const int ra = (trans == 'N') ? n : k, ca = (trans == 'N') ? k : n;
    const size_t es = sizeof(cnum<R>);
    if ((k > 0 && (e = cx.reserve(cx.stage_a, (size_t)ra * ca * es, st)) != cudaSuccess) ||
        (e = cx.reserve(cx.stage_c, (size_t)n * n * es, st)) != cudaSuccess) {
        cuda_status(e, "staging reservation");
        report_gpu_failure(routine);
        return;
    }
    cnum<R>* da = static_cast<cnum<R>*>(cx.stage_a.ptr);
    cnum<R>* dc = static_cast<cnum<R>*>(cx.stage_c.ptr);
    e = cudaSuccess;
    if (k > 0)
        e = cudaMemcpy2DAsync(da, (size_t)ra * es, a, (size_t)lda * es, (size_t)ra * es, ca, cudaMemcpyHostToDevice,
                              st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dc, (size_t)n * es, c, (size_t)ldc * es, (size_t)n * es, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = herm ? run_rank2k_c<R>(uplo, trans, true, false, n, k, alpha, da, ra, da, ra, beta, dc, n, st,
                                   HostScratch{&cx})
                 : run_syrk_c<R>(uplo, trans, n, k, alpha, da, ra, beta, dc, n, st, HostScratch{&cx});
    if (e == cudaSuccess) e = cx.sync(st);
    if (e != cudaSuccess) {
        cuda_status(e, "GPU execution");
        report_gpu_failure(routine);
        return;
    }
    e = cudaMemcpy2DAsync(c, (size_t)ldc * es, dc, (size_t)n * es, (size_t)n * es, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cuda_status(e, "result copy");
        report_gpu_failure(routine);
    }
}

template <typename R>
int device_syrk_c(const char* what, char uplo, char trans, int n, int k, const R* alpha, const R* a, int lda,
                  const R* beta, R* c, int ldc, void* stream) {
    const char ul = up(&uplo), tr = up(&trans);
    int info = syrk_error(ul, tr, n, k, lda, ldc);
    if (info) return info;
    if (n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(run_syrk_c<R>(ul, tr, n, k, cnum<R>(alpha[0], alpha[1]), reinterpret_cast<const cnum<R>*>(a),
                                     lda, cnum<R>(beta[0], beta[1]), reinterpret_cast<cnum<R>*>(c), ldc,
                                     static_cast<cudaStream_t>(stream), StreamScratch{&cx}),
                       what);
}

template <typename T>
int device_trsm(const char* what, char side, char uplo, char transa, char diag, int m, int n, T alpha, const T* a,
                int lda, T* b, int ldb, void* stream, bool multiply = false) {
    const char sd = up(&side), ul = up(&uplo), tr = up(&transa), dg = up(&diag);
    int info = trsm_error(sd, ul, tr, dg, m, n, lda, ldb);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    const TrsmArgs<T> t{sd, ul, tr, dg, m, n, alpha, a, lda, b, ldb};
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    return cuda_status(multiply ? run_trmm(t, st, StreamScratch{&cx}) : run_trsm(t, st, StreamScratch{&cx}), what);
}

template <typename T>
int device_syrk(const char* what, char uplo, char trans, int n, int k, T alpha, const T* a, int lda, T beta, T* c,
                int ldc, void* stream) {
    const char ul = up(&uplo), tr = up(&trans);
    int info = syrk_error(ul, tr, n, k, lda, ldc);
    if (info) return info;
    if (n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(
        run_syrk<T>(ul, tr, n, k, alpha, a, lda, beta, c, ldc, static_cast<cudaStream_t>(stream), StreamScratch{&cx}),
        what);
}

template <typename T>
int device_symm(const char* what, char side, char uplo, int m, int n, T alpha, const T* a, int lda, const T* b,
                int ldb, T beta, T* c, int ldc, void* stream) {
    const char sd = up(&side), ul = up(&uplo);
    int info = symm_error(sd, ul, m, n, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(run_symm<T>(sd, ul, m, n, alpha, a, lda, b, ldb, beta, c, ldc,
                                   static_cast<cudaStream_t>(stream), StreamScratch{&cx}),
                       what);
}

template <typename T>
int device_syr2k(const char* what, char uplo, char trans, int n, int k, T alpha, const T* a, int lda, const T* b,
                 int ldb, T beta, T* c, int ldc, void* stream) {
    const char ul = up(&uplo), tr = up(&trans);
    int info = syr2k_error(ul, tr, n, k, lda, ldb, ldc);
    if (info) return info;
    if (n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(run_syr2k<T>(ul, tr, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                                    static_cast<cudaStream_t>(stream), StreamScratch{&cx}),
                       what);
}

// Complex SYMM / HEMM on device pointers (run_symm's complex overload).
template <typename R>
int device_symm_c(const char* what, char side, char uplo, int m, int n, cnum<R> alpha, const cnum<R>* a, int lda,
                  const cnum<R>* b, int ldb, cnum<R> beta, cnum<R>* c, int ldc, void* stream, bool herm) {
    const char sd = up(&side), ul = up(&uplo);
    int info = symm_error(sd, ul, m, n, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(run_symm(sd, ul, m, n, alpha, a, lda, b, ldb, beta, c, ldc, static_cast<cudaStream_t>(stream),
                                StreamScratch{&cx}, herm),
                       what);
}

// Complex SYR2K / HER2K (two) and HERK (b == a) on device pointers (run_rank2k_c).
template <typename R>
int device_rank2k_c(const char* what, char uplo, char trans, int n, int k, cnum<R> alpha, const cnum<R>* a, int lda,
                    const cnum<R>* b, int ldb, cnum<R> beta, cnum<R>* c, int ldc, void* stream, bool herm,
                    bool two) {
    const char ul = up(&uplo), tr = up(&trans);
    int info = two ? syr2k_error(ul, tr, n, k, lda, ldb, ldc) : syrk_error(ul, tr, n, k, lda, ldc);
    if (info) return info;
    if (n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    return cuda_status(run_rank2k_c<R>(ul, tr, herm, two, n, k, alpha, a, lda, two ? b : a, two ? ldb : lda, beta, c,
                                       ldc, static_cast<cudaStream_t>(stream), StreamScratch{&cx}),
                       what);
}

inline char cblas_uplo_char(int u) { return u == CblasUpper ? 'U' : (u == CblasLower ? 'L' : 'X'); }
inline char cblas_row_uplo_char(int u) { return u == CblasUpper ? 'L' : (u == CblasLower ? 'U' : 'X'); }
inline char cblas_side_char(int s) { return s == CblasLeft ? 'L' : (s == CblasRight ? 'R' : 'X'); }
inline char cblas_row_side_char(int s) { return s == CblasLeft ? 'R' : (s == CblasRight ? 'L' : 'X'); }
inline char cblas_diag_char(int d) { return d == CblasNonUnit ? 'N' : (d == CblasUnit ? 'U' : 'X'); }
inline char cblas_row_trans_char(int t) {
    return t == CblasNoTrans ? 'T' : (t == CblasTrans ? 'N' : (t == CblasConjTrans ? 'C' : 'X'));
}

inline char cblas_trans_char(int t) {
    switch (t) {
        case CblasNoTrans: return 'N';
        case CblasTrans: return 'T';
        case CblasConjTrans: return 'C';
        default: return 'X';
    }
}
inline bool cblas_valid_layout(int l) { return l == CblasRowMajor || l == CblasColMajor; }
inline bool cblas_valid_trans(int t) { return t == CblasNoTrans || t == CblasTrans || t == CblasConjTrans; }

}  // namespace

int zb::gemm_arg_error(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc) {
    return gemm_error(ta, tb, m, n, k, lda, ldb, ldc);
}

extern "C" {

int lsame_(const char* ca, const char* cb) {
    return std::toupper((unsigned char)ca[0]) == std::toupper((unsigned char)cb[0]) ? 1 : 0;
}

void xerbla_(const char* srname, const zynum_blas_int* info) { report_xerbla(srname, *info); }

void zynum_blas_shutdown(void) { context().shutdown(); }
void zynum_blas_shutdown_(void) { context().shutdown(); }

void sgemm_(const char* transa, const char* transb, const zynum_blas_int* m, const zynum_blas_int* n,
            const zynum_blas_int* k, const float* alpha, const float* a, const zynum_blas_int* lda, const float* b,
            const zynum_blas_int* ldb, const float* beta, float* c, const zynum_blas_int* ldc) {
    const char ta = up(transa), tb = up(transb);
    int info = gemm_error(ta, tb, *m, *n, *k, *lda, *ldb, *ldc);
    if (info) {
        report_xerbla("SGEMM ", info);
        return;
    }
    host_gemm<float>("SGEMM", ta, tb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

void dgemm_(const char* transa, const char* transb, const zynum_blas_int* m, const zynum_blas_int* n,
            const zynum_blas_int* k, const double* alpha, const double* a, const zynum_blas_int* lda,
            const double* b, const zynum_blas_int* ldb, const double* beta, double* c, const zynum_blas_int* ldc) {
    const char ta = up(transa), tb = up(transb);
    int info = gemm_error(ta, tb, *m, *n, *k, *lda, *ldb, *ldc);
    if (info) {
        report_xerbla("DGEMM ", info);
        return;
    }
    host_gemm<double>("DGEMM", ta, tb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

// cblas.zig:1415-1439: silent return on a bad enum; row-major C = A B is
// computed as column-major C^T = B^T A^T by swapping the operands.
void cblas_sgemm(int layout, int transa, int transb, int m, int n, int k, float alpha, const float* a, int lda,
                 const float* b, int ldb, float beta, float* c, int ldc) {
    if (!cblas_valid_layout(layout) || !cblas_valid_trans(transa) || !cblas_valid_trans(transb)) return;
    const bool rm = layout == CblasRowMajor;
    char ta = cblas_trans_char(rm ? transb : transa), tb = cblas_trans_char(rm ? transa : transb);
    zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, kk = k, la = rm ? ldb : lda, lb = rm ? lda : ldb, lc = ldc;
    if (rm)
        sgemm_(&ta, &tb, &mm, &nn, &kk, &alpha, b, &la, a, &lb, &beta, c, &lc);
    else
        sgemm_(&ta, &tb, &mm, &nn, &kk, &alpha, a, &la, b, &lb, &beta, c, &lc);
}

void cblas_dgemm(int layout, int transa, int transb, int m, int n, int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* c, int ldc) {
    if (!cblas_valid_layout(layout) || !cblas_valid_trans(transa) || !cblas_valid_trans(transb)) return;
    const bool rm = layout == CblasRowMajor;
    char ta = cblas_trans_char(rm ? transb : transa), tb = cblas_trans_char(rm ? transa : transb);
    zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, kk = k, la = rm ? ldb : lda, lb = rm ? lda : ldb, lc = ldc;
    if (rm)
        dgemm_(&ta, &tb, &mm, &nn, &kk, &alpha, b, &la, a, &lb, &beta, c, &lc);
    else
        dgemm_(&ta, &tb, &mm, &nn, &kk, &alpha, a, &la, b, &lb, &beta, c, &lc);
}

void cgemm_(const char* transa, const char* transb, const zynum_blas_int* m, const zynum_blas_int* n,
            const zynum_blas_int* k, const void* alpha, const void* a, const zynum_blas_int* lda, const void* b,
            const zynum_blas_int* ldb, const void* beta, void* c, const zynum_blas_int* ldc) {
    const char ta = up(transa), tb = up(transb);
    int info = gemm_error(ta, tb, *m, *n, *k, *lda, *ldb, *ldc);
    if (info) {
        report_xerbla("CGEMM ", info);
        return;
    }
    host_complex_gemm<float>("CGEMM", ta, tb, *m, *n, *k, static_cast<const float*>(alpha),
                             static_cast<const float*>(a), *lda, static_cast<const float*>(b), *ldb,
                             static_cast<const float*>(beta), static_cast<float*>(c), *ldc);
}

void zgemm_(const char* transa, const char* transb, const zynum_blas_int* m, const zynum_blas_int* n,
            const zynum_blas_int* k, const void* alpha, const void* a, const zynum_blas_int* lda, const void* b,
            const zynum_blas_int* ldb, const void* beta, void* c, const zynum_blas_int* ldc) {
    const char ta = up(transa), tb = up(transb);
    int info = gemm_error(ta, tb, *m, *n, *k, *lda, *ldb, *ldc);
    if (info) {
        report_xerbla("ZGEMM ", info);
        return;
    }
    host_complex_gemm<double>("ZGEMM", ta, tb, *m, *n, *k, static_cast<const double*>(alpha),
                              static_cast<const double*>(a), *lda, static_cast<const double*>(b), *ldb,
                              static_cast<const double*>(beta), static_cast<double*>(c), *ldc);
}

// cblas.zig:1441-1465: complex alpha / beta by pointer, same row-major swap.
void cblas_cgemm(int layout, int transa, int transb, int m, int n, int k, const void* alpha, const void* a, int lda,
                 const void* b, int ldb, const void* beta, void* c, int ldc) {
    if (!cblas_valid_layout(layout) || !cblas_valid_trans(transa) || !cblas_valid_trans(transb)) return;
    const bool rm = layout == CblasRowMajor;
    char ta = cblas_trans_char(rm ? transb : transa), tb = cblas_trans_char(rm ? transa : transb);
    zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, kk = k, la = rm ? ldb : lda, lb = rm ? lda : ldb, lc = ldc;
    if (rm)
        cgemm_(&ta, &tb, &mm, &nn, &kk, alpha, b, &la, a, &lb, beta, c, &lc);
    else
        cgemm_(&ta, &tb, &mm, &nn, &kk, alpha, a, &la, b, &lb, beta, c, &lc);
}

void cblas_zgemm(int layout, int transa, int transb, int m, int n, int k, const void* alpha, const void* a, int lda,
                 const void* b, int ldb, const void* beta, void* c, int ldc) {
    if (!cblas_valid_layout(layout) || !cblas_valid_trans(transa) || !cblas_valid_trans(transb)) return;
    const bool rm = layout == CblasRowMajor;
    char ta = cblas_trans_char(rm ? transb : transa), tb = cblas_trans_char(rm ? transa : transb);
    zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, kk = k, la = rm ? ldb : lda, lb = rm ? lda : ldb, lc = ldc;
    if (rm)
        zgemm_(&ta, &tb, &mm, &nn, &kk, alpha, b, &la, a, &lb, beta, c, &lc);
    else
        zgemm_(&ta, &tb, &mm, &nn, &kk, alpha, a, &la, b, &lb, beta, c, &lc);
}

int zynum_blas_gpu_zgemm_device(char transa, char transb, int m, int n, int k, const double* alpha, const double* a,
                                int lda, const double* b, int ldb, const double* beta, double* c, int ldc,
                                void* stream) {
    return device_complex_gemm<double>("zgemm_device", transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                                       stream);
}

int zynum_blas_gpu_cgemm_device(char transa, char transb, int m, int n, int k, const float* alpha, const float* a,
                                int lda, const float* b, int ldb, const float* beta, float* c, int ldc, void* stream) {
    return device_complex_gemm<float>("cgemm_device", transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                                      stream);
}

int zynum_blas_gpu_set_complex_method(int method) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.complex_method;
    if (method == COMPLEX_4M || method == COMPLEX_3M) cx.complex_method = method;
    return old;
}

// fortran.zig:869-883 ?trsm_, :802-816 ?syrk_
#define ZB_TRSM(NAME, T, RNAME)                                                                                    \
    void NAME(const char* side, const char* uplo, const char* transa, const char* diag, const zynum_blas_int* m,  \
              const zynum_blas_int* n, const T* alpha, const T* a, const zynum_blas_int* lda, T* b,               \
              const zynum_blas_int* ldb) {                                                                        \
        const char sd = up(side), ul = up(uplo), tr = up(transa), dg = up(diag);                                   \
        int info = trsm_error(sd, ul, tr, dg, *m, *n, *lda, *ldb);                                                 \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        host_trsm<T>(RNAME, sd, ul, tr, dg, *m, *n, *alpha, a, *lda, b, *ldb);                                     \
    }
ZB_TRSM(dtrsm_, double, "DTRSM ")
ZB_TRSM(strsm_, float, "STRSM ")
#undef ZB_TRSM

#define ZB_SYRK(NAME, T, RNAME)                                                                                     \
    void NAME(const char* uplo, const char* trans, const zynum_blas_int* n, const zynum_blas_int* k, const T* alpha, \
              const T* a, const zynum_blas_int* lda, const T* beta, T* c, const zynum_blas_int* ldc) {             \
        const char ul = up(uplo), tr = up(trans);                                                                   \
        int info = syrk_error(ul, tr, *n, *k, *lda, *ldc);                                                          \
        if (info) {                                                                                                 \
            report_xerbla(RNAME, info);                                                                             \
            return;                                                                                                 \
        }                                                                                                           \
        host_syrk<T>(RNAME, ul, tr, *n, *k, *alpha, a, *lda, *beta, c, *ldc);                                       \
    }
ZB_SYRK(dsyrk_, double, "DSYRK ")
ZB_SYRK(ssyrk_, float, "SSYRK ")
#undef ZB_SYRK

// cblas.zig:1729-1756 cblas_?trsm: invalid enums return silently; row-major
// flips side and uplo and swaps m / n, keeping the transpose.
#define ZB_CBLAS_TRSM(NAME, FNAME, T)                                                                            \
    void NAME(int layout, int side, int uplo, int transa, int diag, int m, int n, T alpha, const T* a, int lda, \
              T* b, int ldb) {                                                                                   \
        if (!cblas_valid_layout(layout) || (side != CblasLeft && side != CblasRight) ||                          \
            (uplo != CblasUpper && uplo != CblasLower) || !cblas_valid_trans(transa) ||                          \
            (diag != CblasNonUnit && diag != CblasUnit))                                                         \
            return;                                                                                              \
        const bool rm = layout == CblasRowMajor;                                                                 \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                        \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                        \
        char tt = cblas_trans_char(transa), dd = cblas_diag_char(diag);                                          \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb;                                     \
        FNAME(&ss, &uu, &tt, &dd, &mm, &nn, &alpha, a, &la, b, &lb);                                             \
    }
ZB_CBLAS_TRSM(cblas_dtrsm, dtrsm_, double)
ZB_CBLAS_TRSM(cblas_strsm, strsm_, float)
#undef ZB_CBLAS_TRSM

// cblas.zig:1539-1560 cblas_?syrk: only the layout is checked here; a bad
// uplo / trans reaches the Fortran routine as 'X' and is reported by xerbla.
#define ZB_CBLAS_SYRK(NAME, FNAME, T)                                                                              \
    void NAME(int layout, int uplo, int trans, int n, int k, T alpha, const T* a, int lda, T beta, T* c, int ldc) { \
        if (!cblas_valid_layout(layout)) return;                                                                   \
        const bool rm = layout == CblasRowMajor;                                                                   \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                          \
        char tt = rm ? cblas_row_trans_char(trans) : cblas_trans_char(trans);                                      \
        zynum_blas_int nn = n, kk = k, la = lda, lc = ldc;                                                         \
        FNAME(&uu, &tt, &nn, &kk, &alpha, a, &la, &beta, c, &lc);                                                  \
    }
ZB_CBLAS_SYRK(cblas_dsyrk, dsyrk_, double)
ZB_CBLAS_SYRK(cblas_ssyrk, ssyrk_, float)
#undef ZB_CBLAS_SYRK

int zynum_blas_gpu_dtrsm_device(char side, char uplo, char transa, char diag, int m, int n, double alpha,
                                const double* a, int lda, double* b, int ldb, void* stream) {
    return device_trsm<double>("dtrsm_device", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream);
}
int zynum_blas_gpu_strsm_device(char side, char uplo, char transa, char diag, int m, int n, float alpha,
                                const float* a, int lda, float* b, int ldb, void* stream) {
    return device_trsm<float>("strsm_device", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream);
}

size_t zynum_blas_gpu_dtrsm_inverse_bytes(int n) { return trsm_leaf_inverse_bytes(n); }

int zynum_blas_gpu_dtrsm_inverse_device(char uplo, char diag, int n, const double* a, int lda, double* inv,
                                        void* stream) {
    const char ul = up(&uplo), dg = up(&diag);
    if (!valid_uplo(ul)) return 1;
    if (!valid_diag(dg)) return 2;
    if (n < 0) return 3;
    if (lda < max1(n)) return 5;
    if (n == 0) return 0;
    if (!inv) return 6;
    if (reinterpret_cast<uintptr_t>(a) % 16 != 0 || lda % 2 != 0) {
        set_last_error("dtrsm_inverse_device: A must be 16-byte aligned with an even lda");
        return -(int)cudaErrorInvalidValue;
    }
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    void* ws = nullptr;
    if ((e = cx.stream_scratch(st, trsm_leaf_inverse_scratch_bytes(n), &ws)) != cudaSuccess)
        return cuda_status(e, "dtrsm_inverse_device");
    return cuda_status(trsm_leaf_inverses(ul, dg, n, a, lda, ws, inv, st), "dtrsm_inverse_device");
}

int zynum_blas_gpu_dtrsm_with_inverse_device(char side, char uplo, char transa, char diag, int m, int n, double alpha,
                                             const double* a, int lda, double* b, int ldb, const double* inv,
                                             void* stream) {
    const char sd = up(&side), ul = up(&uplo), tr = up(&transa), dg = up(&diag);
    int info = trsm_error(sd, ul, tr, dg, m, n, lda, ldb);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    if (!inv) return 12;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    const TrsmArgs<double> t{sd, ul, tr, dg, m, n, alpha, a, lda, b, ldb};
    const TrsmInverses given{inv, tr != 'N'};
    return cuda_status(run_trsm(t, static_cast<cudaStream_t>(stream), StreamScratch{&cx}, &given),
                       "dtrsm_with_inverse_device");
}
int zynum_blas_gpu_dsyrk_device(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
                                double beta, double* c, int ldc, void* stream) {
    return device_syrk<double>("dsyrk_device", uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream);
}
int zynum_blas_gpu_ssyrk_device(char uplo, char trans, int n, int k, float alpha, const float* a, int lda, float beta,
                                float* c, int ldc, void* stream) {
    return device_syrk<float>("ssyrk_device", uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream);
}

// fortran.zig:877-884 ctrsm_ / ztrsm_, :810-817 csyrk_ / zsyrk_ (interleaved complex, alpha / beta by pointer)
#define ZB_TRSM_C(NAME, R, RNAME)                                                                                  \
    void NAME(const char* side, const char* uplo, const char* transa, const char* diag, const zynum_blas_int* m,  \
              const zynum_blas_int* n, const void* alpha, const void* a, const zynum_blas_int* lda, void* b,      \
              const zynum_blas_int* ldb) {                                                                        \
        const char sd = up(side), ul = up(uplo), tr = up(transa), dg = up(diag);                                   \
        int info = trsm_error(sd, ul, tr, dg, *m, *n, *lda, *ldb);                                                 \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        const R* al = static_cast<const R*>(alpha);                                                                \
        host_trsm<cnum<R>>(RNAME, sd, ul, tr, dg, *m, *n, cnum<R>(al[0], al[1]), static_cast<const cnum<R>*>(a),  \
                           *lda, static_cast<cnum<R>*>(b), *ldb);                                                  \
    }
ZB_TRSM_C(ztrsm_, double, "ZTRSM ")
ZB_TRSM_C(ctrsm_, float, "CTRSM ")
#undef ZB_TRSM_C

#define ZB_SYRK_C(NAME, R, RNAME)                                                                                  \
    void NAME(const char* uplo, const char* trans, const zynum_blas_int* n, const zynum_blas_int* k,              \
              const void* alpha, const void* a, const zynum_blas_int* lda, const void* beta, void* c,             \
              const zynum_blas_int* ldc) {                                                                        \
        const char ul = up(uplo), tr = up(trans);                                                                  \
        int info = syrk_error(ul, tr, *n, *k, *lda, *ldc);                                                         \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        const R* al = static_cast<const R*>(alpha);                                                                \
        const R* be = static_cast<const R*>(beta);                                                                 \
        host_syrk_c<R>(RNAME, ul, tr, *n, *k, cnum<R>(al[0], al[1]), static_cast<const cnum<R>*>(a), *lda,         \
                       cnum<R>(be[0], be[1]), static_cast<cnum<R>*>(c), *ldc);                                     \
    }
ZB_SYRK_C(zsyrk_, double, "ZSYRK ")
ZB_SYRK_C(csyrk_, float, "CSYRK ")
#undef ZB_SYRK_C

// cblas.zig:1755-1779 cblas_ctrsm / cblas_ztrsm (enums checked, silent return) and :1560-1582
// cblas_csyrk / cblas_zsyrk (layout only)
#define ZB_CBLAS_TRSM_C(NAME, FNAME)                                                                                \
    void NAME(int layout, int side, int uplo, int transa, int diag, int m, int n, const void* alpha, const void* a, \
              int lda, void* b, int ldb) {                                                                          \
        if (!cblas_valid_layout(layout) || (side != CblasLeft && side != CblasRight) ||                             \
            (uplo != CblasUpper && uplo != CblasLower) || !cblas_valid_trans(transa) ||                             \
            (diag != CblasNonUnit && diag != CblasUnit))                                                            \
            return;                                                                                                 \
        const bool rm = layout == CblasRowMajor;                                                                    \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                           \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                           \
        char tt = cblas_trans_char(transa), dd = cblas_diag_char(diag);                                             \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb;                                        \
        FNAME(&ss, &uu, &tt, &dd, &mm, &nn, alpha, a, &la, b, &lb);                                                 \
    }
ZB_CBLAS_TRSM_C(cblas_ztrsm, ztrsm_)
ZB_CBLAS_TRSM_C(cblas_ctrsm, ctrsm_)
#undef ZB_CBLAS_TRSM_C

#define ZB_CBLAS_SYRK_C(NAME, FNAME)                                                                            \
    void NAME(int layout, int uplo, int trans, int n, int k, const void* alpha, const void* a, int lda,        \
              const void* beta, void* c, int ldc) {                                                             \
        if (!cblas_valid_layout(layout)) return;                                                                \
        const bool rm = layout == CblasRowMajor;                                                                \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                       \
        char tt = rm ? cblas_row_trans_char(trans) : cblas_trans_char(trans);                                   \
        zynum_blas_int nn = n, kk = k, la = lda, lc = ldc;                                                      \
        FNAME(&uu, &tt, &nn, &kk, alpha, a, &la, beta, c, &lc);                                                 \
    }
ZB_CBLAS_SYRK_C(cblas_zsyrk, zsyrk_)
ZB_CBLAS_SYRK_C(cblas_csyrk, csyrk_)
#undef ZB_CBLAS_SYRK_C

int zynum_blas_gpu_ztrsm_device(char side, char uplo, char transa, char diag, int m, int n, const double* alpha,
                                const double* a, int lda, double* b, int ldb, void* stream) {
    return device_trsm<cnum<double>>("ztrsm_device", side, uplo, transa, diag, m, n, cnum<double>(alpha[0], alpha[1]),
                                     reinterpret_cast<const cnum<double>*>(a), lda, reinterpret_cast<cnum<double>*>(b),
                                     ldb, stream);
}
int zynum_blas_gpu_ctrsm_device(char side, char uplo, char transa, char diag, int m, int n, const float* alpha,
                                const float* a, int lda, float* b, int ldb, void* stream) {
    return device_trsm<cnum<float>>("ctrsm_device", side, uplo, transa, diag, m, n, cnum<float>(alpha[0], alpha[1]),
                                    reinterpret_cast<const cnum<float>*>(a), lda, reinterpret_cast<cnum<float>*>(b),
                                    ldb, stream);
}
int zynum_blas_gpu_zsyrk_device(char uplo, char trans, int n, int k, const double* alpha, const double* a, int lda,
                                const double* beta, double* c, int ldc, void* stream) {
    return device_syrk_c<double>("zsyrk_device", uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream);
}
int zynum_blas_gpu_csyrk_device(char uplo, char trans, int n, int k, const float* alpha, const float* a, int lda,
                                const float* beta, float* c, int ldc, void* stream) {
    return device_syrk_c<float>("csyrk_device", uplo, trans, n, k, alpha, a, lda, beta, c, ldc, stream);
}

// fortran.zig:785-799 csymm_ / zsymm_ / chemm_ / zhemm_, :860-867 ctrmm_ / ztrmm_,
// :835-849 csyr2k_ / zsyr2k_ / cher2k_ / zher2k_ (beta real), :818-825 cherk_ / zherk_ (alpha, beta real)
#define ZB_SYMM_C(NAME, R, RNAME, HERM)                                                                          \
    void NAME(const char* side, const char* uplo, const zynum_blas_int* m, const zynum_blas_int* n,             \
              const void* alpha, const void* a, const zynum_blas_int* lda, const void* b,                       \
              const zynum_blas_int* ldb, const void* beta, void* c, const zynum_blas_int* ldc) {                \
        const char sd = up(side), ul = up(uplo);                                                                 \
        int info = symm_error(sd, ul, *m, *n, *lda, *ldb, *ldc);                                                 \
        if (info) {                                                                                              \
            report_xerbla(RNAME, info);                                                                          \
            return;                                                                                              \
        }                                                                                                        \
        const R* al = static_cast<const R*>(alpha);                                                              \
        const R* be = static_cast<const R*>(beta);                                                               \
        host_symm<cnum<R>>(RNAME, sd, ul, *m, *n, cnum<R>(al[0], al[1]), static_cast<const cnum<R>*>(a), *lda,  \
                           static_cast<const cnum<R>*>(b), *ldb, cnum<R>(be[0], be[1]), static_cast<cnum<R>*>(c), \
                           *ldc, HERM);                                                                          \
    }
ZB_SYMM_C(zsymm_, double, "ZSYMM ", false)
ZB_SYMM_C(csymm_, float, "CSYMM ", false)
ZB_SYMM_C(zhemm_, double, "ZHEMM ", true)
ZB_SYMM_C(chemm_, float, "CHEMM ", true)
#undef ZB_SYMM_C

#define ZB_TRMM_C(NAME, R, RNAME)                                                                                  \
    void NAME(const char* side, const char* uplo, const char* transa, const char* diag, const zynum_blas_int* m,  \
              const zynum_blas_int* n, const void* alpha, const void* a, const zynum_blas_int* lda, void* b,      \
              const zynum_blas_int* ldb) {                                                                        \
        const char sd = up(side), ul = up(uplo), tr = up(transa), dg = up(diag);                                   \
        int info = trsm_error(sd, ul, tr, dg, *m, *n, *lda, *ldb);                                                 \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        const R* al = static_cast<const R*>(alpha);                                                                \
        host_trsm<cnum<R>>(RNAME, sd, ul, tr, dg, *m, *n, cnum<R>(al[0], al[1]), static_cast<const cnum<R>*>(a),  \
                           *lda, static_cast<cnum<R>*>(b), *ldb, true);                                            \
    }
ZB_TRMM_C(ztrmm_, double, "ZTRMM ")
ZB_TRMM_C(ctrmm_, float, "CTRMM ")
#undef ZB_TRMM_C

// BETA_T: const void* (symmetric, complex beta) or const R* (Hermitian, real beta)
#define ZB_SYR2K_C(NAME, R, RNAME, HERM, BETA_T, BETA_EXPR)                                                      \
    void NAME(const char* uplo, const char* trans, const zynum_blas_int* n, const zynum_blas_int* k,            \
              const void* alpha, const void* a, const zynum_blas_int* lda, const void* b,                       \
              const zynum_blas_int* ldb, BETA_T beta, void* c, const zynum_blas_int* ldc) {                     \
        const char ul = up(uplo), tr = up(trans);                                                                \
        int info = syr2k_error(ul, tr, *n, *k, *lda, *ldb, *ldc);                                                \
        if (info) {                                                                                              \
            report_xerbla(RNAME, info);                                                                          \
            return;                                                                                              \
        }                                                                                                        \
        const R* al = static_cast<const R*>(alpha);                                                              \
        host_syr2k<cnum<R>>(RNAME, ul, tr, *n, *k, cnum<R>(al[0], al[1]), static_cast<const cnum<R>*>(a), *lda, \
                            static_cast<const cnum<R>*>(b), *ldb, BETA_EXPR, static_cast<cnum<R>*>(c), *ldc,     \
                            HERM);                                                                               \
    }
ZB_SYR2K_C(zsyr2k_, double, "ZSYR2K", false, const void*,
           cnum<double>(static_cast<const double*>(beta)[0], static_cast<const double*>(beta)[1]))
ZB_SYR2K_C(csyr2k_, float, "CSYR2K", false, const void*,
           cnum<float>(static_cast<const float*>(beta)[0], static_cast<const float*>(beta)[1]))
ZB_SYR2K_C(zher2k_, double, "ZHER2K", true, const double*, cnum<double>(*beta))
ZB_SYR2K_C(cher2k_, float, "CHER2K", true, const float*, cnum<float>(*beta))
#undef ZB_SYR2K_C

#define ZB_HERK(NAME, R, RNAME)                                                                                    \
    void NAME(const char* uplo, const char* trans, const zynum_blas_int* n, const zynum_blas_int* k, const R* alpha, \
              const void* a, const zynum_blas_int* lda, const R* beta, void* c, const zynum_blas_int* ldc) {       \
        const char ul = up(uplo), tr = up(trans);                                                                   \
        int info = syrk_error(ul, tr, *n, *k, *lda, *ldc);                                                          \
        if (info) {                                                                                                 \
            report_xerbla(RNAME, info);                                                                             \
            return;                                                                                                 \
        }                                                                                                           \
        host_syrk_c<R>(RNAME, ul, tr, *n, *k, cnum<R>(*alpha), static_cast<const cnum<R>*>(a), *lda,               \
                       cnum<R>(*beta), static_cast<cnum<R>*>(c), *ldc, true);                                       \
    }
ZB_HERK(zherk_, double, "ZHERK ")
ZB_HERK(cherk_, float, "CHERK ")
#undef ZB_HERK

// cblas.zig:1491-1537 cblas_[cz]symm / cblas_[cz]hemm, :1703-1728 cblas_[cz]trmm,
// :1629-1676 cblas_[cz]syr2k / cblas_[cz]her2k (beta real), :1583-1603 cblas_[cz]herk (alpha, beta real)
#define ZB_CBLAS_SYMM_C(NAME, FNAME)                                                                              \
    void NAME(int layout, int side, int uplo, int m, int n, const void* alpha, const void* a, int lda,            \
              const void* b, int ldb, const void* beta, void* c, int ldc) {                                       \
        if (!cblas_valid_layout(layout)) return;                                                                  \
        const bool rm = layout == CblasRowMajor;                                                                  \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                         \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                         \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb, lc = ldc;                            \
        FNAME(&ss, &uu, &mm, &nn, alpha, a, &la, b, &lb, beta, c, &lc);                                           \
    }
ZB_CBLAS_SYMM_C(cblas_zsymm, zsymm_)
ZB_CBLAS_SYMM_C(cblas_csymm, csymm_)
ZB_CBLAS_SYMM_C(cblas_zhemm, zhemm_)
ZB_CBLAS_SYMM_C(cblas_chemm, chemm_)
#undef ZB_CBLAS_SYMM_C

#define ZB_CBLAS_TRMM_C(NAME, FNAME)                                                                                \
    void NAME(int layout, int side, int uplo, int transa, int diag, int m, int n, const void* alpha, const void* a, \
              int lda, void* b, int ldb) {                                                                          \
        if (!cblas_valid_layout(layout) || (side != CblasLeft && side != CblasRight) ||                             \
            (uplo != CblasUpper && uplo != CblasLower) || !cblas_valid_trans(transa) ||                             \
            (diag != CblasNonUnit && diag != CblasUnit))                                                            \
            return;                                                                                                 \
        const bool rm = layout == CblasRowMajor;                                                                    \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                           \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                           \
        char tt = cblas_trans_char(transa), dd = cblas_diag_char(diag);                                             \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb;                                        \
        FNAME(&ss, &uu, &tt, &dd, &mm, &nn, alpha, a, &la, b, &lb);                                                 \
    }
ZB_CBLAS_TRMM_C(cblas_ztrmm, ztrmm_)
ZB_CBLAS_TRMM_C(cblas_ctrmm, ctrmm_)
#undef ZB_CBLAS_TRMM_C

#define ZB_CBLAS_SYR2K_C(NAME, FNAME, BETA_T, BETA_ARG)                                                            \
    void NAME(int layout, int uplo, int trans, int n, int k, const void* alpha, const void* a, int lda,           \
              const void* b, int ldb, BETA_T beta, void* c, int ldc) {                                            \
        if (!cblas_valid_layout(layout)) return;                                                                  \
        const bool rm = layout == CblasRowMajor;                                                                  \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                         \
        char tt = rm ? cblas_row_trans_char(trans) : cblas_trans_char(trans);                                     \
        zynum_blas_int nn = n, kk = k, la = lda, lb = ldb, lc = ldc;                                              \
        FNAME(&uu, &tt, &nn, &kk, alpha, a, &la, b, &lb, BETA_ARG, c, &lc);                                       \
    }
ZB_CBLAS_SYR2K_C(cblas_zsyr2k, zsyr2k_, const void*, beta)
ZB_CBLAS_SYR2K_C(cblas_csyr2k, csyr2k_, const void*, beta)
ZB_CBLAS_SYR2K_C(cblas_zher2k, zher2k_, double, &beta)
ZB_CBLAS_SYR2K_C(cblas_cher2k, cher2k_, float, &beta)
#undef ZB_CBLAS_SYR2K_C

#define ZB_CBLAS_HERK(NAME, FNAME, R)                                                                        \
    void NAME(int layout, int uplo, int trans, int n, int k, R alpha, const void* a, int lda, R beta, void* c, \
              int ldc) {                                                                                     \
        if (!cblas_valid_layout(layout)) return;                                                             \
        const bool rm = layout == CblasRowMajor;                                                             \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                    \
        char tt = rm ? cblas_row_trans_char(trans) : cblas_trans_char(trans);                                \
        zynum_blas_int nn = n, kk = k, la = lda, lc = ldc;                                                   \
        FNAME(&uu, &tt, &nn, &kk, &alpha, a, &la, &beta, c, &lc);                                            \
    }
ZB_CBLAS_HERK(cblas_zherk, zherk_, double)
ZB_CBLAS_HERK(cblas_cherk, cherk_, float)
#undef ZB_CBLAS_HERK

// fortran.zig:777-783 ?symm_, :852-858 ?trmm_, :827-833 ?syr2k_
#define ZB_SYMM(NAME, T, RNAME)                                                                                   \
    void NAME(const char* side, const char* uplo, const zynum_blas_int* m, const zynum_blas_int* n, const T* alpha, \
              const T* a, const zynum_blas_int* lda, const T* b, const zynum_blas_int* ldb, const T* beta, T* c,   \
              const zynum_blas_int* ldc) {                                                                         \
        const char sd = up(side), ul = up(uplo);                                                                   \
        int info = symm_error(sd, ul, *m, *n, *lda, *ldb, *ldc);                                                   \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        host_symm<T>(RNAME, sd, ul, *m, *n, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                            \
    }
ZB_SYMM(dsymm_, double, "DSYMM ")
ZB_SYMM(ssymm_, float, "SSYMM ")
#undef ZB_SYMM

#define ZB_TRMM(NAME, T, RNAME)                                                                                    \
    void NAME(const char* side, const char* uplo, const char* transa, const char* diag, const zynum_blas_int* m,  \
              const zynum_blas_int* n, const T* alpha, const T* a, const zynum_blas_int* lda, T* b,               \
              const zynum_blas_int* ldb) {                                                                        \
        const char sd = up(side), ul = up(uplo), tr = up(transa), dg = up(diag);                                   \
        int info = trsm_error(sd, ul, tr, dg, *m, *n, *lda, *ldb);                                                 \
        if (info) {                                                                                                \
            report_xerbla(RNAME, info);                                                                            \
            return;                                                                                                \
        }                                                                                                          \
        host_trsm<T>(RNAME, sd, ul, tr, dg, *m, *n, *alpha, a, *lda, b, *ldb, true);                               \
    }
ZB_TRMM(dtrmm_, double, "DTRMM ")
ZB_TRMM(strmm_, float, "STRMM ")
#undef ZB_TRMM

#define ZB_SYR2K(NAME, T, RNAME)                                                                                    \
    void NAME(const char* uplo, const char* trans, const zynum_blas_int* n, const zynum_blas_int* k, const T* alpha, \
              const T* a, const zynum_blas_int* lda, const T* b, const zynum_blas_int* ldb, const T* beta, T* c,    \
              const zynum_blas_int* ldc) {                                                                          \
        const char ul = up(uplo), tr = up(trans);                                                                   \
        int info = syr2k_error(ul, tr, *n, *k, *lda, *ldb, *ldc);                                                   \
        if (info) {                                                                                                 \
            report_xerbla(RNAME, info);                                                                             \
            return;                                                                                                 \
        }                                                                                                           \
        host_syr2k<T>(RNAME, ul, tr, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                             \
    }
ZB_SYR2K(dsyr2k_, double, "DSYR2K")
ZB_SYR2K(ssyr2k_, float, "SSYR2K")
#undef ZB_SYR2K

// cblas.zig:1479-1489 cblas_?symm: only the layout is checked here (a bad side
// or uplo reaches the Fortran routine as 'X' and is reported by xerbla);
// row-major flips side and uplo and swaps m / n.
#define ZB_CBLAS_SYMM(NAME, FNAME, T)                                                                         \
    void NAME(int layout, int side, int uplo, int m, int n, T alpha, const T* a, int lda, const T* b, int ldb, \
              T beta, T* c, int ldc) {                                                                        \
        if (!cblas_valid_layout(layout)) return;                                                              \
        const bool rm = layout == CblasRowMajor;                                                              \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                     \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                     \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb, lc = ldc;                        \
        FNAME(&ss, &uu, &mm, &nn, &alpha, a, &la, b, &lb, &beta, c, &lc);                                     \
    }
ZB_CBLAS_SYMM(cblas_dsymm, dsymm_, double)
ZB_CBLAS_SYMM(cblas_ssymm, ssymm_, float)
#undef ZB_CBLAS_SYMM

// cblas.zig:1690-1701 cblas_?trmm: invalid enums return silently; row-major
// flips side and uplo and swaps m / n, keeping the transpose.
#define ZB_CBLAS_TRMM(NAME, FNAME, T)                                                                            \
    void NAME(int layout, int side, int uplo, int transa, int diag, int m, int n, T alpha, const T* a, int lda, \
              T* b, int ldb) {                                                                                   \
        if (!cblas_valid_layout(layout) || (side != CblasLeft && side != CblasRight) ||                          \
            (uplo != CblasUpper && uplo != CblasLower) || !cblas_valid_trans(transa) ||                          \
            (diag != CblasNonUnit && diag != CblasUnit))                                                         \
            return;                                                                                              \
        const bool rm = layout == CblasRowMajor;                                                                 \
        char ss = rm ? cblas_row_side_char(side) : cblas_side_char(side);                                        \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                        \
        char tt = cblas_trans_char(transa), dd = cblas_diag_char(diag);                                          \
        zynum_blas_int mm = rm ? n : m, nn = rm ? m : n, la = lda, lb = ldb;                                     \
        FNAME(&ss, &uu, &tt, &dd, &mm, &nn, &alpha, a, &la, b, &lb);                                             \
    }
ZB_CBLAS_TRMM(cblas_dtrmm, dtrmm_, double)
ZB_CBLAS_TRMM(cblas_strmm, strmm_, float)
#undef ZB_CBLAS_TRMM

// cblas.zig:1617-1627 cblas_?syr2k: only the layout is checked here; row-major
// flips uplo and the transpose.
#define ZB_CBLAS_SYR2K(NAME, FNAME, T)                                                                            \
    void NAME(int layout, int uplo, int trans, int n, int k, T alpha, const T* a, int lda, const T* b, int ldb,  \
              T beta, T* c, int ldc) {                                                                           \
        if (!cblas_valid_layout(layout)) return;                                                                 \
        const bool rm = layout == CblasRowMajor;                                                                 \
        char uu = rm ? cblas_row_uplo_char(uplo) : cblas_uplo_char(uplo);                                        \
        char tt = rm ? cblas_row_trans_char(trans) : cblas_trans_char(trans);                                    \
        zynum_blas_int nn = n, kk = k, la = lda, lb = ldb, lc = ldc;                                             \
        FNAME(&uu, &tt, &nn, &kk, &alpha, a, &la, b, &lb, &beta, c, &lc);                                        \
    }
ZB_CBLAS_SYR2K(cblas_dsyr2k, dsyr2k_, double)
ZB_CBLAS_SYR2K(cblas_ssyr2k, ssyr2k_, float)
#undef ZB_CBLAS_SYR2K

int zynum_blas_gpu_dsymm_device(char side, char uplo, int m, int n, double alpha, const double* a, int lda,
                                const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
    return device_symm<double>("dsymm_device", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}
int zynum_blas_gpu_ssymm_device(char side, char uplo, int m, int n, float alpha, const float* a, int lda,
                                const float* b, int ldb, float beta, float* c, int ldc, void* stream) {
    return device_symm<float>("ssymm_device", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}
int zynum_blas_gpu_dtrmm_device(char side, char uplo, char transa, char diag, int m, int n, double alpha,
                                const double* a, int lda, double* b, int ldb, void* stream) {
    return device_trsm<double>("dtrmm_device", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream, true);
}
int zynum_blas_gpu_strmm_device(char side, char uplo, char transa, char diag, int m, int n, float alpha,
                                const float* a, int lda, float* b, int ldb, void* stream) {
    return device_trsm<float>("strmm_device", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, stream, true);
}
int zynum_blas_gpu_dsyr2k_device(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
                                 const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
    return device_syr2k<double>("dsyr2k_device", uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}
int zynum_blas_gpu_ssyr2k_device(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
                                 const float* b, int ldb, float beta, float* c, int ldc, void* stream) {
    return device_syr2k<float>("ssyr2k_device", uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}

// Complex SYMM / HEMM / TRMM / SYR2K / HER2K / HERK on device pointers
// (interleaved complex; complex scalars point to re, im; HERK alpha, beta and
// HER2K beta are real, by value, as in cblas_zherk / cblas_zher2k).
#define ZB_DEV_SYMM_C(NAME, R, WHAT, HERM)                                                                       \
    int NAME(char side, char uplo, int m, int n, const R* alpha, const R* a, int lda, const R* b, int ldb,      \
             const R* beta, R* c, int ldc, void* stream) {                                                      \
        return device_symm_c<R>(WHAT, side, uplo, m, n, cnum<R>(alpha[0], alpha[1]),                            \
                                reinterpret_cast<const cnum<R>*>(a), lda, reinterpret_cast<const cnum<R>*>(b), ldb, \
                                cnum<R>(beta[0], beta[1]), reinterpret_cast<cnum<R>*>(c), ldc, stream, HERM);   \
    }
ZB_DEV_SYMM_C(zynum_blas_gpu_zsymm_device, double, "zsymm_device", false)
ZB_DEV_SYMM_C(zynum_blas_gpu_csymm_device, float, "csymm_device", false)
ZB_DEV_SYMM_C(zynum_blas_gpu_zhemm_device, double, "zhemm_device", true)
ZB_DEV_SYMM_C(zynum_blas_gpu_chemm_device, float, "chemm_device", true)
#undef ZB_DEV_SYMM_C

int zynum_blas_gpu_ztrmm_device(char side, char uplo, char transa, char diag, int m, int n, const double* alpha,
                                const double* a, int lda, double* b, int ldb, void* stream) {
    return device_trsm<cnum<double>>("ztrmm_device", side, uplo, transa, diag, m, n, cnum<double>(alpha[0], alpha[1]),
                                     reinterpret_cast<const cnum<double>*>(a), lda, reinterpret_cast<cnum<double>*>(b),
                                     ldb, stream, true);
}
int zynum_blas_gpu_ctrmm_device(char side, char uplo, char transa, char diag, int m, int n, const float* alpha,
                                const float* a, int lda, float* b, int ldb, void* stream) {
    return device_trsm<cnum<float>>("ctrmm_device", side, uplo, transa, diag, m, n, cnum<float>(alpha[0], alpha[1]),
                                    reinterpret_cast<const cnum<float>*>(a), lda, reinterpret_cast<cnum<float>*>(b),
                                    ldb, stream, true);
}

#define ZB_DEV_SYR2K_C(NAME, R, WHAT)                                                                              \
    int NAME(char uplo, char trans, int n, int k, const R* alpha, const R* a, int lda, const R* b, int ldb,        \
             const R* beta, R* c, int ldc, void* stream) {                                                         \
        return device_rank2k_c<R>(WHAT, uplo, trans, n, k, cnum<R>(alpha[0], alpha[1]),                            \
                                  reinterpret_cast<const cnum<R>*>(a), lda, reinterpret_cast<const cnum<R>*>(b), ldb, \
                                  cnum<R>(beta[0], beta[1]), reinterpret_cast<cnum<R>*>(c), ldc, stream, false, true); \
    }
ZB_DEV_SYR2K_C(zynum_blas_gpu_zsyr2k_device, double, "zsyr2k_device")
ZB_DEV_SYR2K_C(zynum_blas_gpu_csyr2k_device, float, "csyr2k_device")
#undef ZB_DEV_SYR2K_C

#define ZB_DEV_HER2K(NAME, R, WHAT)                                                                                \
    int NAME(char uplo, char trans, int n, int k, const R* alpha, const R* a, int lda, const R* b, int ldb,        \
             R beta, R* c, int ldc, void* stream) {                                                                \
        return device_rank2k_c<R>(WHAT, uplo, trans, n, k, cnum<R>(alpha[0], alpha[1]),                            \
                                  reinterpret_cast<const cnum<R>*>(a), lda, reinterpret_cast<const cnum<R>*>(b), ldb, \
                                  cnum<R>(beta), reinterpret_cast<cnum<R>*>(c), ldc, stream, true, true);          \
    }
ZB_DEV_HER2K(zynum_blas_gpu_zher2k_device, double, "zher2k_device")
ZB_DEV_HER2K(zynum_blas_gpu_cher2k_device, float, "cher2k_device")
#undef ZB_DEV_HER2K

#define ZB_DEV_HERK(NAME, R, WHAT)                                                                                   \
    int NAME(char uplo, char trans, int n, int k, R alpha, const R* a, int lda, R beta, R* c, int ldc,             \
             void* stream) {                                                                                       \
        return device_rank2k_c<R>(WHAT, uplo, trans, n, k, cnum<R>(alpha), reinterpret_cast<const cnum<R>*>(a), lda, \
                                  nullptr, 0, cnum<R>(beta), reinterpret_cast<cnum<R>*>(c), ldc, stream, true, false); \
    }
ZB_DEV_HERK(zynum_blas_gpu_zherk_device, double, "zherk_device")
ZB_DEV_HERK(zynum_blas_gpu_cherk_device, float, "cherk_device")
#undef ZB_DEV_HERK

// GEMM restricted to one triangle of C (the "gemmt" extension): only elements
// with row <= col (uplo 'U') or row >= col ('L') are computed and written.
int zynum_blas_gpu_dgemmt_device(char uplo, char transa, char transb, int n, int k, double alpha, const double* a,
                                 int lda, const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
    const char ul = up(&uplo), ta = up(&transa), tb = up(&transb);
    if (!valid_uplo(ul)) return 1;
    int info = gemm_error(ta, tb, n, n, k, lda, ldb, ldc);
    // dgemm_ numbering -> (uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    if (info) return info <= 2 ? info + 1 : (info <= 4 ? 4 : info);
    if (n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GemmArgsF64 g{ta, tb, n, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    g.tri = (ul == 'U') ? 1 : 2;
    if (k == 0) return cuda_status(syrk_scale_only<double>(n, ul, beta, c, ldc, st), "dgemmt_device");
    GemmPlan p = plan_native_gemm(n, n, k, 8, cx.sm_count);
    void* ws = nullptr;
    const size_t need = splitk_workspace_elems(n, n, p.splits) * sizeof(double);
    if (need && (e = cx.stream_scratch(st, need, &ws)) != cudaSuccess) return cuda_status(e, "dgemmt_device");
    return cuda_status(dgemm_native(g, p, static_cast<double*>(ws), st), "dgemmt_device");
}

int zynum_blas_gpu_dsymmetrize_device(char uplo, int n, double* c, int ldc, void* stream) {
    const char ul = up(&uplo);
    if (!valid_uplo(ul)) return 1;
    if (n < 0) return 2;
    if (ldc < max1(n)) return 4;
    return cuda_status(symmetrize_matrix<double>(ul, n, c, ldc, static_cast<cudaStream_t>(stream)), "dsymmetrize");
}

int zynum_blas_gpu_dgemm_device(char transa, char transb, int m, int n, int k, double alpha, const double* a,
                                int lda, const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
    const char ta = up(&transa), tb = up(&transb);
    int info = gemm_error(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GemmArgsF64 g{ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    return cuda_status(run_dgemm(g, st, StreamScratch{&cx}), "dgemm_device");
}

int zynum_blas_gpu_sgemm_device(char transa, char transb, int m, int n, int k, float alpha, const float* a, int lda,
                                const float* b, int ldb, float beta, float* c, int ldc, void* stream) {
    const char ta = up(&transa), tb = up(&transb);
    int info = gemm_error(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "initialisation");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GemmArgsF32 g{ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc};
    return cuda_status(run_sgemm(g, st, StreamScratch{&cx}), "sgemm_device");
}

int zynum_blas_gpu_set_dgemm_method(int method) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.dgemm_method;
    if (method >= METHOD_NATIVE && method <= METHOD_AUTO) cx.dgemm_method = method;
    return old;
}

int zynum_blas_gpu_set_sgemm_method(int method) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.sgemm_method;
    if (method >= SMETHOD_NATIVE && method <= SMETHOD_OZAKI) cx.sgemm_method = method;
    return old;
}

int zynum_blas_gpu_set_ozaki_slices(int slices) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.ozaki_slices;
    if (slices == 0 || (slices >= 2 && slices <= kOzakiMaxSlices)) cx.ozaki_slices = slices;
    return old;
}

int zynum_blas_gpu_set_ozaki_scheme(int scheme) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.ozaki_scheme;
    if (scheme >= OZAKI_AUTO && scheme <= OZAKI_CRT) cx.ozaki_scheme = scheme;
    return old;
}

int zynum_blas_gpu_set_ozaki_moduli(int moduli) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    cx.init();
    int old = cx.ozaki_moduli;
    if (moduli == 0 || (moduli >= 2 && moduli <= kCrtMaxModuli)) cx.ozaki_moduli = moduli;
    return old;
}

int zynum_blas_gpu_ozaki_plan_ex(int m, int n, int k, int* scheme, int* digits, int* products) {
    Context& cx = context();
    OzakiPlan p;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        p = plan_ozaki(m, n, k, cx.ozaki_slices, cx.ozaki_scheme, cx.ozaki_moduli);
    }
    int d, prods;
    if (p.scheme == OZAKI_CRT) {
        d = p.moduli;
        prods = p.moduli;
    } else {
        d = p.slices ? p.slices : ozaki_last_slices();  // automatic: the count the last call chose
        prods = d * (d + 1) / 2;
    }
    if (scheme) *scheme = p.scheme;
    if (digits) *digits = d;
    if (products) *products = prods;
    return 0;
}

int zynum_blas_gpu_ozaki_plan(int m, int n, int k, int* slices, int* products) {
    return zynum_blas_gpu_ozaki_plan_ex(m, n, k, nullptr, slices, products);
}

const char* zynum_blas_gpu_last_error(void) { return last_error(); }

int zynum_blas_gpu_profile(int enable) { return profile_control(enable); }
int zynum_blas_gpu_profile_read(double* ms, int max) { return profile_read(ms, max); }
long long zynum_blas_gpu_launch_count(void) { return launch_count(); }

void zynum_blas_gpu_inject_fault(int kind, int count) {
    Context& cx = context();
    std::lock_guard<std::recursive_mutex> lock(cx.mutex);
    if (kind == 1) cx.faults.fail_next_reservations = count;
    if (kind == 2) cx.faults.fail_next_sync = count;
    if (kind == 3) cx.faults.hold_next_products.store(count);
}

int zynum_blas_gpu_device_status(void* stream) {
    Context& cx = context();
    cudaError_t e;
    {
        std::lock_guard<std::recursive_mutex> lock(cx.mutex);
        e = cx.init();
    }
    if (e != cudaSuccess) return cuda_status(e, "device_status");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = check_wait_report(st);
    return cuda_status(e, "device_status");
}

}  // extern "C"
