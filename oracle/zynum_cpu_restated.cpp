// Restatement of the reference's x86-64 CPU GEMM path, used ONLY as the timed
// CPU baseline of bench.py (test infrastructure: the product never links it).
//
// The reference is Zig 0.16 and cannot be built in this image; this file
// restates the structure of its real-GEMM route for x86-64:
//   * planner.zig: parallel threshold 192^3 (:14), requested threads =
//     min(maxThreads, n) (:136-144), desiredThreadCount caps (:88-168: work
//     < 256^3 -> <= 6 threads for square f64, < 256^3 -> 2 / < 384^3 -> 4
//     otherwise), column tasks aligned to whole packed-B panels (:50-69),
//     at most 64 tasks (thread_pool.zig:8), one worker thread per task.
//   * packed_simd.zig:306 noTransReal: for every tile_n-column panel pack B
//     (k x tile_n, packing.zig:131), then run a lanes x row_groups by tile_n
//     register tile over the full K (accumulatePackedP :140, k unrolled x4),
//     epilogue alpha*acc + beta*C with beta == 0 not reading C
//     (epilogue.zig:35), tails by narrower row groups then scalars.
//   * x86Shape (packed_params.zig:45-66): AVX-512 f64 = 8 lanes x 2 groups x
//     8 columns, f32 = 16 lanes x 2 groups x 12 columns; AVX2 f64 = 4 x 1 x 8,
//     f32 = 8 x 1 x 12.
//   * transposedAReal (planner.zig:360): TN/TT pack A^T (m x k) first
//     (packing.zig:65), NT reads B transposed while packing (packing.zig:75).
// Threads: min(ZYNUM_MAXIMUM_THREADS or hardware threads, 64) (runtime.zig:54).
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include <immintrin.h>

namespace {

template <typename T>
struct Task {
    char tb;
    size_t m, n0, n1, k;
    T alpha, beta;
    const T* a;
    size_t lda;
    const T* b;
    size_t ldb;
    T* c;
    size_t ldc;
};

template <typename T>
inline T bval(const Task<T>& t, size_t p, size_t j) {
    return t.tb == 'N' ? t.b[p + j * t.ldb] : t.b[j + p * t.ldb];
}

template <typename T>
void pack_panel(const Task<T>& t, size_t j, size_t tile_n, size_t width, T* pack) {
    for (size_t p = 0; p < t.k; ++p)
        for (size_t c = 0; c < tile_n; ++c) pack[p * tile_n + c] = c < width ? bval(t, p, j + c) : T(0);
}

template <typename T>
inline void store(const Task<T>& t, size_t row, size_t col, T acc) {
    T* cp = t.c + row + col * t.ldc;
    *cp = (t.alpha == T(1) && t.beta == T(0)) ? acc : t.alpha * acc + (t.beta == T(0) ? T(0) : t.beta * *cp);
}

// Scalar tail rows for one packed panel.
template <typename T>
void tail_rows(const Task<T>& t, const T* pack, size_t tile_n, size_t width, size_t i0, size_t j) {
    for (size_t i = i0; i < t.m; ++i) {
        T acc[16] = {};
        for (size_t p = 0; p < t.k; ++p) {
            T av = t.a[i + p * t.lda];
            for (size_t c = 0; c < tile_n; ++c) acc[c] += av * pack[p * tile_n + c];
        }
        for (size_t c = 0; c < width; ++c) store(t, i, j + c, acc[c]);
    }
}

// ---------------------------------------------------------------- AVX-512
__attribute__((target("avx512f,fma"))) void panel_f64_avx512(const Task<double>& t, const double* pack, size_t j,
                                                             size_t width) {
    constexpr size_t L = 8, G = 2, TN = 8;
    size_t i = 0;
    for (; i + L * G <= t.m; i += L * G) {
        __m512d acc[G][TN];
        for (size_t g = 0; g < G; ++g)
            for (size_t c = 0; c < TN; ++c) acc[g][c] = _mm512_setzero_pd();
        for (size_t p = 0; p < t.k; ++p) {
            const double* ap = t.a + i + p * t.lda;
            __m512d a0 = _mm512_loadu_pd(ap), a1 = _mm512_loadu_pd(ap + L);
            const double* bp = pack + p * TN;
#pragma GCC unroll 8
            for (size_t c = 0; c < TN; ++c) {
                __m512d bv = _mm512_set1_pd(bp[c]);
                acc[0][c] = _mm512_fmadd_pd(a0, bv, acc[0][c]);
                acc[1][c] = _mm512_fmadd_pd(a1, bv, acc[1][c]);
            }
        }
        for (size_t c = 0; c < width; ++c)
            for (size_t g = 0; g < G; ++g) {
                double* cp = t.c + i + g * L + (j + c) * t.ldc;
                __m512d out = acc[g][c];
                if (!(t.alpha == 1.0 && t.beta == 0.0)) {
                    out = _mm512_mul_pd(out, _mm512_set1_pd(t.alpha));
                    if (t.beta != 0.0) out = _mm512_fmadd_pd(_mm512_set1_pd(t.beta), _mm512_loadu_pd(cp), out);
                }
                _mm512_storeu_pd(cp, out);
            }
    }
    tail_rows(t, pack, TN, width, i, j);
}

__attribute__((target("avx512f,fma"))) void panel_f32_avx512(const Task<float>& t, const float* pack, size_t j,
                                                             size_t width) {
    constexpr size_t L = 16, G = 2, TN = 12;
    size_t i = 0;
    for (; i + L * G <= t.m; i += L * G) {
        __m512 acc[G][TN];
        for (size_t g = 0; g < G; ++g)
            for (size_t c = 0; c < TN; ++c) acc[g][c] = _mm512_setzero_ps();
        for (size_t p = 0; p < t.k; ++p) {
            const float* ap = t.a + i + p * t.lda;
            __m512 a0 = _mm512_loadu_ps(ap), a1 = _mm512_loadu_ps(ap + L);
            const float* bp = pack + p * TN;
#pragma GCC unroll 12
            for (size_t c = 0; c < TN; ++c) {
                __m512 bv = _mm512_set1_ps(bp[c]);
                acc[0][c] = _mm512_fmadd_ps(a0, bv, acc[0][c]);
                acc[1][c] = _mm512_fmadd_ps(a1, bv, acc[1][c]);
            }
        }
        for (size_t c = 0; c < width; ++c)
            for (size_t g = 0; g < G; ++g) {
                float* cp = t.c + i + g * L + (j + c) * t.ldc;
                __m512 out = acc[g][c];
                if (!(t.alpha == 1.0f && t.beta == 0.0f)) {
                    out = _mm512_mul_ps(out, _mm512_set1_ps(t.alpha));
                    if (t.beta != 0.0f) out = _mm512_fmadd_ps(_mm512_set1_ps(t.beta), _mm512_loadu_ps(cp), out);
                }
                _mm512_storeu_ps(cp, out);
            }
    }
    tail_rows(t, pack, TN, width, i, j);
}

// ------------------------------------------------------------------ AVX2
__attribute__((target("avx2,fma"))) void panel_f64_avx2(const Task<double>& t, const double* pack, size_t j,
                                                        size_t width) {
    constexpr size_t L = 4, TN = 8;
    size_t i = 0;
    for (; i + L <= t.m; i += L) {
        __m256d acc[TN];
        for (size_t c = 0; c < TN; ++c) acc[c] = _mm256_setzero_pd();
        for (size_t p = 0; p < t.k; ++p) {
            __m256d a0 = _mm256_loadu_pd(t.a + i + p * t.lda);
            const double* bp = pack + p * TN;
            for (size_t c = 0; c < TN; ++c) acc[c] = _mm256_fmadd_pd(a0, _mm256_set1_pd(bp[c]), acc[c]);
        }
        for (size_t c = 0; c < width; ++c) {
            double tmp[L];
            _mm256_storeu_pd(tmp, acc[c]);
            for (size_t r = 0; r < L; ++r) store(t, i + r, j + c, tmp[r]);
        }
    }
    tail_rows(t, pack, TN, width, i, j);
}

__attribute__((target("avx2,fma"))) void panel_f32_avx2(const Task<float>& t, const float* pack, size_t j,
                                                        size_t width) {
    constexpr size_t L = 8, TN = 12;
    size_t i = 0;
    for (; i + L <= t.m; i += L) {
        __m256 acc[TN];
        for (size_t c = 0; c < TN; ++c) acc[c] = _mm256_setzero_ps();
        for (size_t p = 0; p < t.k; ++p) {
            __m256 a0 = _mm256_loadu_ps(t.a + i + p * t.lda);
            const float* bp = pack + p * TN;
            for (size_t c = 0; c < TN; ++c) acc[c] = _mm256_fmadd_ps(a0, _mm256_set1_ps(bp[c]), acc[c]);
        }
        for (size_t c = 0; c < width; ++c) {
            float tmp[L];
            _mm256_storeu_ps(tmp, acc[c]);
            for (size_t r = 0; r < L; ++r) store(t, i + r, j + c, tmp[r]);
        }
    }
    tail_rows(t, pack, TN, width, i, j);
}

bool has_avx512() {
    static int v = __builtin_cpu_supports("avx512f") ? 1 : 0;
    return v;
}

template <typename T>
size_t tile_n() {
    return sizeof(T) == 8 ? 8 : 12;
}

template <typename T>
void run_task(const Task<T>& t) {
    const size_t tn = tile_n<T>();
    std::vector<T> pack(t.k * tn);
    for (size_t j = t.n0; j < t.n1; j += tn) {
        size_t width = std::min(tn, t.n1 - j);
        pack_panel(t, j, tn, width, pack.data());
        if constexpr (sizeof(T) == 8) {
            if (has_avx512())
                panel_f64_avx512(t, pack.data(), j, width);
            else
                panel_f64_avx2(t, pack.data(), j, width);
        } else {
            if (has_avx512())
                panel_f32_avx512(t, pack.data(), j, width);
            else
                panel_f32_avx2(t, pack.data(), j, width);
        }
    }
}

size_t max_threads() {
    size_t hw = std::max<unsigned>(1, std::thread::hardware_concurrency());
    if (const char* v = std::getenv("ZYNUM_MAXIMUM_THREADS")) {
        long x = std::atol(v);
        if (x > 0) hw = std::min<size_t>(hw, (size_t)x);
    }
    return std::min<size_t>(hw, 64);
}

// planner.zig:88-168 desiredThreadCount, restricted to the packed-SIMD route.
template <typename T>
size_t desired_threads(size_t m, size_t n, size_t k) {
    const size_t work = m * n * k;
    if (work < 192ull * 192 * 192 || n < 2) return 1;
    size_t threads = std::min(max_threads(), n);
    const size_t mn = std::min({m, n, k}), mx = std::max({m, n, k});
    const bool squareish = mx <= 4 * mn;
    if (squareish && sizeof(T) == 8) {
        if (work < 256ull * 256 * 256) threads = std::min<size_t>(threads, 6);
    } else if (work < 256ull * 256 * 256) {
        threads = std::min<size_t>(threads, 2);
    } else if (work < 384ull * 384 * 384) {
        threads = std::min<size_t>(threads, 4);
    }
    return std::max<size_t>(1, std::min<size_t>(threads, 64));
}

template <typename T>
void gemm(char ta, char tb, int m_, int n_, int k_, T alpha, const T* a, int lda, const T* b, int ldb, T beta, T* c,
          int ldc) {
    if (m_ <= 0 || n_ <= 0) return;
    const size_t m = m_, n = n_, k = k_;
    if (k == 0 || alpha == T(0)) {
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < m; ++i) c[i + j * ldc] = beta == T(0) ? T(0) : beta * c[i + j * ldc];
        return;
    }
    std::vector<T> at;
    const T* ap = a;
    size_t la = lda;
    if (ta != 'N') {  // transposedAReal: materialise A^T (m x k)
        at.resize(m * k);
        for (size_t i = 0; i < m; ++i)
            for (size_t p = 0; p < k; ++p) at[i + p * m] = a[p + i * (size_t)lda];
        ap = at.data();
        la = m;
    }
    const size_t threads = desired_threads<T>(m, n, k);
    const size_t tn = tile_n<T>();
    const size_t panels = (n + tn - 1) / tn;
    const size_t tasks = std::max<size_t>(1, std::min(threads, panels));
    std::vector<std::thread> pool;
    for (size_t q = 0; q < tasks; ++q) {
        size_t p0 = q * panels / tasks, p1 = (q + 1) * panels / tasks;
        Task<T> t{tb, m, std::min(n, p0 * tn), std::min(n, p1 * tn), k, alpha, beta, ap, la, b, (size_t)ldb, c,
                  (size_t)ldc};
        if (tasks == 1)
            run_task(t);
        else
            pool.emplace_back([t] { run_task(t); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {
void zynum_cpu_dgemm(char ta, char tb, int m, int n, int k, double alpha, const double* a, int lda, const double* b,
                     int ldb, double beta, double* c, int ldc) {
    gemm<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
void zynum_cpu_sgemm(char ta, char tb, int m, int n, int k, float alpha, const float* a, int lda, const float* b,
                     int ldb, float beta, float* c, int ldc) {
    gemm<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int zynum_cpu_threads(int m, int n, int k) { return (int)desired_threads<double>(m, n, k); }
int zynum_cpu_has_avx512(void) { return has_avx512(); }
}
