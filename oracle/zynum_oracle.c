/*
 * CPU oracle for the Zynum GEMM / TRSM / SYRK path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: the tests, the smoke
 * check and the CPU-baseline leg of bench.py may call it; the product library
 * (zynum_b200/lib/libzynum_blas_gpu.so) never links or calls it.
 *
 * Every routine restates the reference's scalar semantics in plain C
 * (compiled with -ffp-contract=off so that `a*b + c` rounds twice, exactly as
 * Zig's default float mode does):
 *
 *   oracle_?gemm   gemm.zig:1392-1430 (quick returns :1407-1414, portable
 *                  triple loop :1422-1429) and gemmComplexPortable :1234-1246,
 *                  with matrixValue (matrix_vector/access.zig:23-29) for N/T/C.
 *   oracle_?trsm   triangular.zig:233-249 (alpha pre-scale :51-58, then one
 *                  trsv per right-hand side, matrix_vector/triangular.zig
 *                  :400-435, triValue access.zig:54-64) and the right-side
 *                  row solve solveRightRow triangular.zig:72-88.
 *   oracle_?syrk   symmetric.zig:180-199 (runSyrkColumns), z / c with op = C
 *                  conjugating (matrixValue).
 *   oracle_[zc]trsm complex trsm: triValue with conj for op = C, right side per
 *                  solveRightRow (triangular.zig:72-88).
 *   oracle_?symm   symmetric.zig:56-70 (runSymmColumns, symValue access.zig:31-42).
 *   oracle_?trmm   triangular.zig:202-231 (left: trmv + alpha scale per column,
 *                  runLeftColumns :105-110; right: row products :212-229).
 *   oracle_?syr2k  symmetric.zig:301-329 (runSyr2kColumns, real case).
 *   oracle_ddgemm  a double-double (error-free TwoProd/TwoSum, Dekker 1971 /
 *                  Knuth) accumulation of op(A)op(B); used to state the error
 *                  of every GPU result.  No counterpart in the reference.
 *
 * Complex numbers are interleaved (re, im) pairs, column-major, exactly like
 * the reference's ComplexF32/ComplexF64 extern structs (types.zig).
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <string.h>

typedef int32_t blas_int;

static inline size_t ix(blas_int ld, size_t row, size_t col) { return row + col * (size_t)ld; }

static inline int upc(char c) { return (c >= 'a' && c <= 'z') ? c - 32 : c; }

/* ---------------------------------------------------------------- real GEMM */

#define DEFINE_REAL_GEMM(NAME, T)                                                              \
    void NAME(char ta, char tb, blas_int m, blas_int n, blas_int k, T alpha, const T *a,      \
              blas_int lda, const T *b, blas_int ldb, T beta, T *c, blas_int ldc) {            \
        ta = (char)upc(ta);                                                                    \
        tb = (char)upc(tb);                                                                    \
        if (m <= 0 || n <= 0) return;                                                          \
        if (k <= 0 || alpha == (T)0) {                                                         \
            for (size_t j = 0; j < (size_t)n; ++j)                                             \
                for (size_t i = 0; i < (size_t)m; ++i) {                                       \
                    size_t q = ix(ldc, i, j);                                                  \
                    c[q] = (beta == (T)0) ? (T)0 : beta * c[q];                                \
                }                                                                              \
            return;                                                                            \
        }                                                                                      \
        for (size_t j = 0; j < (size_t)n; ++j)                                                 \
            for (size_t i = 0; i < (size_t)m; ++i) {                                           \
                T sum = 0;                                                                     \
                for (size_t p = 0; p < (size_t)k; ++p) {                                       \
                    T av = (ta == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];                  \
                    T bv = (tb == 'N') ? b[ix(ldb, p, j)] : b[ix(ldb, j, p)];                  \
                    sum = sum + av * bv;                                                       \
                }                                                                              \
                size_t q = ix(ldc, i, j);                                                      \
                c[q] = alpha * sum + ((beta == (T)0) ? (T)0 : beta * c[q]);                    \
            }                                                                                  \
    }

DEFINE_REAL_GEMM(oracle_dgemm, double)
DEFINE_REAL_GEMM(oracle_sgemm, float)

/* ------------------------------------------------------------- complex GEMM */

#define DEFINE_COMPLEX_GEMM(NAME, T)                                                              \
    void NAME(char ta, char tb, blas_int m, blas_int n, blas_int k, const T *alpha, const T *a,  \
              blas_int lda, const T *b, blas_int ldb, const T *beta, T *c, blas_int ldc) {        \
        ta = (char)upc(ta);                                                                       \
        tb = (char)upc(tb);                                                                       \
        if (m <= 0 || n <= 0) return;                                                             \
        const T ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];                         \
        const int beta_zero = (br == (T)0 && bi == (T)0);                                         \
        if (k <= 0 || (ar == (T)0 && ai == (T)0)) {                                               \
            for (size_t j = 0; j < (size_t)n; ++j)                                                \
                for (size_t i = 0; i < (size_t)m; ++i) {                                          \
                    T *cv = c + 2 * ix(ldc, i, j);                                                \
                    if (beta_zero) {                                                              \
                        cv[0] = 0;                                                                \
                        cv[1] = 0;                                                                \
                    } else {                                                                      \
                        T r = br * cv[0] - bi * cv[1], s = br * cv[1] + bi * cv[0];               \
                        cv[0] = r;                                                                \
                        cv[1] = s;                                                                \
                    }                                                                             \
                }                                                                                 \
            return;                                                                               \
        }                                                                                         \
        for (size_t j = 0; j < (size_t)n; ++j)                                                    \
            for (size_t i = 0; i < (size_t)m; ++i) {                                              \
                T sr = 0, si = 0;                                                                 \
                for (size_t p = 0; p < (size_t)k; ++p) {                                          \
                    const T *av = a + 2 * ((ta == 'N') ? ix(lda, i, p) : ix(lda, p, i));          \
                    const T *bv = b + 2 * ((tb == 'N') ? ix(ldb, p, j) : ix(ldb, j, p));          \
                    T xr = av[0], xi = (ta == 'C') ? -av[1] : av[1];                              \
                    T yr = bv[0], yi = (tb == 'C') ? -bv[1] : bv[1];                              \
                    T pr = xr * yr - xi * yi, pi = xr * yi + xi * yr;                             \
                    sr = sr + pr;                                                                 \
                    si = si + pi;                                                                 \
                }                                                                                 \
                T *cv = c + 2 * ix(ldc, i, j);                                                    \
                T tr = ar * sr - ai * si, ti = ar * si + ai * sr;                                 \
                T ur = 0, ui = 0;                                                                 \
                if (!beta_zero) {                                                                 \
                    ur = br * cv[0] - bi * cv[1];                                                 \
                    ui = br * cv[1] + bi * cv[0];                                                 \
                }                                                                                 \
                cv[0] = tr + ur;                                                                  \
                cv[1] = ti + ui;                                                                  \
            }                                                                                     \
    }

DEFINE_COMPLEX_GEMM(oracle_zgemm, double)
DEFINE_COMPLEX_GEMM(oracle_cgemm, float)

/* ------------------------------------------------- double-double reference */

/* TwoSum (Knuth) and TwoProd (via FMA): error-free transformations. */
static inline void two_sum(double a, double b, double *s, double *e) {
    double x = a + b;
    double z = x - a;
    *e = (a - (x - z)) + (b - z);
    *s = x;
}
static inline void two_prod(double a, double b, double *p, double *e) {
    double x = a * b;
    *e = fma(a, b, -x);
    *p = x;
}
/* (hi, lo) += (p, q) with the usual double-double add (Bailey's QD "sloppy"
 * add is not enough under heavy cancellation, so both halves are renormalised). */
static inline void dd_add(double *hi, double *lo, double p, double q) {
    double s, e, t, f;
    two_sum(*hi, p, &s, &e);
    two_sum(*lo, q, &t, &f);
    e += t;
    double u, v;
    two_sum(s, e, &u, &v);
    v += f;
    two_sum(u, v, hi, lo);
}

/* C_hi + C_lo = op(A) op(B) in double-double (alpha = 1, beta = 0).  The
 * caller forms alpha/beta itself in extended precision when it needs them. */
void oracle_ddgemm(char ta, char tb, blas_int m, blas_int n, blas_int k, const double *a, blas_int lda,
                   const double *b, blas_int ldb, double *c_hi, double *c_lo, blas_int ldc) {
    ta = (char)upc(ta);
    tb = (char)upc(tb);
    for (size_t j = 0; j < (size_t)n; ++j)
        for (size_t i = 0; i < (size_t)m; ++i) {
            double hi = 0, lo = 0;
            for (size_t p = 0; p < (size_t)k; ++p) {
                double av = (ta == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];
                double bv = (tb == 'N') ? b[ix(ldb, p, j)] : b[ix(ldb, j, p)];
                double pp, pe;
                two_prod(av, bv, &pp, &pe);
                dd_add(&hi, &lo, pp, pe);
            }
            c_hi[ix(ldc, i, j)] = hi;
            c_lo[ix(ldc, i, j)] = lo;
        }
}

/* Sampled double-double entries: out_hi[q] + out_lo[q] = (op(A) op(B))[rows[q], cols[q]]. */
void oracle_ddgemm_sampled(char ta, char tb, blas_int k, const double *a, blas_int lda, const double *b,
                           blas_int ldb, int64_t count, const int64_t *rows, const int64_t *cols,
                           double *out_hi, double *out_lo, double *out_abs) {
    ta = (char)upc(ta);
    tb = (char)upc(tb);
    for (int64_t q = 0; q < count; ++q) {
        size_t i = (size_t)rows[q], j = (size_t)cols[q];
        double hi = 0, lo = 0, absum = 0;
        for (size_t p = 0; p < (size_t)k; ++p) {
            double av = (ta == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];
            double bv = (tb == 'N') ? b[ix(ldb, p, j)] : b[ix(ldb, j, p)];
            double pp, pe;
            two_prod(av, bv, &pp, &pe);
            dd_add(&hi, &lo, pp, pe);
            absum += fabs(av * bv);
        }
        out_hi[q] = hi;
        out_lo[q] = lo;
        if (out_abs) out_abs[q] = absum;
    }
}

/* Sampled float-input double-double reference for SGEMM error statements. */
void oracle_ddgemm_sampled_f32(char ta, char tb, blas_int k, const float *a, blas_int lda, const float *b,
                               blas_int ldb, int64_t count, const int64_t *rows, const int64_t *cols,
                               double *out_hi, double *out_lo, double *out_abs) {
    ta = (char)upc(ta);
    tb = (char)upc(tb);
    for (int64_t q = 0; q < count; ++q) {
        size_t i = (size_t)rows[q], j = (size_t)cols[q];
        double hi = 0, lo = 0, absum = 0;
        for (size_t p = 0; p < (size_t)k; ++p) {
            double av = (ta == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];
            double bv = (tb == 'N') ? b[ix(ldb, p, j)] : b[ix(ldb, j, p)];
            double pp, pe;
            two_prod(av, bv, &pp, &pe);
            dd_add(&hi, &lo, pp, pe);
            absum += fabs(av * bv);
        }
        out_hi[q] = hi;
        out_lo[q] = lo;
        if (out_abs) out_abs[q] = absum;
    }
}

/* ---------------------------------------------------------------- real TRSM */

/* triValue (access.zig:54-64): element (row, col) of op(A) for a triangular A. */
#define DEFINE_TRI_VALUE(NAME, T)                                                                   \
    static inline T NAME(char uplo, char diag, char trans, const T *a, blas_int lda, size_t row,    \
                         size_t col) {                                                              \
        size_t ar = (trans == 'N') ? row : col, ac = (trans == 'N') ? col : row;                    \
        if (ar == ac && diag == 'U') return (T)1;                                                   \
        if (uplo == 'U' && ar > ac) return (T)0;                                                    \
        if (uplo == 'L' && ar < ac) return (T)0;                                                    \
        return a[ix(lda, ar, ac)];                                                                  \
    }
DEFINE_TRI_VALUE(tri_d, double)
DEFINE_TRI_VALUE(tri_s, float)

/* op(A) is upper triangular (triangular.zig:47-49 opIsUpper). */
static inline int op_is_upper(char uplo, char trans) {
    return (trans == 'N' && uplo == 'U') || (trans != 'N' && uplo == 'L');
}

#define DEFINE_REAL_TRSM(NAME, T, TRI)                                                                 \
    void NAME(char side, char uplo, char trans, char diag, blas_int m, blas_int n, T alpha,          \
              const T *a, blas_int lda, T *b, blas_int ldb) {                                          \
        side = (char)upc(side); uplo = (char)upc(uplo); trans = (char)upc(trans); diag = (char)upc(diag); \
        if (m <= 0 || n <= 0) return;                                                                  \
        if (alpha != (T)1)                                                                             \
            for (size_t j = 0; j < (size_t)n; ++j)                                                     \
                for (size_t i = 0; i < (size_t)m; ++i) b[ix(ldb, i, j)] = alpha * b[ix(ldb, i, j)];    \
        if (side == 'L') {                                                                             \
            for (size_t j = 0; j < (size_t)n; ++j) {                                                   \
                T *x = b + (size_t)ldb * j;                                                            \
                if (op_is_upper(uplo, trans)) {                                                        \
                    for (size_t r = (size_t)m; r-- > 0;) {                                             \
                        T t = x[r];                                                                    \
                        for (size_t q = r + 1; q < (size_t)m; ++q) t = t - TRI(uplo, diag, trans, a, lda, r, q) * x[q]; \
                        if (diag == 'N') t = t / TRI(uplo, diag, trans, a, lda, r, r);                 \
                        x[r] = t;                                                                      \
                    }                                                                                  \
                } else {                                                                               \
                    for (size_t r = 0; r < (size_t)m; ++r) {                                           \
                        T t = x[r];                                                                    \
                        for (size_t q = 0; q < r; ++q) t = t - TRI(uplo, diag, trans, a, lda, r, q) * x[q]; \
                        if (diag == 'N') t = t / TRI(uplo, diag, trans, a, lda, r, r);                 \
                        x[r] = t;                                                                      \
                    }                                                                                  \
                }                                                                                      \
            }                                                                                          \
        } else {                                                                                       \
            /* X op(A) = B, row by row: x^T = solve(op(A)^T, b^T). */                                  \
            char tt = (trans == 'N') ? 'T' : 'N';                                                      \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                   \
                if (op_is_upper(uplo, tt)) {                                                           \
                    for (size_t r = (size_t)n; r-- > 0;) {                                             \
                        T t = b[ix(ldb, i, r)];                                                        \
                        for (size_t q = r + 1; q < (size_t)n; ++q)                                     \
                            t = t - TRI(uplo, diag, tt, a, lda, r, q) * b[ix(ldb, i, q)];              \
                        if (diag == 'N') t = t / TRI(uplo, diag, tt, a, lda, r, r);                    \
                        b[ix(ldb, i, r)] = t;                                                          \
                    }                                                                                  \
                } else {                                                                               \
                    for (size_t r = 0; r < (size_t)n; ++r) {                                           \
                        T t = b[ix(ldb, i, r)];                                                        \
                        for (size_t q = 0; q < r; ++q) t = t - TRI(uplo, diag, tt, a, lda, r, q) * b[ix(ldb, i, q)]; \
                        if (diag == 'N') t = t / TRI(uplo, diag, tt, a, lda, r, r);                    \
                        b[ix(ldb, i, r)] = t;                                                          \
                    }                                                                                  \
                }                                                                                      \
            }                                                                                          \
        }                                                                                              \
    }

DEFINE_REAL_TRSM(oracle_dtrsm, double, tri_d)
DEFINE_REAL_TRSM(oracle_strsm, float, tri_s)

/* ---------------------------------------------------------------- real SYRK */

#define DEFINE_REAL_SYRK(NAME, T)                                                                  \
    void NAME(char uplo, char trans, blas_int n, blas_int k, T alpha, const T *a, blas_int lda,   \
              T beta, T *c, blas_int ldc) {                                                        \
        uplo = (char)upc(uplo); trans = (char)upc(trans);                                          \
        if (n <= 0) return;                                                                        \
        for (size_t j = 0; j < (size_t)n; ++j) {                                                   \
            size_t r0 = (uplo == 'U') ? 0 : j, r1 = (uplo == 'U') ? j + 1 : (size_t)n;             \
            for (size_t i = r0; i < r1; ++i) {                                                     \
                T sum = 0;                                                                         \
                for (size_t p = 0; p < (size_t)(k > 0 ? k : 0); ++p) {                              \
                    T ai = (trans == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];                   \
                    T aj = (trans == 'N') ? a[ix(lda, j, p)] : a[ix(lda, p, j)];                   \
                    sum = sum + ai * aj;                                                           \
                }                                                                                  \
                size_t q = ix(ldc, i, j);                                                          \
                c[q] = alpha * sum + ((beta == (T)0) ? (T)0 : beta * c[q]);                        \
            }                                                                                      \
        }                                                                                          \
    }

DEFINE_REAL_SYRK(oracle_dsyrk, double)
DEFINE_REAL_SYRK(oracle_ssyrk, float)

/* ---------------------------------------------------------------- real SYMM */

/* symmetric.zig:56-70 runSymmColumns with symValue (access.zig:31-42): the
 * element (i, p) of the symmetric A comes from the stored uplo triangle. */
#define DEFINE_REAL_SYMM(NAME, T)                                                                    \
    void NAME(char side, char uplo, blas_int m, blas_int n, T alpha, const T *a, blas_int lda,      \
              const T *b, blas_int ldb, T beta, T *c, blas_int ldc) {                                \
        side = (char)upc(side); uplo = (char)upc(uplo);                                              \
        if (m <= 0 || n <= 0) return;                                                                \
        for (size_t j = 0; j < (size_t)n; ++j)                                                       \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                 \
                T sum = 0;                                                                           \
                if (side == 'L') {                                                                   \
                    for (size_t p = 0; p < (size_t)m; ++p) {                                         \
                        int st = (uplo == 'U') ? (i <= p) : (i >= p);                                \
                        T av = st ? a[ix(lda, i, p)] : a[ix(lda, p, i)];                             \
                        sum = sum + av * b[ix(ldb, p, j)];                                           \
                    }                                                                                \
                } else {                                                                             \
                    for (size_t p = 0; p < (size_t)n; ++p) {                                         \
                        int st = (uplo == 'U') ? (p <= j) : (p >= j);                                \
                        T av = st ? a[ix(lda, p, j)] : a[ix(lda, j, p)];                             \
                        sum = sum + b[ix(ldb, i, p)] * av;                                           \
                    }                                                                                \
                }                                                                                    \
                size_t q = ix(ldc, i, j);                                                            \
                c[q] = alpha * sum + ((beta == (T)0) ? (T)0 : beta * c[q]);                          \
            }                                                                                        \
    }

DEFINE_REAL_SYMM(oracle_dsymm, double)
DEFINE_REAL_SYMM(oracle_ssymm, float)

/* ---------------------------------------------------------------- real TRMM */

/* triangular.zig:202-231: left side, per column x := op(A) x (trmv) then
 * x := alpha x when alpha != 1 (runLeftColumns :105-110, scaleDenseColumns
 * :52-59); right side, per row b(i, :) := alpha b(i, :) op(A), columns taken
 * in the order that leaves the inputs of later columns unchanged (:212-229). */
#define DEFINE_REAL_TRMM(NAME, T, TRI)                                                                  \
    void NAME(char side, char uplo, char trans, char diag, blas_int m, blas_int n, T alpha,           \
              const T *a, blas_int lda, T *b, blas_int ldb) {                                           \
        side = (char)upc(side); uplo = (char)upc(uplo); trans = (char)upc(trans); diag = (char)upc(diag); \
        if (m <= 0 || n <= 0) return;                                                                   \
        int upper = op_is_upper(uplo, trans);                                                           \
        if (side == 'L') {                                                                              \
            for (size_t j = 0; j < (size_t)n; ++j) {                                                    \
                T *x = b + (size_t)ldb * j;                                                             \
                if (upper) {                                                                            \
                    for (size_t r = 0; r < (size_t)m; ++r) {                                            \
                        T t = 0;                                                                        \
                        for (size_t q = r; q < (size_t)m; ++q) t = t + TRI(uplo, diag, trans, a, lda, r, q) * x[q]; \
                        x[r] = t;                                                                       \
                    }                                                                                   \
                } else {                                                                                \
                    for (size_t r = (size_t)m; r-- > 0;) {                                              \
                        T t = 0;                                                                        \
                        for (size_t q = 0; q <= r; ++q) t = t + TRI(uplo, diag, trans, a, lda, r, q) * x[q]; \
                        x[r] = t;                                                                       \
                    }                                                                                   \
                }                                                                                       \
                if (alpha != (T)1)                                                                      \
                    for (size_t r = 0; r < (size_t)m; ++r) x[r] = alpha * x[r];                         \
            }                                                                                           \
        } else {                                                                                        \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                    \
                if (upper) {                                                                            \
                    for (size_t cc = (size_t)n; cc-- > 0;) {                                            \
                        T sum = 0;                                                                      \
                        for (size_t p = 0; p < (size_t)n; ++p)                                          \
                            sum = sum + b[ix(ldb, i, p)] * TRI(uplo, diag, trans, a, lda, p, cc);       \
                        b[ix(ldb, i, cc)] = alpha * sum;                                                \
                    }                                                                                   \
                } else {                                                                                \
                    for (size_t cc = 0; cc < (size_t)n; ++cc) {                                         \
                        T sum = 0;                                                                      \
                        for (size_t p = 0; p < (size_t)n; ++p)                                          \
                            sum = sum + b[ix(ldb, i, p)] * TRI(uplo, diag, trans, a, lda, p, cc);       \
                        b[ix(ldb, i, cc)] = alpha * sum;                                                \
                    }                                                                                   \
                }                                                                                       \
            }                                                                                           \
        }                                                                                               \
    }

DEFINE_REAL_TRMM(oracle_dtrmm, double, tri_d)
DEFINE_REAL_TRMM(oracle_strmm, float, tri_s)

/* --------------------------------------------------------------- real SYR2K */

/* symmetric.zig:301-329 runSyr2kColumns (real case): one accumulator of
 * a_i b_j + b_i a_j over p, then alpha sum + beta c on the uplo triangle. */
#define DEFINE_REAL_SYR2K(NAME, T)                                                                      \
    void NAME(char uplo, char trans, blas_int n, blas_int k, T alpha, const T *a, blas_int lda,        \
              const T *b, blas_int ldb, T beta, T *c, blas_int ldc) {                                   \
        uplo = (char)upc(uplo); trans = (char)upc(trans);                                               \
        if (n <= 0) return;                                                                             \
        for (size_t j = 0; j < (size_t)n; ++j) {                                                        \
            size_t r0 = (uplo == 'U') ? 0 : j, r1 = (uplo == 'U') ? j + 1 : (size_t)n;                  \
            for (size_t i = r0; i < r1; ++i) {                                                          \
                T sum = 0;                                                                              \
                for (size_t p = 0; p < (size_t)(k > 0 ? k : 0); ++p) {                                   \
                    T ai = (trans == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];                        \
                    T bi = (trans == 'N') ? b[ix(ldb, i, p)] : b[ix(ldb, p, i)];                        \
                    T aj = (trans == 'N') ? a[ix(lda, j, p)] : a[ix(lda, p, j)];                        \
                    T bj = (trans == 'N') ? b[ix(ldb, j, p)] : b[ix(ldb, p, j)];                        \
                    sum = sum + (ai * bj + bi * aj);                                                    \
                }                                                                                       \
                size_t q = ix(ldc, i, j);                                                               \
                c[q] = alpha * sum + ((beta == (T)0) ? (T)0 : beta * c[q]);                             \
            }                                                                                           \
        }                                                                                               \
    }

DEFINE_REAL_SYR2K(oracle_dsyr2k, double)
DEFINE_REAL_SYR2K(oracle_ssyr2k, float)

/* ------------------------------------------------------- complex TRSM / SYRK */

/* Interleaved complex with the reference's scalar arithmetic (core/shared/
 * scalar.zig: sub :63, mul :77, divv :84, conj :92). */
#define DEFINE_CX(CT, R)                                                                     \
    typedef struct { R re, im; } CT;                                                         \
    static inline CT CT##_mul(CT a, CT b) {                                                  \
        CT r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }           \
    static inline CT CT##_add(CT a, CT b) { CT r = {a.re + b.re, a.im + b.im}; return r; }   \
    static inline CT CT##_sub(CT a, CT b) { CT r = {a.re - b.re, a.im - b.im}; return r; }   \
    static inline CT CT##_div(CT a, CT b) {                                                  \
        R den = b.re * b.re + b.im * b.im;                                                   \
        CT r = {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den}; return r; } \
    static inline CT CT##_conj(CT a) { CT r = {a.re, -a.im}; return r; }                     \
    static inline int CT##_is_one(CT a) { return a.re == (R)1 && a.im == (R)0; }             \
    static inline int CT##_is_zero(CT a) { return a.re == (R)0 && a.im == (R)0; }            \
    /* triValue access.zig:54-64: element (row, col) of op(A), conj for op = C */           \
    static inline CT CT##_tri(char uplo, char diag, char trans, const CT *a, blas_int lda,   \
                              size_t row, size_t col) {                                      \
        size_t ar = (trans == 'N') ? row : col, ac = (trans == 'N') ? col : row;             \
        CT one = {(R)1, (R)0}, zero = {(R)0, (R)0};                                          \
        if (ar == ac && diag == 'U') return one;                                             \
        if (uplo == 'U' && ar > ac) return zero;                                             \
        if (uplo == 'L' && ar < ac) return zero;                                             \
        CT v = a[ix(lda, ar, ac)];                                                           \
        return trans == 'C' ? CT##_conj(v) : v;                                              \
    }                                                                                        \
    /* trsv (matrix_vector/triangular.zig, the unit-stride solve) on x[i * inc] */           \
    static void CT##_trsv(char uplo, char trans, char diag, blas_int n, const CT *a,         \
                          blas_int lda, CT *x, size_t inc) {                                 \
        if (op_is_upper(uplo, trans)) {                                                      \
            for (size_t r = (size_t)n; r-- > 0;) {                                           \
                CT t = x[r * inc];                                                           \
                for (size_t q = r + 1; q < (size_t)n; ++q)                                   \
                    t = CT##_sub(t, CT##_mul(CT##_tri(uplo, diag, trans, a, lda, r, q), x[q * inc])); \
                if (diag == 'N') t = CT##_div(t, CT##_tri(uplo, diag, trans, a, lda, r, r)); \
                x[r * inc] = t;                                                              \
            }                                                                                \
        } else {                                                                             \
            for (size_t r = 0; r < (size_t)n; ++r) {                                         \
                CT t = x[r * inc];                                                           \
                for (size_t q = 0; q < r; ++q)                                               \
                    t = CT##_sub(t, CT##_mul(CT##_tri(uplo, diag, trans, a, lda, r, q), x[q * inc])); \
                if (diag == 'N') t = CT##_div(t, CT##_tri(uplo, diag, trans, a, lda, r, r)); \
                x[r * inc] = t;                                                              \
            }                                                                                \
        }                                                                                    \
    }

DEFINE_CX(cxd, double)
DEFINE_CX(cxf, float)

/* triangular.zig:233-249 trsm for complex types: alpha pre-scale (:51-58), one
 * trsv per column (left side); per row (right side, solveRightRow :72-88):
 * op N -> trsv with trans T, op T -> trsv with N, op C -> conj the row, trsv
 * with N, conj the row. */
#define DEFINE_CX_TRSM(NAME, CT)                                                                   \
    void NAME(char side, char uplo, char trans, char diag, blas_int m, blas_int n, const CT *alpha, \
              const CT *a, blas_int lda, CT *b, blas_int ldb) {                                      \
        side = (char)upc(side); uplo = (char)upc(uplo); trans = (char)upc(trans); diag = (char)upc(diag); \
        if (m <= 0 || n <= 0) return;                                                                \
        if (!CT##_is_one(*alpha))                                                                    \
            for (size_t j = 0; j < (size_t)n; ++j)                                                   \
                for (size_t i = 0; i < (size_t)m; ++i) b[ix(ldb, i, j)] = CT##_mul(*alpha, b[ix(ldb, i, j)]); \
        if (side == 'L') {                                                                           \
            for (size_t j = 0; j < (size_t)n; ++j) CT##_trsv(uplo, trans, diag, m, a, lda, b + (size_t)ldb * j, 1); \
        } else {                                                                                     \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                 \
                CT *x = b + i;                                                                       \
                if (trans == 'N') {                                                                  \
                    CT##_trsv(uplo, 'T', diag, n, a, lda, x, (size_t)ldb);                           \
                } else if (trans == 'T') {                                                           \
                    CT##_trsv(uplo, 'N', diag, n, a, lda, x, (size_t)ldb);                           \
                } else {                                                                             \
                    for (size_t q = 0; q < (size_t)n; ++q) x[q * ldb] = CT##_conj(x[q * ldb]);       \
                    CT##_trsv(uplo, 'N', diag, n, a, lda, x, (size_t)ldb);                           \
                    for (size_t q = 0; q < (size_t)n; ++q) x[q * ldb] = CT##_conj(x[q * ldb]);       \
                }                                                                                    \
            }                                                                                        \
        }                                                                                            \
    }

DEFINE_CX_TRSM(oracle_ztrsm, cxd)
DEFINE_CX_TRSM(oracle_ctrsm, cxf)

/* symmetric.zig:180-199 runSyrkColumns for complex types with herm = false:
 * op(A)(i, p) by matrixValue (access.zig:23-29; conj for op = C). */
#define DEFINE_CX_SYRK(NAME, CT)                                                                     \
    void NAME(char uplo, char trans, blas_int n, blas_int k, const CT *alpha, const CT *a, blas_int lda, \
              const CT *beta, CT *c, blas_int ldc) {                                                  \
        uplo = (char)upc(uplo); trans = (char)upc(trans);                                             \
        if (n <= 0) return;                                                                           \
        for (size_t j = 0; j < (size_t)n; ++j) {                                                      \
            size_t r0 = (uplo == 'U') ? 0 : j, r1 = (uplo == 'U') ? j + 1 : (size_t)n;                \
            for (size_t i = r0; i < r1; ++i) {                                                        \
                CT sum = {0, 0};                                                                      \
                for (size_t p = 0; p < (size_t)(k > 0 ? k : 0); ++p) {                                 \
                    CT ai = (trans == 'N') ? a[ix(lda, i, p)] : a[ix(lda, p, i)];                     \
                    CT aj = (trans == 'N') ? a[ix(lda, j, p)] : a[ix(lda, p, j)];                     \
                    if (trans == 'C') { ai = CT##_conj(ai); aj = CT##_conj(aj); }                     \
                    sum = CT##_add(sum, CT##_mul(ai, aj));                                            \
                }                                                                                     \
                size_t q = ix(ldc, i, j);                                                             \
                CT zero = {0, 0};                                                                     \
                c[q] = CT##_add(CT##_mul(*alpha, sum), CT##_is_zero(*beta) ? zero : CT##_mul(*beta, c[q])); \
            }                                                                                         \
        }                                                                                             \
    }

DEFINE_CX_SYRK(oracle_zsyrk, cxd)
DEFINE_CX_SYRK(oracle_csyrk, cxf)

/* ----------------------------------- complex SYMM / HEMM, TRMM, HERK, SYR2K / HER2K */

/* matrixValue (access.zig:23-29): element (row, col) of op(X), conj for op = C;
 * symValue (access.zig:31-42): stored triangle as is (diagonal real when herm),
 * the other triangle mirrored, conjugated when herm. */
#define DEFINE_CX_OPVAL(CT)                                                                   \
    static inline CT CT##_opval(char trans, const CT *x, blas_int ld, size_t row, size_t col) { \
        if (trans == 'N') return x[ix(ld, row, col)];                                         \
        CT v = x[ix(ld, col, row)];                                                           \
        return trans == 'C' ? CT##_conj(v) : v;                                               \
    }                                                                                         \
    static inline CT CT##_symval(char uplo, const CT *a, blas_int lda, size_t row, size_t col, int herm) { \
        if ((uplo == 'U' && row <= col) || (uplo == 'L' && row >= col)) {                     \
            CT v = a[ix(lda, row, col)];                                                      \
            if (herm && row == col) v.im = 0;                                                 \
            return v;                                                                         \
        }                                                                                     \
        CT v = a[ix(lda, col, row)];                                                          \
        return herm ? CT##_conj(v) : v;                                                       \
    }

DEFINE_CX_OPVAL(cxd)
DEFINE_CX_OPVAL(cxf)

/* symmetric.zig:107-157 symm -> runSymmColumns: C := alpha A B + beta C (side L)
 * or alpha B A + beta C (side R), A by symValue with herm (zsymm_ herm = false,
 * zhemm_ herm = true, fortran.zig:785-799). */
#define DEFINE_CX_SYMM(NAME, CT)                                                                     \
    void NAME(char side, char uplo, blas_int m, blas_int n, const CT *alpha, const CT *a, blas_int lda, \
              const CT *b, blas_int ldb, const CT *beta, CT *c, blas_int ldc, int herm) {             \
        side = (char)upc(side); uplo = (char)upc(uplo);                                              \
        if (m <= 0 || n <= 0) return;                                                                \
        CT zero = {0, 0};                                                                            \
        for (size_t j = 0; j < (size_t)n; ++j)                                                       \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                 \
                CT sum = zero;                                                                       \
                if (side == 'L') {                                                                   \
                    for (size_t p = 0; p < (size_t)m; ++p)                                           \
                        sum = CT##_add(sum, CT##_mul(CT##_symval(uplo, a, lda, i, p, herm), b[ix(ldb, p, j)])); \
                } else {                                                                             \
                    for (size_t p = 0; p < (size_t)n; ++p)                                           \
                        sum = CT##_add(sum, CT##_mul(b[ix(ldb, i, p)], CT##_symval(uplo, a, lda, p, j, herm))); \
                }                                                                                    \
                size_t q = ix(ldc, i, j);                                                            \
                c[q] = CT##_add(CT##_mul(*alpha, sum), CT##_is_zero(*beta) ? zero : CT##_mul(*beta, c[q])); \
            }                                                                                        \
    }

DEFINE_CX_SYMM(oracle_zsymm, cxd)
DEFINE_CX_SYMM(oracle_csymm, cxf)

/* triangular.zig:202-231 trmm for complex types: left side trmv per column
 * (op = C conjugates, triValue access.zig:54-64) then alpha when alpha != 1;
 * right side per row, columns in the order that keeps later inputs intact. */
#define DEFINE_CX_TRMM(NAME, CT)                                                                        \
    void NAME(char side, char uplo, char trans, char diag, blas_int m, blas_int n, const CT *alpha,   \
              const CT *a, blas_int lda, CT *b, blas_int ldb) {                                         \
        side = (char)upc(side); uplo = (char)upc(uplo); trans = (char)upc(trans); diag = (char)upc(diag); \
        if (m <= 0 || n <= 0) return;                                                                   \
        int upper = op_is_upper(uplo, trans);                                                           \
        CT zero = {0, 0};                                                                               \
        if (side == 'L') {                                                                              \
            for (size_t j = 0; j < (size_t)n; ++j) {                                                    \
                CT *x = b + (size_t)ldb * j;                                                            \
                if (upper) {                                                                            \
                    for (size_t r = 0; r < (size_t)m; ++r) {                                            \
                        CT t = zero;                                                                    \
                        for (size_t q = r; q < (size_t)m; ++q)                                          \
                            t = CT##_add(t, CT##_mul(CT##_tri(uplo, diag, trans, a, lda, r, q), x[q])); \
                        x[r] = t;                                                                       \
                    }                                                                                   \
                } else {                                                                                \
                    for (size_t r = (size_t)m; r-- > 0;) {                                              \
                        CT t = zero;                                                                    \
                        for (size_t q = 0; q <= r; ++q)                                                 \
                            t = CT##_add(t, CT##_mul(CT##_tri(uplo, diag, trans, a, lda, r, q), x[q])); \
                        x[r] = t;                                                                       \
                    }                                                                                   \
                }                                                                                       \
                if (!CT##_is_one(*alpha))                                                               \
                    for (size_t r = 0; r < (size_t)m; ++r) x[r] = CT##_mul(*alpha, x[r]);               \
            }                                                                                           \
        } else {                                                                                        \
            for (size_t i = 0; i < (size_t)m; ++i) {                                                    \
                for (size_t s = 0; s < (size_t)n; ++s) {                                                \
                    size_t cc = upper ? (size_t)n - 1 - s : s;                                          \
                    CT sum = zero;                                                                      \
                    for (size_t p = 0; p < (size_t)n; ++p)                                              \
                        sum = CT##_add(sum, CT##_mul(b[ix(ldb, i, p)], CT##_tri(uplo, diag, trans, a, lda, p, cc))); \
                    b[ix(ldb, i, cc)] = CT##_mul(*alpha, sum);                                          \
                }                                                                                       \
            }                                                                                           \
        }                                                                                               \
    }

DEFINE_CX_TRMM(oracle_ztrmm, cxd)
DEFINE_CX_TRMM(oracle_ctrmm, cxf)

/* symmetric.zig:180-199 runSyrkColumns with herm = true (zherk_ / cherk_,
 * fortran.zig:818-825: alpha and beta real, widened by realScalar): sum of
 * op(A)(i, p) conj(op(A)(j, p)), C := alpha sum + beta C, diagonal made real. */
#define DEFINE_CX_HERK(NAME, CT, R)                                                                  \
    void NAME(char uplo, char trans, blas_int n, blas_int k, R alpha_r, const CT *a, blas_int lda,  \
              R beta_r, CT *c, blas_int ldc) {                                                       \
        uplo = (char)upc(uplo); trans = (char)upc(trans);                                            \
        if (n <= 0) return;                                                                          \
        CT alpha = {alpha_r, 0}, beta = {beta_r, 0}, zero = {0, 0};                                  \
        for (size_t j = 0; j < (size_t)n; ++j) {                                                     \
            size_t r0 = (uplo == 'U') ? 0 : j, r1 = (uplo == 'U') ? j + 1 : (size_t)n;               \
            for (size_t i = r0; i < r1; ++i) {                                                       \
                CT sum = zero;                                                                       \
                for (size_t p = 0; p < (size_t)(k > 0 ? k : 0); ++p)                                  \
                    sum = CT##_add(sum, CT##_mul(CT##_opval(trans, a, lda, i, p),                    \
                                                 CT##_conj(CT##_opval(trans, a, lda, j, p))));       \
                size_t q = ix(ldc, i, j);                                                            \
                c[q] = CT##_add(CT##_mul(alpha, sum), CT##_is_zero(beta) ? zero : CT##_mul(beta, c[q])); \
                if (i == j) c[q].im = 0;                                                             \
            }                                                                                        \
        }                                                                                            \
    }

DEFINE_CX_HERK(oracle_zherk, cxd, double)
DEFINE_CX_HERK(oracle_cherk, cxf, float)

/* symmetric.zig:301-329 runSyr2kColumns for complex types: herm = false sums
 * a_i b_j + b_i a_j and scales by alpha; herm = true sums alpha a_i conj(b_j) +
 * conj(alpha) b_i conj(a_j) and makes the diagonal real (zher2k_ beta is real,
 * fortran.zig:843-849). */
#define DEFINE_CX_SYR2K(NAME, CT)                                                                       \
    void NAME(char uplo, char trans, blas_int n, blas_int k, const CT *alpha, const CT *a, blas_int lda, \
              const CT *b, blas_int ldb, const CT *beta, CT *c, blas_int ldc, int herm) {                \
        uplo = (char)upc(uplo); trans = (char)upc(trans);                                               \
        if (n <= 0) return;                                                                             \
        CT zero = {0, 0};                                                                               \
        for (size_t j = 0; j < (size_t)n; ++j) {                                                        \
            size_t r0 = (uplo == 'U') ? 0 : j, r1 = (uplo == 'U') ? j + 1 : (size_t)n;                  \
            for (size_t i = r0; i < r1; ++i) {                                                          \
                CT sum = zero;                                                                          \
                for (size_t p = 0; p < (size_t)(k > 0 ? k : 0); ++p) {                                   \
                    CT ai = CT##_opval(trans, a, lda, i, p), bi = CT##_opval(trans, b, ldb, i, p);      \
                    CT aj = CT##_opval(trans, a, lda, j, p), bj = CT##_opval(trans, b, ldb, j, p);      \
                    if (herm) {                                                                         \
                        aj = CT##_conj(aj); bj = CT##_conj(bj);                                         \
                        sum = CT##_add(sum, CT##_add(CT##_mul(*alpha, CT##_mul(ai, bj)),                \
                                                     CT##_mul(CT##_conj(*alpha), CT##_mul(bi, aj))));   \
                    } else {                                                                            \
                        sum = CT##_add(sum, CT##_add(CT##_mul(ai, bj), CT##_mul(bi, aj)));              \
                    }                                                                                   \
                }                                                                                       \
                size_t q = ix(ldc, i, j);                                                               \
                CT prod = herm ? sum : CT##_mul(*alpha, sum);                                           \
                c[q] = CT##_add(prod, CT##_is_zero(*beta) ? zero : CT##_mul(*beta, c[q]));              \
                if (herm && i == j) c[q].im = 0;                                                        \
            }                                                                                           \
        }                                                                                               \
    }

DEFINE_CX_SYR2K(oracle_zsyr2k, cxd)
DEFINE_CX_SYR2K(oracle_csyr2k, cxf)

/* Library self-identification for the loader in the tests. */
int oracle_version(void) { return 1; }
