/*
 * zynum_blas_gpu.h — C ABI of the B200 GEMM backend for Zynum BLAS.
 *
 * The Fortran and CBLAS entry points have exactly the signatures, argument
 * checks, error reports and quick returns of the reference library's exports,
 * so a program linked against libzynum_blas can link against
 * libzynum_blas_gpu.so instead.  Each declaration cites the reference export
 * it replaces (paths inside the Zynum project).
 *
 * Host entry points take HOST pointers, stage them to the GPU, compute there
 * and copy the result window back; padding rows [m, ldc) of C are never
 * written.  The *_device entry points take DEVICE pointers and a CUDA stream
 * (as `void *`, a cudaStream_t), enqueue the work and return a status:
 *   0              success (work enqueued),
 *   1 .. 13        index of the first illegal argument (same numbering as the
 *                  Fortran routine; nothing was enqueued),
 *   < 0            a CUDA error (negated cudaError_t); zynum_blas_gpu_last_error()
 *                  gives the text.
 */
#ifndef ZYNUM_BLAS_GPU_H
#define ZYNUM_BLAS_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ZYNUM_BLAS_GPU_API __attribute__((visibility("default")))
#else
#define ZYNUM_BLAS_GPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t zynum_blas_int; /* BlasInt = i32: src/blas/types.zig:4; include/zynum/blas/cblas.h:18 */

/* ------------------------------------------------------------- Fortran ABI */

/* src/blas/abi/fortran.zig:20 xerbla_ — prints
 * " ** On entry to NAME parameter number N had an illegal value". */
ZYNUM_BLAS_GPU_API void xerbla_(const char *srname, const zynum_blas_int *info);
/* src/blas/abi/fortran.zig:16 lsame_ */
ZYNUM_BLAS_GPU_API int lsame_(const char *ca, const char *cb);
/* src/blas/abi/fortran.zig:41-47 zynum_blas_shutdown(_) — also frees every GPU buffer of the shim. */
ZYNUM_BLAS_GPU_API void zynum_blas_shutdown(void);
ZYNUM_BLAS_GPU_API void zynum_blas_shutdown_(void);

/* src/blas/abi/fortran.zig:760 sgemm_ */
ZYNUM_BLAS_GPU_API void sgemm_(const char *transa, const char *transb, const zynum_blas_int *m, const zynum_blas_int *n,
            const zynum_blas_int *k, const float *alpha, const float *a, const zynum_blas_int *lda, const float *b,
            const zynum_blas_int *ldb, const float *beta, float *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:764 dgemm_ */
ZYNUM_BLAS_GPU_API void dgemm_(const char *transa, const char *transb, const zynum_blas_int *m, const zynum_blas_int *n,
            const zynum_blas_int *k, const double *alpha, const double *a, const zynum_blas_int *lda,
            const double *b, const zynum_blas_int *ldb, const double *beta, double *c, const zynum_blas_int *ldc);

/* src/blas/abi/fortran.zig:768 cgemm_ (alpha, beta, a, b, c: interleaved single-precision complex) */
ZYNUM_BLAS_GPU_API void cgemm_(const char *transa, const char *transb, const zynum_blas_int *m, const zynum_blas_int *n,
            const zynum_blas_int *k, const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
            const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:772 zgemm_ (interleaved double-precision complex) */
ZYNUM_BLAS_GPU_API void zgemm_(const char *transa, const char *transb, const zynum_blas_int *m, const zynum_blas_int *n,
            const zynum_blas_int *k, const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
            const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);

/* src/blas/abi/fortran.zig:869-883 strsm_ / dtrsm_ (B := alpha op(A)^-1 B or B op(A)^-1) */
ZYNUM_BLAS_GPU_API void strsm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const float *alpha, const float *a,
                               const zynum_blas_int *lda, float *b, const zynum_blas_int *ldb);
ZYNUM_BLAS_GPU_API void dtrsm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const double *alpha, const double *a,
                               const zynum_blas_int *lda, double *b, const zynum_blas_int *ldb);
/* src/blas/abi/fortran.zig:802-809 ssyrk_ / dsyrk_ (C := alpha op(A) op(A)^T + beta C, one triangle) */
ZYNUM_BLAS_GPU_API void ssyrk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const float *alpha, const float *a, const zynum_blas_int *lda, const float *beta,
                               float *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void dsyrk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const double *alpha, const double *a, const zynum_blas_int *lda, const double *beta,
                               double *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:877-884 ctrsm_ / ztrsm_ (interleaved complex; op = C conjugates) */
ZYNUM_BLAS_GPU_API void ctrsm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const void *alpha, const void *a,
                               const zynum_blas_int *lda, void *b, const zynum_blas_int *ldb);
ZYNUM_BLAS_GPU_API void ztrsm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const void *alpha, const void *a,
                               const zynum_blas_int *lda, void *b, const zynum_blas_int *ldb);
/* src/blas/abi/fortran.zig:810-817 csyrk_ / zsyrk_ (C := alpha op(A) op(A)^T + beta C, one triangle) */
ZYNUM_BLAS_GPU_API void csyrk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *beta, void *c,
                               const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zsyrk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *beta, void *c,
                               const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:785-799 csymm_ / zsymm_ / chemm_ / zhemm_ (A symmetric, or Hermitian:
 * the unstored triangle is the conjugate mirror and the diagonal's imaginary part is ignored) */
ZYNUM_BLAS_GPU_API void csymm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                               const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zsymm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                               const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void chemm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                               const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zhemm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                               const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:818-825 cherk_ / zherk_ (C := alpha op(A) op(A)^H + beta C, alpha and beta real) */
ZYNUM_BLAS_GPU_API void cherk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const float *alpha, const void *a, const zynum_blas_int *lda, const float *beta,
                               void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zherk_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                               const double *alpha, const void *a, const zynum_blas_int *lda, const double *beta,
                               void *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:835-849 csyr2k_ / zsyr2k_ (C := alpha (op(A) op(B)^T + op(B) op(A)^T) + beta C),
 * cher2k_ / zher2k_ (C := alpha op(A) op(B)^H + conj(alpha) op(B) op(A)^H + beta C, beta real) */
ZYNUM_BLAS_GPU_API void csyr2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                                const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zsyr2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                                const zynum_blas_int *ldb, const void *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void cher2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                                const zynum_blas_int *ldb, const float *beta, void *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void zher2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const void *alpha, const void *a, const zynum_blas_int *lda, const void *b,
                                const zynum_blas_int *ldb, const double *beta, void *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:860-867 ctrmm_ / ztrmm_ (B := alpha op(A) B or alpha B op(A), op = C conjugates) */
ZYNUM_BLAS_GPU_API void ctrmm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const void *alpha, const void *a,
                               const zynum_blas_int *lda, void *b, const zynum_blas_int *ldb);
ZYNUM_BLAS_GPU_API void ztrmm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const void *alpha, const void *a,
                               const zynum_blas_int *lda, void *b, const zynum_blas_int *ldb);
/* src/blas/abi/fortran.zig:777-783 ssymm_ / dsymm_ (C := alpha A B + beta C or alpha B A + beta C, A symmetric) */
ZYNUM_BLAS_GPU_API void ssymm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const float *alpha, const float *a, const zynum_blas_int *lda, const float *b,
                               const zynum_blas_int *ldb, const float *beta, float *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void dsymm_(const char *side, const char *uplo, const zynum_blas_int *m, const zynum_blas_int *n,
                               const double *alpha, const double *a, const zynum_blas_int *lda, const double *b,
                               const zynum_blas_int *ldb, const double *beta, double *c, const zynum_blas_int *ldc);
/* src/blas/abi/fortran.zig:852-858 strmm_ / dtrmm_ (B := alpha op(A) B or alpha B op(A), A triangular) */
ZYNUM_BLAS_GPU_API void strmm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const float *alpha, const float *a,
                               const zynum_blas_int *lda, float *b, const zynum_blas_int *ldb);
ZYNUM_BLAS_GPU_API void dtrmm_(const char *side, const char *uplo, const char *transa, const char *diag,
                               const zynum_blas_int *m, const zynum_blas_int *n, const double *alpha, const double *a,
                               const zynum_blas_int *lda, double *b, const zynum_blas_int *ldb);
/* src/blas/abi/fortran.zig:827-833 ssyr2k_ / dsyr2k_ (C := alpha (op(A) op(B)^T + op(B) op(A)^T) + beta C, one triangle) */
ZYNUM_BLAS_GPU_API void ssyr2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const float *alpha, const float *a, const zynum_blas_int *lda, const float *b,
                                const zynum_blas_int *ldb, const float *beta, float *c, const zynum_blas_int *ldc);
ZYNUM_BLAS_GPU_API void dsyr2k_(const char *uplo, const char *trans, const zynum_blas_int *n, const zynum_blas_int *k,
                                const double *alpha, const double *a, const zynum_blas_int *lda, const double *b,
                                const zynum_blas_int *ldb, const double *beta, double *c, const zynum_blas_int *ldc);

/* ---------------------------------------------------------------- CBLAS ABI */

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };          /* cblas.zig:123-124 */
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 }; /* :125-127 */
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };                  /* :128-129 */
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };                 /* :130-131 */
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };                   /* :132-133 */

/* src/blas/abi/cblas.zig:1415 cblas_sgemm */
ZYNUM_BLAS_GPU_API void cblas_sgemm(int layout, int transa, int transb, int m, int n, int k, float alpha, const float *a, int lda,
                 const float *b, int ldb, float beta, float *c, int ldc);
/* src/blas/abi/cblas.zig:1428 cblas_dgemm */
ZYNUM_BLAS_GPU_API void cblas_dgemm(int layout, int transa, int transb, int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);

/* src/blas/abi/cblas.zig:1441 cblas_cgemm */
ZYNUM_BLAS_GPU_API void cblas_cgemm(int layout, int transa, int transb, int m, int n, int k, const void *alpha, const void *a,
                 int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
/* src/blas/abi/cblas.zig:1454 cblas_zgemm */
ZYNUM_BLAS_GPU_API void cblas_zgemm(int layout, int transa, int transb, int m, int n, int k, const void *alpha, const void *a,
                 int lda, const void *b, int ldb, const void *beta, void *c, int ldc);

/* src/blas/abi/cblas.zig:1729-1756 cblas_strsm / cblas_dtrsm */
ZYNUM_BLAS_GPU_API void cblas_strsm(int layout, int side, int uplo, int transa, int diag, int m, int n, float alpha,
                                    const float *a, int lda, float *b, int ldb);
ZYNUM_BLAS_GPU_API void cblas_dtrsm(int layout, int side, int uplo, int transa, int diag, int m, int n, double alpha,
                                    const double *a, int lda, double *b, int ldb);
/* src/blas/abi/cblas.zig:1539-1560 cblas_ssyrk / cblas_dsyrk */
ZYNUM_BLAS_GPU_API void cblas_ssyrk(int layout, int uplo, int trans, int n, int k, float alpha, const float *a,
                                    int lda, float beta, float *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_dsyrk(int layout, int uplo, int trans, int n, int k, double alpha, const double *a,
                                    int lda, double beta, double *c, int ldc);
/* src/blas/abi/cblas.zig:1755-1779 cblas_ctrsm / cblas_ztrsm (alpha by pointer) */
ZYNUM_BLAS_GPU_API void cblas_ctrsm(int layout, int side, int uplo, int transa, int diag, int m, int n,
                                    const void *alpha, const void *a, int lda, void *b, int ldb);
ZYNUM_BLAS_GPU_API void cblas_ztrsm(int layout, int side, int uplo, int transa, int diag, int m, int n,
                                    const void *alpha, const void *a, int lda, void *b, int ldb);
/* src/blas/abi/cblas.zig:1560-1582 cblas_csyrk / cblas_zsyrk (alpha / beta by pointer) */
ZYNUM_BLAS_GPU_API void cblas_csyrk(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                    int lda, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zsyrk(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                    int lda, const void *beta, void *c, int ldc);
/* src/blas/abi/cblas.zig:1491-1537 cblas_csymm / cblas_zsymm / cblas_chemm / cblas_zhemm (scalars by pointer) */
ZYNUM_BLAS_GPU_API void cblas_csymm(int layout, int side, int uplo, int m, int n, const void *alpha, const void *a,
                                    int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zsymm(int layout, int side, int uplo, int m, int n, const void *alpha, const void *a,
                                    int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_chemm(int layout, int side, int uplo, int m, int n, const void *alpha, const void *a,
                                    int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zhemm(int layout, int side, int uplo, int m, int n, const void *alpha, const void *a,
                                    int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
/* src/blas/abi/cblas.zig:1583-1603 cblas_cherk / cblas_zherk (alpha, beta real, by value) */
ZYNUM_BLAS_GPU_API void cblas_cherk(int layout, int uplo, int trans, int n, int k, float alpha, const void *a,
                                    int lda, float beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zherk(int layout, int uplo, int trans, int n, int k, double alpha, const void *a,
                                    int lda, double beta, void *c, int ldc);
/* src/blas/abi/cblas.zig:1629-1676 cblas_csyr2k / cblas_zsyr2k, cblas_cher2k / cblas_zher2k (beta real, by value) */
ZYNUM_BLAS_GPU_API void cblas_csyr2k(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                     int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zsyr2k(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                     int lda, const void *b, int ldb, const void *beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_cher2k(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                     int lda, const void *b, int ldb, float beta, void *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_zher2k(int layout, int uplo, int trans, int n, int k, const void *alpha, const void *a,
                                     int lda, const void *b, int ldb, double beta, void *c, int ldc);
/* src/blas/abi/cblas.zig:1703-1728 cblas_ctrmm / cblas_ztrmm (alpha by pointer) */
ZYNUM_BLAS_GPU_API void cblas_ctrmm(int layout, int side, int uplo, int transa, int diag, int m, int n,
                                    const void *alpha, const void *a, int lda, void *b, int ldb);
ZYNUM_BLAS_GPU_API void cblas_ztrmm(int layout, int side, int uplo, int transa, int diag, int m, int n,
                                    const void *alpha, const void *a, int lda, void *b, int ldb);
/* src/blas/abi/cblas.zig:1467-1489 cblas_ssymm / cblas_dsymm */
ZYNUM_BLAS_GPU_API void cblas_ssymm(int layout, int side, int uplo, int m, int n, float alpha, const float *a, int lda,
                                    const float *b, int ldb, float beta, float *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_dsymm(int layout, int side, int uplo, int m, int n, double alpha, const double *a,
                                    int lda, const double *b, int ldb, double beta, double *c, int ldc);
/* src/blas/abi/cblas.zig:1677-1701 cblas_strmm / cblas_dtrmm */
ZYNUM_BLAS_GPU_API void cblas_strmm(int layout, int side, int uplo, int transa, int diag, int m, int n, float alpha,
                                    const float *a, int lda, float *b, int ldb);
ZYNUM_BLAS_GPU_API void cblas_dtrmm(int layout, int side, int uplo, int transa, int diag, int m, int n, double alpha,
                                    const double *a, int lda, double *b, int ldb);
/* src/blas/abi/cblas.zig:1605-1627 cblas_ssyr2k / cblas_dsyr2k */
ZYNUM_BLAS_GPU_API void cblas_ssyr2k(int layout, int uplo, int trans, int n, int k, float alpha, const float *a,
                                     int lda, const float *b, int ldb, float beta, float *c, int ldc);
ZYNUM_BLAS_GPU_API void cblas_dsyr2k(int layout, int uplo, int trans, int n, int k, double alpha, const double *a,
                                     int lda, const double *b, int ldb, double beta, double *c, int ldc);

/* ------------------------------------------------------ GPU device entry points
 * Added by the GPU backend (no counterpart in the reference's ABI; the planned
 * addition is described for src/blas/abi/fortran.zig's dgemm_ path).  Same
 * argument meaning as dgemm_/sgemm_, passed by value, device pointers. */

/* Native FP64 (DMMA tensor pipe) or Ozaki-emulated DGEMM, chosen by
 * zynum_blas_gpu_set_dgemm_method / ZYNUM_GPU_DGEMM_METHOD (default native). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dgemm_device(char transa, char transb, int m, int n, int k, double alpha, const double *a,
                                int lda, const double *b, int ldb, double beta, double *c, int ldc, void *stream);
/* Native FP32 (FFMA), 3xBF16 or INT8 CRT SGEMM, chosen by zynum_blas_gpu_set_sgemm_method. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_sgemm_device(char transa, char transb, int m, int n, int k, float alpha, const float *a, int lda,
                                const float *b, int ldb, float beta, float *c, int ldc, void *stream);

/* Allocation-free DGEMM (no counterpart in the reference: an addition of the
 * GPU backend).  For callers that cannot let the library call cudaMalloc —
 * code whose device memory belongs to its own pool allocator, or latency-
 * critical loops where cudaMalloc/cudaFree would synchronise the device.
 * Same arguments and result as zynum_blas_gpu_dgemm_device with the native
 * method (the Ozaki method setting does not apply here); `splits` > 0 forces
 * that many split-K ranges (at most 64), 0 lets the planner choose.  Split-K
 * partial sums go to a fixed 32 MiB device array inside the library, so the
 * partial sums of the K ranges the call really uses (splits * m * n; none on
 * the tall-skinny route) must not exceed 4194304 doubles; larger requests are
 * rejected with a negative status and a message in zynum_blas_gpu_last_error().
 * The array's memory is committed on a GPU when the library's module for it
 * loads there: with CUDA's lazy module loading (the default) that is the
 * first call on that GPU, which also looks up the array's device address and
 * checks that the GPU is an sm_100 part.  So make one call per GPU before
 * reserving a memory pool and before any stream capture; later calls on that
 * GPU allocate nothing.  All calls share the one array: calls that overlap on
 * the GPU (other streams, other threads) race on it. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dgemm_noalloc_device(char transa, char transb, int m, int n, int k, double alpha,
                                                           const double *a, int lda, const double *b, int ldb,
                                                           double beta, double *c, int ldc, int splits, void *stream);

/* Complex GEMM through real GEMMs (expanded-real 4M or 3M, zynum_blas_gpu_set_complex_method);
 * alpha / beta point to HOST (re, im) pairs, matrices are device pointers. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zgemm_device(char transa, char transb, int m, int n, int k, const double *alpha,
                                                   const double *a, int lda, const double *b, int ldb,
                                                   const double *beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_cgemm_device(char transa, char transb, int m, int n, int k, const float *alpha,
                                                   const float *a, int lda, const float *b, int ldb, const float *beta,
                                                   float *c, int ldc, void *stream);

/* TRSM on device pointers: blocked, inverted 64 x 64 diagonal blocks + GEMM updates
 * (the GEMMs follow the DGEMM / SGEMM method).  Argument numbering as dtrsm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dtrsm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   double alpha, const double *a, int lda, double *b, int ldb,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_strsm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   float alpha, const float *a, int lda, float *b, int ldb,
                                                   void *stream);
/* Several FP64 solves with one triangular matrix.  The reference has no
 * counterpart (its trsm, triangular.zig:233, keeps no state between calls):
 * zynum_blas_gpu_dtrsm_device inverts the diagonal blocks of A on every call;
 * these two split that work off so that callers solving repeatedly with the
 * same A (forward and adjoint solves, batches of right-hand sides arriving
 * one after another) form it once.
 * dtrsm_inverse_bytes(n): size of the buffer for an n x n A (0 when n <= 0).
 * dtrsm_inverse_device: inv := the inverses of A's 256-row diagonal blocks
 *   (uplo, diag as for dtrsm_; A a 16-byte aligned device pointer with an
 *   even lda, else -cudaErrorInvalidValue; positive returns number the bad
 *   argument: 1 uplo, 2 diag, 3 n, 5 lda, 6 inv).
 * dtrsm_with_inverse_device: dtrsm_device with those inverses instead of
 *   forming them; inv must come from dtrsm_inverse_device on the same A, uplo,
 *   diag and order (m for side L, n for side R), unchanged since; side and
 *   transa are free.  Argument numbering as dtrsm_, 12 for inv. */
ZYNUM_BLAS_GPU_API size_t zynum_blas_gpu_dtrsm_inverse_bytes(int n);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dtrsm_inverse_device(char uplo, char diag, int n, const double *a, int lda,
                                                           double *inv, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dtrsm_with_inverse_device(char side, char uplo, char transa, char diag, int m,
                                                                int n, double alpha, const double *a, int lda,
                                                                double *b, int ldb, const double *inv, void *stream);
/* SYRK on device pointers: the native GEMM tiles in triangle mode.  Argument numbering as dsyrk_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dsyrk_device(char uplo, char trans, int n, int k, double alpha, const double *a,
                                                   int lda, double beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ssyrk_device(char uplo, char trans, int n, int k, float alpha, const float *a,
                                                   int lda, float beta, float *c, int ldc, void *stream);
/* Complex TRSM on device pointers (interleaved complex; alpha points to re, im): the recursive solve with
 * complex GEMM couplings (4M / 3M per the complex method).  Argument numbering as ztrsm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ztrsm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   const double *alpha, const double *a, int lda, double *b, int ldb,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ctrsm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   const float *alpha, const float *a, int lda, float *b, int ldb,
                                                   void *stream);
/* Complex SYRK on device pointers: one complex GEMM into scratch and a triangle update.  Argument
 * numbering as zsyrk_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zsyrk_device(char uplo, char trans, int n, int k, const double *alpha,
                                                   const double *a, int lda, const double *beta, double *c, int ldc,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_csyrk_device(char uplo, char trans, int n, int k, const float *alpha,
                                                   const float *a, int lda, const float *beta, float *c, int ldc,
                                                   void *stream);
/* Complex SYMM / HEMM on device pointers (interleaved complex; alpha, beta point to re, im): the stored
 * triangle mirrored (conjugated for HEMM, real diagonal) into scratch, one complex GEMM.  Argument
 * numbering as zsymm_ / zhemm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zsymm_device(char side, char uplo, int m, int n, const double *alpha,
                                                   const double *a, int lda, const double *b, int ldb,
                                                   const double *beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zhemm_device(char side, char uplo, int m, int n, const double *alpha,
                                                   const double *a, int lda, const double *b, int ldb,
                                                   const double *beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_csymm_device(char side, char uplo, int m, int n, const float *alpha,
                                                   const float *a, int lda, const float *b, int ldb,
                                                   const float *beta, float *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_chemm_device(char side, char uplo, int m, int n, const float *alpha,
                                                   const float *a, int lda, const float *b, int ldb,
                                                   const float *beta, float *c, int ldc, void *stream);
/* Complex TRMM on device pointers (op = C conjugates).  Argument numbering as ztrmm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ztrmm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   const double *alpha, const double *a, int lda, double *b, int ldb,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ctrmm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   const float *alpha, const float *a, int lda, float *b, int ldb,
                                                   void *stream);
/* Complex SYR2K / HER2K / HERK on device pointers: one complex GEMM into scratch and a triangle update
 * (HER2K: beta real; HERK: alpha and beta real, diagonal made real).  Argument numbering as zsyr2k_,
 * zher2k_, zherk_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zsyr2k_device(char uplo, char trans, int n, int k, const double *alpha,
                                                    const double *a, int lda, const double *b, int ldb,
                                                    const double *beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zher2k_device(char uplo, char trans, int n, int k, const double *alpha,
                                                    const double *a, int lda, const double *b, int ldb, double beta,
                                                    double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_zherk_device(char uplo, char trans, int n, int k, double alpha, const double *a,
                                                   int lda, double beta, double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_csyr2k_device(char uplo, char trans, int n, int k, const float *alpha,
                                                    const float *a, int lda, const float *b, int ldb,
                                                    const float *beta, float *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_cher2k_device(char uplo, char trans, int n, int k, const float *alpha,
                                                    const float *a, int lda, const float *b, int ldb, float beta,
                                                    float *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_cherk_device(char uplo, char trans, int n, int k, float alpha, const float *a,
                                                   int lda, float beta, float *c, int ldc, void *stream);
/* SYMM on device pointers: the stored triangle of A is mirrored into a dense scratch copy, then one
 * GEMM (following the DGEMM / SGEMM method).  Argument numbering as dsymm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dsymm_device(char side, char uplo, int m, int n, double alpha, const double *a,
                                                   int lda, const double *b, int ldb, double beta, double *c, int ldc,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ssymm_device(char side, char uplo, int m, int n, float alpha, const float *a,
                                                   int lda, const float *b, int ldb, float beta, float *c, int ldc,
                                                   void *stream);
/* TRMM on device pointers: dense 256 x 256 diagonal blocks + off-diagonal GEMMs on a copy of B
 * (following the DGEMM / SGEMM method).  Argument numbering as dtrmm_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dtrmm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   double alpha, const double *a, int lda, double *b, int ldb,
                                                   void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_strmm_device(char side, char uplo, char transa, char diag, int m, int n,
                                                   float alpha, const float *a, int lda, float *b, int ldb,
                                                   void *stream);
/* SYR2K on device pointers: two native triangle-mode GEMMs.  Argument numbering as dsyr2k_. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dsyr2k_device(char uplo, char trans, int n, int k, double alpha,
                                                    const double *a, int lda, const double *b, int ldb, double beta,
                                                    double *c, int ldc, void *stream);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ssyr2k_device(char uplo, char trans, int n, int k, float alpha, const float *a,
                                                    int lda, const float *b, int ldb, float beta, float *c, int ldc,
                                                    void *stream);

/* Triangle-restricted GEMM ("gemmt"; no counterpart in the reference, used by
 * the TRSM adjoint): C := alpha op(A) op(B) + beta C computed and written only
 * on the uplo triangle of the n x n matrix C (A: n x k after op, B: k x n).
 * Argument numbering: uplo 1, transa 2, transb 3, n 4, k 5, lda 8, ldb 10, ldc 13. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dgemmt_device(char uplo, char transa, char transb, int n, int k, double alpha,
                                                    const double *a, int lda, const double *b, int ldb, double beta,
                                                    double *c, int ldc, void *stream);
/* Copy the uplo triangle of an n x n device matrix onto the other triangle
 * (turns a SYRK result into the full symmetric matrix). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dsymmetrize_device(char uplo, int n, double *c, int ldc, void *stream);

/* ------------------------------------------------- variable-size batches
 * No counterpart in the reference (Zynum has no batched API).  A batch plan is
 * created once from HOST arrays of problem sizes; running it is one
 * persistent-kernel launch, preceded by a 4-byte reset of the plan's work
 * counter (or a replay of a CUDA graph holding both when use_graph != 0), with
 * no allocation.  Runs of one plan must not overlap on the GPU (they share its
 * work counter); separate plans may.  The per-problem operand arrays
 * passed to *_run (pointers and leading dimensions) are DEVICE arrays with one
 * entry per problem.  dtype: 0 = FP64, 1 = FP32.  Create returns 0 or the
 * index of the first illegal argument; run returns 0 or a negated CUDA error. */
typedef struct zynum_blas_gpu_batch *zynum_blas_gpu_batch_t;
/* GEMM batch: C_q = alpha op(A_q) op(B_q) + beta C_q with m[q] x n[q] x k[q] sizes and
 * the same transposes.  tune != 0 times the candidate tile configs of every size
 * bucket not yet in the tuning table (kept in the JSON file ZYNUM_GPU_TUNE_CACHE names). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_gemm_batch_create(zynum_blas_gpu_batch_t *out, int dtype, char transa,
                                                        char transb, int count, const int *m, const int *n,
                                                        const int *k, int tune);
/* Left-side TRSM batch: B_q (m[q] x n[q], n[q] <= 64) := alpha op(A_q)^-1 B_q, A_q m[q] x m[q] triangular. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_trsm_batch_create(zynum_blas_gpu_batch_t *out, int dtype, char side, char uplo,
                                                        char transa, char diag, int count, const int *m,
                                                        const int *n);
ZYNUM_BLAS_GPU_API void zynum_blas_gpu_batch_destroy(zynum_blas_gpu_batch_t batch);
/* Number of scheduled work items, persistent grid size and tiles per config (32, 64, 128). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_batch_info(zynum_blas_gpu_batch_t batch, int *items, int *grid, int *cfg_counts);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dgemm_batch_run(zynum_blas_gpu_batch_t batch, double alpha,
                                                      const double *const *a, const int *lda, const double *const *b,
                                                      const int *ldb, double beta, double *const *c, const int *ldc,
                                                      void *stream, int use_graph);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_sgemm_batch_run(zynum_blas_gpu_batch_t batch, float alpha, const float *const *a,
                                                      const int *lda, const float *const *b, const int *ldb,
                                                      float beta, float *const *c, const int *ldc, void *stream,
                                                      int use_graph);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_dtrsm_batch_run(zynum_blas_gpu_batch_t batch, double alpha,
                                                      const double *const *a, const int *lda, double *const *b,
                                                      const int *ldb, void *stream, int use_graph);
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_strsm_batch_run(zynum_blas_gpu_batch_t batch, float alpha, const float *const *a,
                                                      const int *lda, float *const *b, const int *ldb, void *stream,
                                                      int use_graph);

/* -------------------------------------------------------------- control */
/* 0 = expanded-real 4M (one real GEMM of 2m x n x 2k), 1 = 3M (three real GEMMs). Returns the previous value. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_complex_method(int method);
/* 0 = native FP64, 1 = Ozaki INT8 emulation, 2 = automatic. Returns the previous value. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_dgemm_method(int method);
/* 0 = native FP32, 1 = 3xBF16 split product (about 16 bits), 2 = INT8 CRT
 * emulation (exact integer products, one rounding to FP32).  Returns the previous value. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_sgemm_method(int method);
/* Ozaki slice count (2..12), 0 = automatic. Returns the previous value. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_ozaki_slices(int slices);
/* Ozaki scheme: 0 = automatic (CRT residues unless a slice count is set or
 * K > 130816), 1 = INT8 slices (Ozaki scheme I), 2 = CRT residues (Ozaki
 * scheme II; slices beyond K = 130816).  Returns the previous value.
 * No reference counterpart (the reference has no emulated DGEMM). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_ozaki_scheme(int scheme);
/* CRT moduli (2..16), 0 = default (16).  Returns the previous value. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_set_ozaki_moduli(int moduli);
/* Scheme (1 slices, 2 CRT), digit count (slices, or moduli) and INT8 product
 * GEMM count (s(s+1)/2 slice products, or one per modulus) the Ozaki method
 * uses for an m x n x k DGEMM under the current settings; with automatic
 * slices: the count the most recent slice-scheme call chose from its data. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ozaki_plan_ex(int m, int n, int k, int *scheme, int *digits, int *products);
/* zynum_blas_gpu_ozaki_plan_ex without the scheme. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_ozaki_plan(int m, int n, int k, int *slices, int *products);
/* Text of the last error seen by this thread ("" if none). */
ZYNUM_BLAS_GPU_API const char *zynum_blas_gpu_last_error(void);
/* Host-side fault injection for tests: the next `count` device-memory
 * reservations fail (kind 1), the next stream synchronisation reports
 * CUDA error `count` (kind 2), or the next `count` Ozaki DGEMM product
 * kernels run with a hold (kind 3): their MMA issuer first waits on a
 * barrier that nothing arrives on, with a 1 ms limit, so the kernel's
 * bounded-wait abort path runs (no GPU fault, trap or hang is made).
 * No reference counterpart (the reference has no GPU). */
ZYNUM_BLAS_GPU_API void zynum_blas_gpu_inject_fault(int kind, int count);
/* Synchronises `stream` and reports whether a tensor-core product kernel of
 * this device abandoned its work because a bounded wait ran out since the
 * last call: 0 if none, else -(cudaErrorLaunchTimeout) with the site in
 * zynum_blas_gpu_last_error().  Such a CRT-scheme Ozaki call leaves C as it
 * was.  Host entry points make this check themselves before copying C back.
 * No reference counterpart (the reference has no GPU). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_device_status(void *stream);
/* Measured raw issue rate of a tensor pipe on the current GPU, for roofline
 * fractions against a measured denominator: pipe 0 = FP64 DMMA (register-only
 * mma.sync m16n8k8 loop on every SM; TFLOP/s), pipe 1 = INT8 tcgen05
 * (cta_group::2 M = 256, N = 256, K = 32 MMAs on shared-memory operands, one
 * CTA pair per two SMs; TOP/s).  Runs on `stream` and synchronises it; takes
 * about 0.1 s.  Returns 0 and writes *rate, 1 for a bad argument, or a
 * negative CUDA status.  No reference counterpart (measurement only). */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_measure_pipe_rate(int pipe, double *rate, void *stream);
/* Dominant-kernel timing: enable != 0 starts recording CUDA events around the
 * main contraction kernel of every call (on the launching stream) and clears
 * earlier records; returns the previous state. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_profile(int enable);
/* Writes up to `max` recorded kernel durations (milliseconds, in launch order)
 * to `ms`, waiting for them to complete; returns the count, or -1. */
ZYNUM_BLAS_GPU_API int zynum_blas_gpu_profile_read(double *ms, int max);
/* Number of kernels this library has launched in this process so far. */
ZYNUM_BLAS_GPU_API long long zynum_blas_gpu_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* ZYNUM_BLAS_GPU_H */
