/*
 * Stand-in for Intel MKL's <mkl.h>, used ONLY to compile the reference's own evaluator
 * sources (codeGen/H2GEMM.h, codeGen/HSSGEMM.h, codeGen/cholUtils.h) into the oracle
 * library under oracle/_ref.  MKL is not in this image; the reference only calls
 * cblas_dgemm and the mkl_set_* threading knobs on the evaluation path, so the shim
 * forwards cblas_dgemm to the OpenBLAS that scipy bundles (LP64 build, symbols exported
 * with a "scipy_" prefix) and turns the threading knobs into no-ops.
 */
#ifndef MATROX_ORACLE_MKL_SHIM_H
#define MATROX_ORACLE_MKL_SHIM_H
#include <stdlib.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

void scipy_cblas_dgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double,
                       const double *, int, const double *, int, double, double *, int);
double scipy_cblas_ddot(int, const double *, int, const double *, int);
void scipy_cblas_dtrsm(CBLAS_LAYOUT, CBLAS_SIDE, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int,
                       int, double, const double *, int, double *, int);
void scipy_openblas_set_num_threads(int);
#ifdef __cplusplus
}
#endif

static inline void cblas_dgemm(CBLAS_LAYOUT L, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m,
                               int n, int k, double alpha, const double *A, int lda,
                               const double *B, int ldb, double beta, double *C, int ldc)
{
    scipy_cblas_dgemm(L, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}
static inline double cblas_ddot(int n, const double *x, int incx, const double *y, int incy)
{
    return scipy_cblas_ddot(n, x, incx, y, incy);
}
static inline void cblas_dtrsm(CBLAS_LAYOUT L, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t,
                               CBLAS_DIAG d, int m, int n, double alpha, const double *A,
                               int lda, double *B, int ldb)
{
    scipy_cblas_dtrsm(L, s, u, t, d, m, n, alpha, A, lda, B, ldb);
}
static inline void mkl_set_dynamic(int on) { (void)on; }
static inline void mkl_set_num_threads(int n) { (void)n; }
static inline void *mkl_malloc(size_t n, int align)
{
    void *p = NULL;
    if (posix_memalign(&p, (size_t)align < sizeof(void *) ? sizeof(void *) : (size_t)align, n)) return NULL;
    return p;
}
static inline void mkl_free(void *p) { free(p); }
#endif
