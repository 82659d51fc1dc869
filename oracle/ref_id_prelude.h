/*
 * ORACLE -- test infrastructure only.
 *
 * Prelude of oracle/_ref/ref_id.cpp, which the Makefile assembles from this file, the
 * reference's `decomposition` function (matroxTest-V1/compression.h:446-523, copied by line
 * range at build time into oracle/_ref/ only) and ref_id_export.inc.  compression.h itself
 * cannot be included on its own: its header tree declares `Ktype` twice (matroxTest-V1/Util.h
 * and sympiler/config.h).  The function needs only the C/C++ runtime, OpenMP and three MKL
 * calls: mkl_malloc and cblas_dtrsm come from mkl_shim/mkl.h, LAPACKE_dgeqp3 is forwarded here
 * to the OpenBLAS that scipy bundles (exported as scipy_LAPACKE_dgeqp3).
 */
#include <mkl.h>
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define LAPACK_COL_MAJOR 102
extern "C" int scipy_LAPACKE_dgeqp3(int layout, int m, int n, double *a, int lda, int *jpvt, double *tau);
static inline int LAPACKE_dgeqp3(int layout, int m, int n, double *a, int lda, int *jpvt, double *tau)
{
    return scipy_LAPACKE_dgeqp3(layout, m, n, a, lda, jpvt, tau);
}
