/*
 * ORACLE -- test infrastructure only.
 *
 * Forced include (-include) for the reference's host pipeline, compiled from a scratch copy of
 * its sources under oracle/_ref/src by oracle/Makefile: the structure generator
 * (sympiler/HTree.cpp and friends, driven by ref_structure.cpp) and the compression / CDS
 * packing headers (matroxTest-V1/compression.h, hcds.h, driven by ref_cds.cpp).
 *
 * - MKL is not in this image: mkl_shim/mkl.h forwards the CBLAS calls to the OpenBLAS that
 *   scipy bundles, and LAPACKE_dgeqp3 is forwarded here (exported as scipy_LAPACKE_dgeqp3).
 * - The reference hard-codes its leaf size (sympiler/HTree.cpp:34, `setup.m = 256`) and its
 *   maximum ID rank (matroxTest-V1/compression.h:449, `int maxRank = 256`).  The Makefile's
 *   copy replaces those two constants with calls of the functions declared below, which the
 *   drivers define from their command lines.
 */
#ifndef MATROX_ORACLE_REF_PIPELINE_PRELUDE_H
#define MATROX_ORACLE_REF_PIPELINE_PRELUDE_H
#include <cstdint>
#include <mkl.h>

#define LAPACK_COL_MAJOR 102
extern "C" int scipy_LAPACKE_dgeqp3(int layout, int m, int n, double *a, int lda, int *jpvt, double *tau);
static inline int LAPACKE_dgeqp3(int layout, int m, int n, double *a, int lda, int *jpvt, double *tau)
{
    return scipy_LAPACKE_dgeqp3(layout, m, n, a, lda, jpvt, tau);
}

int mxb_ref_leaf_size();
int mxb_ref_max_rank();
#endif
