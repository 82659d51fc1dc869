/*
 * ORACLE -- test infrastructure only.
 *
 * Compiles the reference's own structure-generic evaluators, exactly as they lie in the
 * reference tree (codeGen/H2GEMM.h, codeGen/cholUtils.h; codeGen/HSSGEMM.h in
 * ref_wrap_hss.c), into
 * oracle/_ref/libmatrox_ref.so, and exports them under "ref_" names so they can never be
 * confused with this repository's drop-in symbols.  <mkl.h> resolves to the shim in
 * oracle/mkl_shim.  Everything else in the library is hidden (-fvisibility=hidden).
 */
#include <mkl.h>
#include <omp.h>
/* H2GEMM.h takes float_from_bits from the HSS header, which is compiled as C in
 * ref_wrap_hss.c; this is the same bit cast. */
static inline float float_from_bits(uint32_t bits)
{
    union { uint32_t u; float f; } v;
    v.u = bits;
    return v.f;
}
#include "H2GEMM.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT void ref_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }
REF_EXPORT void ref_set_omp_threads(int n) { omp_set_num_threads(n); }
REF_EXPORT int ref_get_omp_threads(void) { return omp_get_max_threads(); }

/* codeGen/H2GEMM.h:380 -- coarsened + blocked H2-b evaluation (the generated HGEMM's
 * structure-generic form). */
REF_EXPORT int32_t ref_CBHGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                               int32_t *VTptr, int32_t *lchildren, int32_t *rchildren,
                               int32_t *levelset, int32_t *idx, double *mrhs, double *apres,
                               int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr,
                               double *wskel, int32_t *wskeloffset, double *uskel,
                               int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                               int32_t *nblockSet, int32_t *nblocks, int32_t *npairx,
                               int32_t *npairy, int32_t *fblockSet, int32_t *fblocks,
                               int32_t *fpairx, int32_t *fpairy, int32_t ncount, int32_t fcount,
                               int32_t *wpart, int32_t *clevelset, int cdepth)
{
    return CBHGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres,
                   nrhs, Ddim, wptr, uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen,
                   nblockSet, nblocks, npairx, npairy, fblockSet, fblocks, fpairx, fpairy,
                   ncount, fcount, wpart, clevelset, cdepth);
}

/* codeGen/H2GEMM.h:255 -- blocked H2-b evaluation over uncoarsened level sets. */
REF_EXPORT int32_t ref_blockGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                                 int32_t *VTptr, int32_t *lchildren, int32_t *rchildren,
                                 int32_t *levelset, int32_t *idx, double *mrhs, double *apres,
                                 int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr,
                                 double *wskel, int32_t *wskeloffset, double *uskel,
                                 int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                                 int32_t *nblockSet, int32_t *nblocks, int32_t *npairx,
                                 int32_t *npairy, int32_t *fblockSet, int32_t *fblocks,
                                 int32_t *fpairx, int32_t *fpairy, int32_t ncount,
                                 int32_t fcount, int32_t depth)
{
    return blockGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs,
                     apres, nrhs, Ddim, wptr, uptr, wskel, wskeloffset, uskel, uskeloffset, lm,
                     slen, nblockSet, nblocks, npairx, npairy, fblockSet, fblocks, fpairx,
                     fpairy, ncount, fcount, depth);
}

