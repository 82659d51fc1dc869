/*
 * ORACLE -- test infrastructure only.
 *
 * The reference's HSS evaluators (codeGen/HSSGEMM.h), compiled as C where they lie in the
 * reference tree.  parHSSGEMM flows off the end of a non-void function; g++ turns that
 * into a trap instruction, while in C it is defined as long as the caller ignores the
 * value, which the wrapper below does.
 */
#include <stdbool.h>
#include <mkl.h>
#include "HSSGEMM.h"

#define HSS_EXPORT __attribute__((visibility("default")))

/* codeGen/HSSGEMM.h:131 -- coarsened HSS evaluation. */
HSS_EXPORT int32_t ref_parHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr,
                                  uint64_t *Bptr, int32_t *VTptr, int32_t *lchildren,
                                  int32_t *rchildren, int32_t *levelset, int32_t *idx,
                                  double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                                  int32_t *wptr, int32_t *uptr, double *wskel,
                                  int32_t *wskeloffset, double *uskel, int32_t *uskeloffset,
                                  int32_t *lm, int32_t *slen, int32_t *wpart, int32_t *clevelset,
                                  int ncount, int fcount, int cdepth)
{
    parHSSGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres,
               nrhs, Ddim, wptr, uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen, wpart,
               clevelset, ncount, fcount, cdepth);
    return 0;
}

/* codeGen/HSSGEMM.h:18 -- sequential HSS evaluation over uncoarsened level sets. */
HSS_EXPORT int32_t ref_seqHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr,
                                  uint64_t *Bptr, int32_t *VTptr, int32_t *lchildren,
                                  int32_t *rchildren, int32_t *levelset, int32_t *idx,
                                  double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                                  int32_t *wptr, int32_t *uptr, double *wskel,
                                  int32_t *wskeloffset, double *uskel, int32_t *uskeloffset,
                                  int32_t *lm, int32_t *slen, int32_t ncount, int32_t fcount,
                                  int32_t depth)
{
    return seqHSSGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs,
                      apres, nrhs, Ddim, wptr, uptr, wskel, wskeloffset, uskel, uskeloffset,
                      lm, slen, ncount, fcount, depth);
}
