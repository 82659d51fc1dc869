/*
 * matrox_b200.h -- C-ABI of the B200 (sm_100a) evaluator of Y = K~ W for HSS and H2-b
 * compressed kernel matrices in MatRox's compressed data storage (CDS).
 *
 * Two groups of entry points:
 *
 * 1. Drop-ins with the reference's own signatures.  They take HOST arrays exactly as
 *    the reference's generated or structure-generic evaluators do, copy what is needed
 *    to the GPU, evaluate there and copy `apres` back before returning.  The device
 *    copy of the CDS is cached between calls (see mxb_cache_invalidate).  On entry,
 *    `wskel` is ignored and `uskel` is not read; on return neither workspace is written
 *    unless MXB_FLAG_MIRROR_WORKSPACES is set (mxb_set_flags).  Unlike the reference they
 *    return 0 on success and a negative MXB_ERR_* code on failure (message in
 *    mxb_last_error()).
 *
 * 2. A plan API on DEVICE pointers (mxb_plan_*), used by the Python binding, the
 *    torch.autograd.Function and the benchmarks: the CDS is uploaded once, every
 *    evaluation is a handful of kernel launches on a caller stream.
 *
 * Array conventions (all from the reference): column-major blocks; D / B / VT hold the
 * near blocks, far couplings and projections at element offsets Dptr / Bptr (uint64) and
 * VTptr (int32); W ("mrhs") and Y ("apres") are leaf-blocked: leaf i owns a Ddim[i] x nrhs
 * column-major block at element offset wptr[i] / uptr[i]; lchildren[v] == -1 marks a leaf.
 */
#ifndef MATROX_B200_H
#define MATROX_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define MXB_API __attribute__((visibility("default")))
#else
#define MXB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define MXB_OK 0
#define MXB_ERR_ARG (-1)        /* null pointer, negative size, bad mode               */
#define MXB_ERR_STRUCTURE (-2)  /* index out of range, cycle, rank/size inconsistency  */
#define MXB_ERR_CUDA (-3)       /* CUDA runtime error (message has the CUDA string)    */
#define MXB_ERR_NOMEM (-4)      /* device or host allocation failed                    */
#define MXB_ERR_TIMEOUT (-5)    /* a bounded device-side wait gave up                  */
#define MXB_ERR_UNSUPPORTED (-6)/* shape outside what a kernel variant supports        */

/* ---- precision modes --------------------------------------------------------------- */
#define MXB_PREC_FP64 0       /* FP64 everywhere (reference mode)                        */
#define MXB_PREC_SPLIT_BF16 1 /* tensor cores (tcgen05, BF16 in, FP32 accumulate), both
                                 operands split: near and far couplings hi+mid with 3
                                 products, transfers hi+mid+lo with 6 products (FP32
                                 accuracy); FP64 final Y                                  */
#define MXB_PREC_SPLIT_BF16_FAR6 2 /* as MXB_PREC_SPLIT_BF16 with 6-product far couplings */
#define MXB_PREC_SPLIT_BF16_X6 3   /* 6 products (hi+mid+lo) for every GEMM               */
/* OR'd into the precision of mxb_plan_create (no counterpart in the reference): a split-BF16
 * plan also tiles the near blocks and far couplings transposed, so mxb_plan_adjoint runs the
 * transposed traversal on the tensor cores with the plan's own product counts (the plan holds
 * the near and far operand tiles twice).  FP64 plans always have the adjoint. */
#define MXB_PLAN_ADJOINT 0x100

/* ---- flags for the drop-ins ---------------------------------------------------------- */
#define MXB_FLAG_MIRROR_WORKSPACES 1u /* copy wskel/uskel back to the caller's arrays    */
#define MXB_FLAG_OUTPUT_IS_ZERO 2u    /* caller guarantees apres == 0 on entry (H2-b):
                                         skip its upload                                */

/* ---- library state ------------------------------------------------------------------- */
MXB_API const char *mxb_last_error(void);
MXB_API const char *mxb_version(void);
/* Precision used by the drop-ins (default MXB_PREC_FP64). */
MXB_API int32_t mxb_set_precision(int32_t mode);
MXB_API int32_t mxb_set_flags(uint32_t flags);
/* Drop every cached device copy of a CDS.  Required, in the default mode, after changing CDS
 * values in place AND after freeing a CDS and allocating a new one that may land at the same
 * addresses with the same sizes: the default key covers the pool pointers, every index array
 * and about 4096 sampled values per pool, not every value. */
MXB_API int32_t mxb_cache_invalidate(void);
/* How the drop-ins recognise a CDS they have already uploaded (no counterpart in the
 * reference, which reads the host CDS on every call).  Setting a mode drops the cache.
 *   MXB_CACHE_SAMPLED (default): pointers, index arrays, ~4096 sampled values per pool.
 *   MXB_CACHE_FULL: pointers, index arrays and every value of D, B and VT (a host pass over
 *     the pools on every call, ~0.5 s per GB on one core; no invalidation needed).
 *   MXB_CACHE_OFF: upload the CDS on every call, as the reference reads it on every call. */
#define MXB_CACHE_SAMPLED 0
#define MXB_CACHE_FULL 1
#define MXB_CACHE_OFF 2
MXB_API int32_t mxb_cache_set_mode(int32_t mode);

/* Test hook, no counterpart in the reference (host code only, no device needed): the unit order
 * that a chained tree sweep runs in when its units wait on per-node counters, for a synthetic
 * dependency forest.  Node i reads the outputs of nodes deps[dep_first[i] .. dep_first[i + 1])
 * (at most two; dep_first has nnodes + 1 entries), has ntask[i] row tiles of kt[i] K tiles and
 * ncol column tiles, and `workers` CTAs claim the units.  Unit u (u < *count <= cap) is written as
 * its node, its column tile, the counters it waits for (dep0, dep1; -1: none) with the units each
 * must count (need: low and high 16 bits) and the counter it signals (sig; -1: none).
 * MXB_ERR_UNSUPPORTED when the dependencies are not a tree (the sweep then keeps level
 * barriers). */
MXB_API int32_t mxb_debug_dataflow_order(int32_t nnodes, const int32_t *dep_first, const int32_t *deps,
                                         const int32_t *ntask, const int32_t *kt, int32_t ncol, int32_t workers,
                                         int32_t *node, int32_t *col, int32_t *dep0, int32_t *dep1,
                                         int32_t *need, int32_t *sig, int64_t cap, int64_t *count);

/* ---- drop-ins: H2-b -------------------------------------------------------------------- */

/* Replaces CBHGEMM, codeGen/H2GEMM.h:380-389 (coarsened + blocked H2-b evaluation).
 * ncount / fcount are the numbers of near / far block ROWS (nblockSet has ncount+1
 * entries, fblockSet fcount+1); cdepth is the number of coarsened levels. */
MXB_API int32_t CBHGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy,
                int32_t *fblockSet, int32_t *fblocks, int32_t *fpairx, int32_t *fpairy,
                int32_t ncount, int32_t fcount, int32_t *wpart, int32_t *clevelset,
                int cdepth);

/* Replaces lowH2GEMM, codeGen/H2GEMM.h:506-515 (same arguments and result as CBHGEMM). */
MXB_API int32_t lowH2GEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                  int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                  int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                  int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                  double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy,
                  int32_t *fblockSet, int32_t *fblocks, int32_t *fpairx, int32_t *fpairy,
                  int32_t ncount, int32_t fcount, int32_t *wpart, int32_t *clevelset,
                  int cdepth);

/* Replaces blockGEMM, codeGen/H2GEMM.h:255-262 (blocked H2-b over uncoarsened level sets;
 * levelset / idx are top-down, depth levels, root excluded). */
MXB_API int32_t blockGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                  int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                  int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                  int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                  double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy,
                  int32_t *fblockSet, int32_t *fblocks, int32_t *fpairx, int32_t *fpairy,
                  int32_t ncount, int32_t fcount, int32_t depth);

/* Replaces the generated H2-b evaluator HGEMM, symGen/HGEMM_gen.h:120-124.  The generated
 * code bakes the number of near block rows, far block rows and coarsened levels into its
 * loop bounds; here they are set once with mxb_hgemm_set_shape (nrow, frow, cdepth as in
 * CBHGEMM's ncount, fcount, cdepth). */
MXB_API int32_t mxb_hgemm_set_shape(int32_t nrow, int32_t frow, int32_t cdepth);
MXB_API int32_t HGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
              int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
              int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
              int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
              double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
              int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy,
              int32_t *fblockSet, int32_t *fblocks, int32_t *fpairx, int32_t *fpairy,
              int32_t *wpart, int32_t *clevelset);

/* ---- drop-ins: HSS ----------------------------------------------------------------------- */

/* Replaces parHSSGEMM, codeGen/HSSGEMM.h:131-134: ncount = number of leaves,
 * fcount = numnodes - 1 (far couplings are sibling pairs, B of node i at Bptr[i-1]). */
MXB_API int32_t parHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                   int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                   int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                   int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                   double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t *wpart, int32_t *clevelset, int ncount, int fcount, int cdepth);

/* Replaces lowHSSGEMM, codeGen/HSSGEMM.h:246-249 (same arguments and result). */
MXB_API int32_t lowHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                   int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                   int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                   int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                   double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t *wpart, int32_t *clevelset, int ncount, int fcount, int cdepth);

/* Replaces seqHSSGEMM, codeGen/HSSGEMM.h:18-21 (levelset / idx top-down, depth levels). */
MXB_API int32_t seqHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                   int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                   int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                   int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                   double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t ncount, int32_t fcount, int32_t depth);

/* Replaces the generated HSS evaluator (codeGen/HGEMM_gen.h:120-124, exported there as
 * HGEMM; renamed here so both generated forms can live in one library).  nleaf / numnodes
 * / cdepth come from mxb_hgemm_hss_set_shape. */
MXB_API int32_t mxb_hgemm_hss_set_shape(int32_t nleaf, int32_t cdepth);
MXB_API int32_t HGEMM_HSS(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr,
                  int32_t *VTptr, int32_t *lchildren, int32_t *rchildren, int32_t *levelset,
                  int32_t *idx, double *mrhs, double *apres, int32_t nrhs, int32_t *Ddim,
                  int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset,
                  double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *wpart, int32_t *clevelset);

/* ---- input / output permutation (matroxTest-V1/hcds.h:766-788 `transform`) -------------- */

/* TW[leaf-blocked] = W[perm rows]: W is n x nrhs column-major (ldw >= n) in the original
 * point order; perm[t] is the original row of tree position t; leaf i owns tree positions
 * [leafofs[i], leafofs[i+1]) and its block starts at TW + wptr[i] with leading dimension
 * leafofs[i+1]-leafofs[i].  Host pointers, synchronous. */
MXB_API int32_t mxb_transform(const int32_t *perm, const int32_t *leafofs, const int32_t *wptr,
                      int32_t nleaf, const double *W, int64_t n, int64_t ldw, int32_t nrhs,
                      double *TW);
/* Inverse: Y[perm rows] = TY[leaf-blocked] (the reference has no inverse; its output stays
 * in tree order, matroxTest-V1/Util.h:320). */
MXB_API int32_t mxb_untransform(const int32_t *perm, const int32_t *leafofs, const int32_t *uptr,
                        int32_t nleaf, const double *TY, int64_t n, int64_t ldy, int32_t nrhs,
                        double *Y);

/* Device-pointer form of both directions, asynchronous on `stream`.  direction 0:
 * dst(leaf-blocked) = src[perm rows]; direction 1: dst[perm rows] (+)= src(leaf-blocked).
 * The caller-order matrix has element (p, j) at p*row_stride + j*col_stride (row-major
 * (N, r): row_stride = r, col_stride = 1; column-major: 1, ld).  d_blockofs[i] is the
 * element offset of leaf i's block (Ddim[i] x nrhs, column-major). */
MXB_API int32_t mxb_permute_rows(const int32_t *d_perm, const int32_t *d_leafofs, const int32_t *d_blockofs,
                         int32_t nleaf, int64_t n, const double *src, double *dst, int64_t row_stride,
                         int64_t col_stride, int32_t nrhs, int32_t direction, int32_t accumulate,
                         void *stream);

/* ---- plan API (device pointers, caller stream) -------------------------------------------- */

typedef struct mxb_plan mxb_plan;

/* Host description of a CDS.  Pair lists are flat: near pair k is (npairx[k], npairy[k])
 * with block D + Dptr[k]; far pair k is (fpairx[k], fpairy[k]) with B + Bptr[k].  For an
 * HSS CDS set is_hss = 1 and give the far pairs as (i, sibling(i)), i = 1..numnodes-1. */
typedef struct mxb_cds_desc {
    int32_t nleaf, numnodes, is_hss;
    const double *D;   uint64_t D_len;
    const double *B;   uint64_t B_len;
    const double *VT;  uint64_t VT_len;
    const uint64_t *Dptr; const uint64_t *Bptr; const int32_t *VTptr;
    const int32_t *lchildren, *rchildren, *lm, *slen, *Ddim;
    const int32_t *npairx, *npairy; int32_t ncount;
    const int32_t *fpairx, *fpairy; int32_t fcount;
} mxb_cds_desc;

/* Uploads and repacks the CDS for `precision`, builds the task lists; device = current.
 * desc->D, desc->B and desc->VT may be host arrays or device arrays of the current device
 * (e.g. blocks from mxb_kernel_blocks); the plan keeps its own copy either way. */
MXB_API int32_t mxb_plan_create(const mxb_cds_desc *desc, int32_t precision, mxb_plan **out);
MXB_API int32_t mxb_plan_destroy(mxb_plan *plan);
/* dY (+)= K~ dW on `stream` (a cudaStream_t, 0 = legacy default).  dW / dY are device
 * arrays in the leaf-blocked layout with per-leaf offsets wptr / uptr (host arrays, nleaf
 * entries; NULL = packed: offset of leaf i = (sum of Ddim[<i]) * nrhs).  accumulate = 1
 * adds to dY (H2-b reference semantics), 0 overwrites it.  Asynchronous. */
MXB_API int32_t mxb_plan_evaluate(mxb_plan *plan, const double *dW, double *dY, int32_t nrhs,
                          const int32_t *wptr, const int32_t *uptr, int32_t accumulate,
                          void *stream);
/* dGW (+)= K~^T dG by the transposed traversal (no counterpart in the reference).  FP64 plans,
 * and split-BF16 plans created with MXB_PLAN_ADJOINT (MXB_ERR_UNSUPPORTED otherwise).
 * A plan's evaluations and adjoints share its device workspaces: calls on one plan that overlap
 * on the GPU (different streams without ordering between them) race; order them or use one
 * stream, or one plan per stream. */
MXB_API int32_t mxb_plan_adjoint(mxb_plan *plan, const double *dG, double *dGW, int32_t nrhs,
                         const int32_t *gptr, const int32_t *gwptr, int32_t accumulate,
                         void *stream);
/* W and Y in the caller's point order.  The reference permutes W into tree order before
 * HGEMM (`transform`, matroxTest-V1/hcds.h:766-788, called from matroxTest-V1/main.cpp:91) and
 * leaves Y in tree order (matroxTest-V1/Util.h:320).  Here the permutation is registered once:
 * perm[t] is the caller's row of tree position t (the reference's `lids`; host or device
 * array of sum(Ddim) entries, checked to be a permutation).  Synchronous. */
MXB_API int32_t mxb_plan_set_permutation(mxb_plan *plan, const int32_t *perm);
/* dY (+)= K~ dW with dW / dY in the caller's point order: element (p, j) of dW at
 * dW[p * w_rs + j * w_cs] (row-major (N, nrhs): w_rs = nrhs, w_cs = 1; column-major: 1, ld),
 * likewise dY.  Split-BF16 plans gather W's rows inside the launch that splits W into operand
 * tiles and scatter Y's rows in the epilogues that write Y, so the permutation costs no pass of
 * its own; FP64 plans permute into leaf-blocked copies and back.  Asynchronous. */
MXB_API int32_t mxb_plan_evaluate_ordered(mxb_plan *plan, const double *dW, int64_t w_rs, int64_t w_cs,
                                          double *dY, int64_t y_rs, int64_t y_cs, int32_t nrhs,
                                          int32_t accumulate, void *stream);
/* dGW (+)= K~^T dG in the caller's point order (permuted copies; the plans mxb_plan_adjoint takes). */
MXB_API int32_t mxb_plan_adjoint_ordered(mxb_plan *plan, const double *dG, int64_t g_rs, int64_t g_cs,
                                         double *dGW, int64_t gw_rs, int64_t gw_cs, int32_t nrhs,
                                         int32_t accumulate, void *stream);
/* Algorithmic flops of one evaluation (matroxTest-V1/compression.h:1079-1130). */
MXB_API int32_t mxb_plan_flops(const mxb_plan *plan, int32_t nrhs, uint64_t *flops);
/* Bytes of CDS held on the device and number of kernel launches of one evaluation. */
MXB_API int32_t mxb_plan_info(const mxb_plan *plan, uint64_t *device_bytes, int32_t *launches,
                      int32_t *precision);
/* Waits for the device and reports a kernel-side failure of earlier evaluations on the plan
 * (MXB_ERR_TIMEOUT when a bounded wait of a tensor-core kernel gave up); clears it. */
MXB_API int32_t mxb_plan_status(mxb_plan *plan);
/* Test hook for failure detection, no counterpart in the reference.  With
 * MXB_DEBUG_STALL_ONE_WAIT, the first tensor-core launch of the next evaluations has one CTA
 * withhold a pipeline stage, so its bounded wait runs out: the CTA gives up, frees its TMEM
 * and mxb_plan_status() reports MXB_ERR_TIMEOUT, with the GPU context still usable.
 * wait_cycles > 0 shortens every kernel wait limit (default ~4e9 SM cycles).  flags = 0
 * restores normal operation.  Split-BF16 plans only. */
#define MXB_DEBUG_STALL_ONE_WAIT 1
/* MXB_DEBUG_CHAIN_LEVELS: every run of consecutive up-sweep (or down-sweep) launches of one
 * product count runs as one launch whose levels wait for each other on the device (otherwise
 * the autotuner chains a run only where that is faster).  MXB_DEBUG_STALL_LEVEL (implies
 * chaining): the first level of each chained launch never reports its units done, so the
 * bounded wait of the next level runs out and mxb_plan_status() reports MXB_ERR_TIMEOUT. */
#define MXB_DEBUG_CHAIN_LEVELS 2
#define MXB_DEBUG_STALL_LEVEL 4
/* MXB_DEBUG_ONE_LAUNCH: the plan's evaluation runs as one launch, as a batch in
 * MXB_BATCH_ONE_LAUNCH mode does (with MXB_DEBUG_STALL_LEVEL, its level barriers run out). */
#define MXB_DEBUG_ONE_LAUNCH 8
MXB_API int32_t mxb_plan_set_test_hooks(mxb_plan *plan, int32_t flags, int64_t wait_cycles);
/* Copies the last evaluation's skeleton workspaces (wskel, uskel) to host arrays laid out
 * with the caller's wskeloffset / uskeloffset (for callers that inspect them). */
MXB_API int32_t mxb_plan_read_workspaces(mxb_plan *plan, int32_t nrhs, const int32_t *wskeloffset,
                                 double *wskel, const int32_t *uskeloffset, double *uskel);

/* ---- batches: many H-matrices in one launch sequence ---------------------------------------- */

/* No counterpart in the reference (which evaluates one matrix per HGEMM call).  A batch merges
 * the launch sequences of several split-BF16 plans (same device; uneven N, ranks and nrhs and
 * any mix of split modes allowed -- couplings of different product counts run in separate
 * launches): one tensor-core launch per level serves every plan, the whole evaluation is
 * captured as one CUDA graph, and the column-tile width of every launch is picked by timing
 * the candidates (64 / 128 / 256 right-hand sides) on the first evaluation of an nrhs
 * signature (MXB_AUTOTUNE=0 disables the measurement); runs of up-sweep or down-sweep levels
 * are chained into one launch with device-side level barriers where that measures faster.
 * The plans must outlive the batch; dW[i] / dY[i] are packed leaf-blocked device arrays of
 * plan i with nrhs[i] columns. */
typedef struct mxb_batch mxb_batch;
MXB_API int32_t mxb_batch_create(mxb_plan *const *plans, int32_t count, mxb_batch **out);
MXB_API int32_t mxb_batch_evaluate(mxb_batch *batch, const double *const *dW, double *const *dY,
                                   const int32_t *nrhs, int32_t accumulate, void *stream);
/* Synchronises and reports a kernel-side failure (MXB_ERR_TIMEOUT) of any plan; clears it. */
MXB_API int32_t mxb_batch_status(mxb_batch *batch);
/* Launches per evaluation and the tuned tile of every tensor-core launch of the last
 * evaluation: the column-tile width, plus MXB_TILE_PAIR when the launch runs on pairs of SMs
 * (a 2-CTA cluster computing 256-row tiles with tcgen05.mma.cta_group::2). */
#define MXB_TILE_PAIR 4096
MXB_API int32_t mxb_batch_info(const mxb_batch *batch, int32_t *launches, int32_t *widths, int32_t cap,
                               int32_t *nwidths);
/* How a batch evaluation is launched (no counterpart in the reference).
 * MXB_BATCH_LEVEL_LAUNCHES (default): a W-split launch, then one tensor-core launch per level of
 *   the merged sequence, runs of up-sweep or down-sweep levels chained into one launch where
 *   the autotuner measures that faster.
 * MXB_BATCH_ONE_LAUNCH: the whole evaluation -- the W split, up-sweep, couplings, near field,
 *   down-sweep and leaf down of every plan -- is ONE launch of the persistent kernel: every
 *   level is a group of work units that waits on the device (bounded) until the level before
 *   it is written.  One column-tile width (64 or 128, timed on the first evaluation) and
 *   3-part stages serve every level; units of bf16x3 couplings load 2 parts and issue 3
 *   products.  W and Y leaf-blocked (MXB_ERR_UNSUPPORTED in the caller's point order).
 * Changing the mode drops the batch's captured evaluations. */
#define MXB_BATCH_LEVEL_LAUNCHES 0
#define MXB_BATCH_ONE_LAUNCH 1
MXB_API int32_t mxb_batch_set_launch_mode(mxb_batch *batch, int32_t mode);
MXB_API int32_t mxb_batch_destroy(mxb_batch *batch);

/* ---- per-launch timing (no counterpart in the reference, which times the whole HGEMM
 * call with omp_get_wtime in matroxTest-V1/main.cpp:94-108) ----
 * Evaluates Y = K~W (overwriting Y) once through the ordinary path, then twice launch by launch
 * outside any graph, bracketing every launch with CUDA events on `stream`, and reports the
 * second pass.  The launches are the ones the evaluation graph holds, in order, so Y on return
 * is the ordinary result.  The call synchronises `stream`. */
#define MXB_PHASE_SPLIT_W 0        /* W -> bf16 operand tiles (split-BF16 plans) */
#define MXB_PHASE_UP 1             /* leaf projection (level 0) or transfer at height `level` */
#define MXB_PHASE_FAR 2            /* far couplings of every depth (one launch) */
#define MXB_PHASE_DOWN 3           /* downward transfer into the nodes at depth `level` */
#define MXB_PHASE_NEAR 4           /* near field */
#define MXB_PHASE_LEAF_DOWN 5      /* leaf downward projection into Y */
#define MXB_PHASE_FAR_DOWN 6       /* FP64 plans: far + downward transfer, depth `level` */
#define MXB_PHASE_NEAR_LEAF_DOWN 7 /* FP64 plans: near field + leaf downward projection */
#define MXB_PHASE_FAR_NEAR 8       /* far couplings of every depth and the near field, one launch
                                      (split plans whose near and far products agree)    */
typedef struct mxb_op_profile {
    int32_t phase;        /* MXB_PHASE_* */
    int32_t level;        /* height or depth, see the phase */
    int32_t width;        /* right-hand sides per work unit (0: no tensor-core work) */
    int32_t units;        /* work units: output row tile x column tile */
    double flops;         /* algorithmic flops, 2 m k n summed over the launch's products */
    double issued_flops;  /* tensor-pipe flops issued: padded tiles, x3 / x6 for split products */
    float ms;             /* device time of the launch */
    int32_t pair;         /* 1: runs on pairs of SMs (256-row tiles) */
    int32_t chained;      /* 1: ran inside the launch of the record before it, as a later tree
                             level that waits on the device for the level before; ms is 0 and
                             that launch's ms covers both */
    float level_ms;       /* one-launch batches: this level's span inside the launch, from the
                             kernel's own timer (last unit of the level before to its own last
                             unit written); 0 elsewhere */
} mxb_op_profile;
/* `*nops` receives the number of launches; at most `cap` records are written. */
MXB_API int32_t mxb_plan_profile(mxb_plan *plan, const double *dW, double *dY, int32_t nrhs, void *stream,
                                 mxb_op_profile *out, int32_t cap, int32_t *nops);
MXB_API int32_t mxb_batch_profile(mxb_batch *batch, const double *const *dW, double *const *dY,
                                  const int32_t *nrhs, void *stream, mxb_op_profile *out, int32_t cap,
                                  int32_t *nops);

/* ---- CDS blocks generated on the GPU ---------------------------------------------------- */

/* Replaces the host-side block assembly of the CDS: Fsubmatrix, matroxTest-V1/compression.h:
 * 256-360, packed by CacheNear / CacheFar, matroxTest-V1/hcds.h:339-460.  Computes kernel blocks
 * K(X[rows], X[cols]) on the device, each stored column-major (element (i, j) at
 * out + blk_ofs[b] + i + j * rows) as in the reference's D / B pools.  dX: device points,
 * n x d row-major FP64 (d <= 128).  Index sets: host CSR, set s = set_idx[set_ofs[s] ..
 * set_ofs[s + 1]) (point indices; leaf points for near blocks, skeleton points for far
 * couplings).  Block b has rows from set blk_row[b] and columns from set blk_col[b].  dOut:
 * device array of out_len elements.  kind: MXB_KERNEL_*; h: bandwidth (unused for
 * MXB_KERNEL_NEWTON).  Asynchronous on `stream`; allocates its tile list with
 * cudaMallocAsync. */
#define MXB_KERNEL_GAUSSIAN 0 /* exp(-|x-y|^2 / (2 h^2))                               */
#define MXB_KERNEL_IMQ 1      /* 1 / sqrt(1 + |x-y|^2 / h^2)                            */
#define MXB_KERNEL_NEWTON 2   /* 1 / |x-y|, 1 on coincident points (compression.h:338)  */
MXB_API int32_t mxb_kernel_blocks(const double *dX, int64_t n, int32_t d, int32_t kind, double h,
                                  const int64_t *set_ofs, const int32_t *set_idx, int32_t nsets,
                                  const int32_t *blk_row, const int32_t *blk_col, const uint64_t *blk_ofs,
                                  int32_t nblk, double *dOut, uint64_t out_len, void *stream);

/* ---- ID compression on the GPU ------------------------------------------------------------ */

/* Replaces the per-node host ID of the CDS build, matroxTest-V1/compression.h:446-523
 * (`decomposition`: LAPACKE_dgeqp3, the rank rule, cblas_dtrsm).  count sample matrices A_b
 * (nrows[b] x ncols[b], column-major, packed back to back in dA, which is overwritten) are
 * factored in one launch, one CTA per matrix: Householder QR with column pivoting, rank
 * s_b = the first s >= 1 with |R[s,s] / R[0,0]| < tol (at most max_rank and min(nrows, ncols)),
 * and P_b (s_b x ncols[b]) with R11 P_b[:, piv] = R[0:s_b, :].  Outputs (device arrays):
 * dRank[b] = s_b; dPiv holds ncols[b] pivots per matrix, packed (the first s_b are the
 * skeleton columns); dP holds min(max_rank, ncols[b]) x ncols[b] doubles per matrix, packed,
 * of which the first s_b x ncols[b] are P_b (column-major, leading dimension s_b).  A zero
 * matrix gets P_b = 0, as in the reference.  ncols <= 8192.  Asynchronous on `stream`. */
MXB_API int32_t mxb_batched_id(double *dA, const int32_t *nrows, const int32_t *ncols, int32_t count,
                               double tol, int32_t max_rank, int32_t *dRank, int32_t *dPiv, double *dP,
                               void *stream);

/* ---- evaluation without device allocation ------------------------------------------------ */

/* No counterpart in the reference (its evaluator runs on the host).  For callers that may
 * not allocate device memory -- a framework whose pooling allocator owns the whole GPU, or a
 * steady-state loop that must not call cudaMalloc / cudaFree because they can synchronise
 * the device -- this computes dY (+)= K~ dW in FP64 like mxb_plan_evaluate and allocates
 * nothing: `desc` carries HOST index arrays but DEVICE pointers in desc->D, desc->B and
 * desc->VT (with their lengths); dW and dY are device arrays in the packed leaf-blocked
 * layout.  Pools, dW and dY that are not device memory of the current device (or managed
 * memory) are rejected with MXB_ERR_ARG before anything is launched.  Task lists, per-leaf offsets and skeleton workspaces live in one static device
 * array of MXB_NOALLOC_SCRATCH_BYTES (32 MiB) that every GPU loading the library keeps until
 * exit; larger problems (skeleton rows x nrhs x 16 bytes plus the task lists) are rejected
 * with MXB_ERR_UNSUPPORTED.  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress), so make it before any stream capture.  Each call copies its task
 * lists from temporary host memory (pageable, so the copy may block the host), and returns
 * MXB_ERR_UNSUPPORTED on a stream that is capturing.  Every call shares the array and
 * overwrites all of it that it reads, so nothing needs clearing, but calls that overlap on
 * the GPU (other streams, other host threads) race on it.  Asynchronous on `stream`. */
#define MXB_NOALLOC_SCRATCH_BYTES (32u << 20)
MXB_API int32_t mxb_evaluate_noalloc(const mxb_cds_desc *desc, const double *dW, double *dY, int32_t nrhs,
                                     int32_t accumulate, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MATROX_B200_H */
