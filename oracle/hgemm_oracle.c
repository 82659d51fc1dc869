/*
 * ORACLE -- test infrastructure only.
 *
 * Plain-C FP64 restatement of MatRox's evaluation Y = K~ W (the generated HGEMM).
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this
 * file's library; it is the checker, never the product.
 *
 * Every function takes the reference's CDS arrays with the reference's meaning:
 *   near   Y[x] += D_xy W[y]                  symGen/HGEMM_gen.h:125-141
 *   up     wskel[v] = P_v W[leaf v]            symGen/HGEMM_gen.h:152-160
 *          wskel[v] = P_v[:, :sl] wskel[l] + P_v[:, sl:] wskel[r]   :161-175
 *   far    uskel[x] += B_xy wskel[y]            symGen/HGEMM_gen.h:179-195
 *   down   uskel[l] += P_v[:, :sl]^T uskel[v] ... (top-down)       :219-233
 *          Y[leaf v] += P_v^T uskel[v]          symGen/HGEMM_gen.h:211-218
 * HSS form (codeGen/HGEMM_gen.h:125-188, codeGen/HSSGEMM.h:131-243):
 *   near   Y[i] = D_ii W[i]  (beta 0);  far  uskel[i] = B_{i,sib(i)} wskel[sib(i)] (beta 0)
 * The schedule arrays (clevelset / wpart / idx, coarsened post-order) are walked in
 * the reference's order: coarse levels ascending for the up-sweep with the nodes of a
 * partition in order, descending for the down-sweep with the nodes reversed
 * (codeGen/H2GEMM.h:380-504).
 *
 * The adjoint (K~^T G) has no counterpart in the reference: it walks the same tree
 * with every near block and far coupling transposed.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>

/* C (m x n, ldc) += alpha * op(A) * B, column-major; op(A) = A (m x k, lda) or
 * A^T (A is k x m, lda).  beta == 0 overwrites C first. */
static void dgemm_cm(int transA, int m, int n, int k, const double *A, int lda,
                     const double *B, int ldb, double beta, double *C, int ldc)
{
    for (int j = 0; j < n; ++j) {
        double *c = C + (size_t)j * ldc;
        const double *b = B + (size_t)j * ldb;
        if (beta == 0.0) memset(c, 0, sizeof(double) * (size_t)m);
        if (!transA) {
            for (int p = 0; p < k; ++p) {
                const double bp = b[p];
                const double *a = A + (size_t)p * lda;
                for (int i = 0; i < m; ++i) c[i] += a[i] * bp;
            }
        } else {
            for (int i = 0; i < m; ++i) {
                const double *a = A + (size_t)i * lda;
                double s = 0.0;
                for (int p = 0; p < k; ++p) s += a[p] * b[p];
                c[i] += s;
            }
        }
    }
}

/* Upward pass for one node v: leaf projection or two-child transfer. */
static void up_node(int v, const double *VT, const int32_t *VTptr, const int32_t *lch,
                    const int32_t *rch, const double *W, int32_t nrhs, const int32_t *Ddim,
                    const int32_t *wptr, double *wskel, const int32_t *wskeloffset,
                    const int32_t *lm, const int32_t *slen)
{
    const int s = slen[v];
    if (lch[v] == -1) {
        const int leaf = lm[v];
        dgemm_cm(0, s, nrhs, Ddim[leaf], VT + VTptr[v], s, W + wptr[leaf], Ddim[leaf], 0.0,
                 wskel + wskeloffset[v], s);
    } else {
        const int l = lch[v], r = rch[v];
        dgemm_cm(0, s, nrhs, slen[l], VT + VTptr[v], s, wskel + wskeloffset[l], slen[l], 0.0,
                 wskel + wskeloffset[v], s);
        dgemm_cm(0, s, nrhs, slen[r], VT + VTptr[v] + (size_t)s * slen[l], s,
                 wskel + wskeloffset[r], slen[r], 1.0, wskel + wskeloffset[v], s);
    }
}

/* Downward pass for one node v. */
static void down_node(int v, const double *VT, const int32_t *VTptr, const int32_t *lch,
                      const int32_t *rch, double *Y, int32_t nrhs, const int32_t *Ddim,
                      const int32_t *uptr, double *uskel, const int32_t *uskeloffset,
                      const int32_t *lm, const int32_t *slen)
{
    const int s = slen[v];
    if (lch[v] == -1) {
        const int leaf = lm[v];
        dgemm_cm(1, Ddim[leaf], nrhs, s, VT + VTptr[v], s, uskel + uskeloffset[v], s, 1.0,
                 Y + uptr[leaf], Ddim[leaf]);
    } else {
        const int l = lch[v], r = rch[v];
        dgemm_cm(1, slen[l], nrhs, s, VT + VTptr[v], s, uskel + uskeloffset[v], s, 1.0,
                 uskel + uskeloffset[l], slen[l]);
        dgemm_cm(1, slen[r], nrhs, s, VT + VTptr[v] + (size_t)s * slen[l], s,
                 uskel + uskeloffset[v], s, 1.0, uskel + uskeloffset[r], slen[r]);
    }
}

static void sweeps(const double *VT, const int32_t *VTptr, const int32_t *lch, const int32_t *rch,
                   const int32_t *idx, const double *W, double *Y, int32_t nrhs,
                   const int32_t *Ddim, const int32_t *wptr, const int32_t *uptr, double *wskel,
                   const int32_t *wskeloffset, double *uskel, const int32_t *uskeloffset,
                   const int32_t *lm, const int32_t *slen, const int32_t *wpart,
                   const int32_t *clevelset, int32_t cdepth, int phase)
{
    if (phase == 0) {
        for (int i = 0; i < cdepth; ++i)
            for (int k = clevelset[i]; k < clevelset[i + 1]; ++k)
                for (int j = wpart[k]; j < wpart[k + 1]; ++j)
                    up_node(idx[j], VT, VTptr, lch, rch, W, nrhs, Ddim, wptr, wskel,
                            wskeloffset, lm, slen);
    } else {
        for (int i = cdepth - 1; i >= 0; --i)
            for (int k = clevelset[i]; k < clevelset[i + 1]; ++k)
                for (int j = wpart[k + 1] - 1; j >= wpart[k]; --j)
                    down_node(idx[j], VT, VTptr, lch, rch, Y, nrhs, Ddim, uptr, uskel,
                              uskeloffset, lm, slen);
    }
}

/* H2-b evaluation with the argument list of CBHGEMM (codeGen/H2GEMM.h:380-389);
 * nrow / frow are the numbers of near / far block rows. Returns 0. */
int32_t oracle_h2b(const double *D, const double *B, const double *VT, const uint64_t *Dptr,
                   const uint64_t *Bptr, const int32_t *VTptr, const int32_t *lchildren,
                   const int32_t *rchildren, const int32_t *levelset, const int32_t *idx,
                   const double *mrhs, double *apres, int32_t nrhs, const int32_t *Ddim,
                   const int32_t *wptr, const int32_t *uptr, double *wskel,
                   const int32_t *wskeloffset, double *uskel, const int32_t *uskeloffset,
                   const int32_t *lm, const int32_t *slen, const int32_t *nblockSet,
                   const int32_t *nblocks, const int32_t *npairx, const int32_t *npairy,
                   const int32_t *fblockSet, const int32_t *fblocks, const int32_t *fpairx,
                   const int32_t *fpairy, int32_t nrow, int32_t frow, const int32_t *wpart,
                   const int32_t *clevelset, int32_t cdepth)
{
    (void)levelset;
    for (int i = 0; i < nrow; ++i)
        for (int j = nblockSet[i]; j < nblockSet[i + 1]; ++j)
            for (int k = nblocks[j]; k < nblocks[j + 1]; ++k) {
                const int x = npairx[k], y = npairy[k];
                dgemm_cm(0, Ddim[x], nrhs, Ddim[y], D + Dptr[k], Ddim[x], mrhs + wptr[y],
                         Ddim[y], 1.0, apres + uptr[x], Ddim[x]);
            }
    sweeps(VT, VTptr, lchildren, rchildren, idx, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 0);
    for (int i = 0; i < frow; ++i)
        for (int j = fblockSet[i]; j < fblockSet[i + 1]; ++j)
            for (int k = fblocks[j]; k < fblocks[j + 1]; ++k) {
                const int x = fpairx[k], y = fpairy[k];
                dgemm_cm(0, slen[x], nrhs, slen[y], B + Bptr[k], slen[x],
                         wskel + wskeloffset[y], slen[y], 1.0, uskel + uskeloffset[x], slen[x]);
            }
    sweeps(VT, VTptr, lchildren, rchildren, idx, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 1);
    return 0;
}

/* HSS evaluation with the argument list of parHSSGEMM (codeGen/HSSGEMM.h:131-134):
 * ncount = number of leaves, fcount = numnodes - 1. Returns 0. */
int32_t oracle_hss(const double *D, const double *B, const double *VT, const uint64_t *Dptr,
                   const uint64_t *Bptr, const int32_t *VTptr, const int32_t *lchildren,
                   const int32_t *rchildren, const int32_t *levelset, const int32_t *idx,
                   const double *mrhs, double *apres, int32_t nrhs, const int32_t *Ddim,
                   const int32_t *wptr, const int32_t *uptr, double *wskel,
                   const int32_t *wskeloffset, double *uskel, const int32_t *uskeloffset,
                   const int32_t *lm, const int32_t *slen, const int32_t *wpart,
                   const int32_t *clevelset, int32_t ncount, int32_t fcount, int32_t cdepth)
{
    (void)levelset;
    for (int i = 0; i < ncount; ++i)
        dgemm_cm(0, Ddim[i], nrhs, Ddim[i], D + Dptr[i], Ddim[i], mrhs + wptr[i], Ddim[i], 0.0,
                 apres + uptr[i], Ddim[i]);
    sweeps(VT, VTptr, lchildren, rchildren, idx, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 0);
    for (int i = 1; i < fcount + 1; ++i) {
        const int sib = (i & 1) == 0 ? i - 1 : i + 1;
        dgemm_cm(0, slen[i], nrhs, slen[sib], B + Bptr[i - 1], slen[i],
                 wskel + wskeloffset[sib], slen[sib], 0.0, uskel + uskeloffset[i], slen[i]);
    }
    sweeps(VT, VTptr, lchildren, rchildren, idx, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 1);
    return 0;
}

/* Adjoint G_W += K~^T G over an H2-b (or HSS, given as pair lists) structure.
 * Near pairs and far pairs are given as flat lists of length ncount / fcount in the
 * order of Dptr / Bptr.  wskel / uskel are workspaces (uskel must be zero on entry). */
int32_t oracle_adjoint(const double *D, const double *B, const double *VT, const uint64_t *Dptr,
                       const uint64_t *Bptr, const int32_t *VTptr, const int32_t *lchildren,
                       const int32_t *rchildren, const int32_t *idx, const double *G,
                       double *GW, int32_t nrhs, const int32_t *Ddim, const int32_t *wptr,
                       const int32_t *uptr, double *wskel, const int32_t *wskeloffset,
                       double *uskel, const int32_t *uskeloffset, const int32_t *lm,
                       const int32_t *slen, const int32_t *npairx, const int32_t *npairy,
                       int32_t ncount, const int32_t *fpairx, const int32_t *fpairy,
                       int32_t fcount, const int32_t *wpart, const int32_t *clevelset,
                       int32_t cdepth)
{
    /* near, transposed: GW[y] += D_xy^T G[x] */
    for (int k = 0; k < ncount; ++k) {
        const int x = npairx[k], y = npairy[k];
        dgemm_cm(1, Ddim[y], nrhs, Ddim[x], D + Dptr[k], Ddim[x], G + uptr[x], Ddim[x], 1.0,
                 GW + wptr[y], Ddim[y]);
    }
    /* up-sweep on G (rows addressed through uptr) */
    sweeps(VT, VTptr, lchildren, rchildren, idx, G, GW, nrhs, Ddim, uptr, wptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 0);
    /* far, transposed: uskel[y] += B_xy^T wskel[x] */
    for (int k = 0; k < fcount; ++k) {
        const int x = fpairx[k], y = fpairy[k];
        dgemm_cm(1, slen[y], nrhs, slen[x], B + Bptr[k], slen[x], wskel + wskeloffset[x],
                 slen[x], 1.0, uskel + uskeloffset[y], slen[y]);
    }
    /* down-sweep into GW (rows addressed through wptr) */
    sweeps(VT, VTptr, lchildren, rchildren, idx, G, GW, nrhs, Ddim, uptr, wptr, wskel,
           wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, cdepth, 1);
    return 0;
}
