/*
 * ORACLE -- test infrastructure only.
 *
 * Runs the reference's host pipeline between the structure files and the evaluator, as
 * matroxTest-V1/main.cpp:22-92 does: read the structure (readHtree, matroxTest-V1/HTree.h:76-260,
 * from ../sympiler/*.bin relative to the working directory), coarsened level sets
 * (coarloadtree), ID compression with the reference's k-NN row sampling (compression,
 * matroxTest-V1/compression.h:1057-1076), CDS packing (DUV2CDS, matroxTest-V1/hcds.h:433-460)
 * and the skeleton workspace offsets (allocatewuskel, hcds.h:487-496).  It then writes every
 * array the evaluator takes, exactly as the reference leaves them, into <outdir>:
 * one raw little-endian file per array plus meta.txt ("name dtype count" lines and scalars).
 *
 *   ref_cds <points.bin> <n> <dim> <id tolerance> <h> <max rank> <samples m> <hss 0|1> <outdir>
 *
 * Gaussian kernel exp(-|x-y|^2 / (2 h^2)) (KS_GAUSSIAN, matroxTest-V1/main.cpp:51).  `samples m`
 * is the reference's `m` argument of compression (main.cpp:85 passes 256): a node samples
 * max(2 |node|, 2 m) rows.  The workspace offsets are written for one right-hand side; they
 * scale linearly with nrhs (hcds.h:362-413).
 *
 * One deviation: readHtree sets nrow / frow to the LENGTH of nblockset.bin / fblockset.bin,
 * one more than the number of block rows, and CacheNearBlock / CacheFarBlock then read one
 * entry past the end of those arrays (hcds.h:45-47, 106-108).  This driver sets them to the
 * number of rows before packing, so the packing stays in bounds.
 *
 * The reference's sampling draws with rand() inside OpenMP loops; run with OMP_NUM_THREADS=1
 * for a reproducible CDS.  The coarsened partition counts follow omp_get_max_threads()
 * (compression.h:1016-1021), as in the reference.
 */
#include "Util.h"
#include "../sympiler/HMatrix.h"
#include "compression.h"
#include "hcds.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace Sympiler::Internal;
using namespace Sympiler;

static int g_max_rank = 256;
int mxb_ref_leaf_size() { return 256; }
int mxb_ref_max_rank() { return g_max_rank; }

namespace {

FILE *g_meta = nullptr;
std::string g_out;

template <class T>
void dump(const char *name, const char *dtype, const T *p, size_t count)
{
    const std::string path = g_out + "/" + name + ".bin";
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f || (count && std::fwrite(p, sizeof(T), count, f) != count)) {
        std::fprintf(stderr, "ref_cds: cannot write %s\n", path.c_str());
        std::exit(1);
    }
    std::fclose(f);
    std::fprintf(g_meta, "array %s %s %zu\n", name, dtype, count);
}

void scalar(const char *name, long long v) { std::fprintf(g_meta, "scalar %s %lld\n", name, v); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc != 10) {
        std::fprintf(stderr, "usage: %s points.bin n dim tol h max_rank m hss outdir\n", argv[0]);
        return 2;
    }
    const std::string points = argv[1];
    const int n = std::atoi(argv[2]), dim = std::atoi(argv[3]);
    const double acc = std::atof(argv[4]), h = std::atof(argv[5]);
    g_max_rank = std::atoi(argv[6]);
    const int m = std::atoi(argv[7]);
    const bool cbs = std::atoi(argv[8]) == 0;  // H2-b: blocked lists; HSS: flat lists
    g_out = argv[9];
    if (n <= 0 || dim <= 0 || h <= 0 || g_max_rank <= 0 || m <= 0) {
        std::fprintf(stderr, "ref_cds: bad arguments\n");
        return 2;
    }

    auto X = (double *)mkl_malloc(sizeof(double) * n * dim, 64);
    const int size1 = preprocesbin(points);
    if (size1 != n * dim) {
        std::fprintf(stderr, "ref_cds: %s holds %d doubles, expected %d\n", points.c_str(), size1, n * dim);
        return 1;
    }
    bin2read(points, X, size1);

    const Internal::Ktype kfun = Internal::KS_GAUSSIAN;
    HTree tree;
    readHtree(tree, true, cbs);
    tree.X = X;
    tree.ktype = kfun;
    tree.h = h;
    tree.dim = dim;
    if (cbs) {  // rows, not the lengths of the offset arrays (see the header comment)
        tree.nrow -= 1;
        tree.frow -= 1;
    }

    clustertree ctree;
    coarloadtree(tree, ctree);
    std::vector<ret> rtmp(tree.numnodes);
    compression(ctree, tree, rtmp.data(), X, m, n, kfun, dim, h, acc);
    hcds cds;
    DUV2CDS(tree, cds, ctree, rtmp.data(), 1, true, cbs);
    allocatewuskel(tree, cds, ctree, rtmp.data(), 1, true);
    std::printf("\n");

    const int nn = tree.numnodes, nl = tree.nleaf;
    size_t dlen = 0, blen = 0, plen = 0;
    for (int k = 0; k < tree.ncount; ++k)
        dlen = std::max<size_t>(dlen, cds.nearoffset[k] + (size_t)tree.Dim[tree.nxval[k]] * tree.Dim[tree.nyval[k]]);
    for (int k = 0; k < tree.fcount; ++k)
        blen = std::max<size_t>(blen, cds.faroffset[k] + (size_t)rtmp[tree.fxval[k]].skels_length *
                                                             rtmp[tree.fyval[k]].skels_length);
    size_t nskel = 0;
    for (int v = 1; v < nn; ++v) {
        plen = std::max<size_t>(plen, cds.projoffset[v] + (size_t)rtmp[v].skels_length * rtmp[v].proj_column);
        nskel += rtmp[v].skels_length;
    }
    std::vector<int> skels;
    skels.reserve(nskel);
    for (int v = 1; v < nn; ++v) skels.insert(skels.end(), rtmp[v].skels, rtmp[v].skels + rtmp[v].skels_length);

    g_meta = std::fopen((g_out + "/meta.txt").c_str(), "w");
    if (!g_meta) {
        std::fprintf(stderr, "ref_cds: cannot write %s/meta.txt\n", g_out.c_str());
        return 1;
    }
    scalar("n", n);
    scalar("dim", dim);
    scalar("nleaf", nl);
    scalar("numnodes", nn);
    scalar("depth", tree.depth);
    scalar("cdepth", tree.cdepth);
    scalar("is_hss", cbs ? 0 : 1);
    scalar("ncount", tree.ncount);
    scalar("fcount", tree.fcount);
    scalar("nrow", cbs ? tree.nrow : 0);
    scalar("frow", cbs ? tree.frow : 0);
    dump("D", "f64", cds.CacheNear, dlen);
    dump("B", "f64", cds.CacheFar, blen);
    dump("VT", "f64", cds.Proj, plen);
    dump("Dptr", "u64", cds.nearoffset, tree.ncount);
    dump("Bptr", "u64", cds.faroffset, tree.fcount);
    dump("VTptr", "i32", cds.projoffset, nn);
    dump("lchildren", "i32", tree.tlchildren, nn);
    dump("rchildren", "i32", tree.trchildren, nn);
    dump("levelset", "i32", tree.levelset, tree.depth + 1);
    dump("idx", "i32", tree.idx, nn - 1);
    dump("cidx", "i32", tree.cidx, nn - 1);
    dump("wpart", "i32", tree.wpart, tree.clevelset[tree.cdepth] + 1);
    dump("clevelset", "i32", tree.clevelset, tree.cdepth + 1);
    dump("Ddim", "i32", tree.Dim, nl);
    dump("lm", "i32", tree.lm, nn);
    dump("slen", "i32", cds.skel_length, nn);
    dump("proj_column", "i32", cds.proj_column, nn);
    dump("wptr1", "i32", cds.woffset, nl);
    dump("wskeloffset1", "i32", cds.w_skeloffset, nn);
    dump("npairx", "i32", tree.nxval, tree.ncount);
    dump("npairy", "i32", tree.nyval, tree.ncount);
    dump("fpairx", "i32", tree.fxval, tree.fcount);
    dump("fpairy", "i32", tree.fyval, tree.fcount);
    if (cbs) {
        dump("nblockset", "i32", tree.nblockset, tree.nrow + 1);
        dump("nblocks", "i32", tree.nblocks, tree.nb);
        dump("fblockset", "i32", tree.fblockset, tree.frow + 1);
        dump("fblocks", "i32", tree.fblocks, tree.fb);
    }
    size_t nlids = 0;  // lids.bin covers every node but the root (sympiler/HTree.cpp:441-462)
    for (int v = 0; v < nn; ++v) nlids = std::max<size_t>(nlids, (size_t)tree.lidsoffset[v] + tree.lidslen[v]);
    dump("lids", "i32", tree.lids, nlids);
    dump("lidsoffset", "i32", tree.lidsoffset, nn);
    dump("lidslen", "i32", tree.lidslen, nn);
    dump("leaf", "i32", tree.leaf, nl);
    dump("skels", "i32", skels.data(), skels.size());
    std::fclose(g_meta);
    std::printf("ref_cds: ok\n");
    return 0;
}
