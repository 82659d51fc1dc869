/*
 * ORACLE -- test infrastructure only.
 *
 * Runs the reference's structure generator, as its entry point sympiler/MatRox.cpp:15-43 does,
 * on a points file: cluster tree, budget near / far lists and k-NN sampling
 * (sympiler/HTree.cpp:13-26), the code generator's inspector (coarsened level sets and the
 * near / far blocking, sympiler/DSInspector.cpp:64-86, run by HGEMM::sympile_to_c, which also
 * writes the generated evaluator <prefix>_gen.h), then the .bin structure files
 * (sympiler/HTree.cpp:299-543) into the working directory.
 *
 *   ref_structure <points.bin> <n> <dim> <budget> <leaf size> <generated-code prefix>
 *
 * The points file is n x dim doubles, point-major (sympiler/HTree.cpp:51-63).  The leaf size
 * replaces the reference's hard-coded 256 (see ref_pipeline_prelude.h).
 */
#include <cstdio>
#include <cstdlib>
#include <string>

#include "HGEMM.h"
#include "HMatrix.h"

using namespace Sympiler;
using namespace Sympiler::Internal;

static int g_leaf_size = 256;
int mxb_ref_leaf_size() { return g_leaf_size; }
int mxb_ref_max_rank() { return 256; }

int main(int argc, char **argv)
{
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s points.bin n dim budget leaf_size gen_prefix\n", argv[0]);
        return 2;
    }
    const std::string points = argv[1];
    const int n = std::atoi(argv[2]), dim = std::atoi(argv[3]);
    const double budget = std::atof(argv[4]);
    g_leaf_size = std::atoi(argv[5]);
    if (n <= 0 || dim <= 0 || g_leaf_size <= 0 || budget < 0) {
        std::fprintf(stderr, "ref_structure: bad arguments\n");
        return 2;
    }
    HTree tree(Float(64), points, n, dim, budget);
    HGEMM codegen(tree);
    codegen.sympile_to_c(argv[6]);
    tree.savetree();
    tree.savetree2disk();
    tree.SaveSampling();
    std::printf("ref_structure: ok\n");
    return 0;
}
