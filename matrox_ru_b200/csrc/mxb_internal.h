// Internal types of the B200 evaluator.  Every pass of Y = K~ W is expressed as a list
// of GEMM tasks: a task owns one row tile of one output block C (M x nrhs, column-major,
// leading dimension ldc) and sums a short list of items op(A) * B into it.  The same
// kernels therefore run the near field, the leaf and transfer projections, the far
// couplings and the down-sweep; only the task lists differ.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace mxb {

// Operand / output kinds.  Kinds 0/1 are the caller's leaf-blocked W and Y: the row
// field holds a leaf index and the block starts at base + offs[leaf].  Kinds 2/3 are the
// evaluator's skeleton workspaces: the row field holds a row offset and the block starts
// at base + row * nrhs.
enum Kind : int16_t { KIND_W = 0, KIND_Y = 1, KIND_WSKEL = 2, KIND_USKEL = 3 };

struct Item {
    uint64_t a_off;  // element offset of A in its pool
    int64_t b_row;   // leaf index (KIND_W) or skeleton row offset (KIND_WSKEL/USKEL)
    int32_t lda;
    int32_t ldb;
    int32_t K;
    int16_t trans;   // 1: op(A) = A^T
    int16_t b_kind;
    int16_t a_pool;  // 0 = D (near), 1 = B (far), 2 = VT (projections)
    int16_t pad0;
    int32_t pad1;
};
static_assert(sizeof(Item) == 40, "Item layout");

struct Task {
    int64_t c_row;   // leaf index (KIND_Y) or skeleton row offset
    int32_t ldc;
    int32_t M;       // rows of the whole output block
    int32_t m0;      // first row of this task's tile
    int32_t item0;
    int32_t nitem;
    int16_t c_kind;
    int16_t beta;    // 0 overwrite, 1 accumulate, 2 = take the launch's beta argument
};
static_assert(sizeof(Task) == 32, "Task layout");

struct Launch {
    int32_t task0;
    int32_t ntasks;
    int32_t max_m;   // largest M of the launch (row tile count is implied by tasks)
    int32_t kind;    // MXB_PHASE_* of the launch, for profiling
    int32_t level;   // height (up) or depth (far + down)
};

// Device pointers an evaluation needs; passed by value to every kernel.
struct Operands {
    const double *pool[3];     // D, B, VT (FP64)
    const double *W;           // caller input (leaf-blocked)
    double *Y;                 // caller output (leaf-blocked)
    double *wskel;
    double *uskel;
    const int32_t *wofs;       // per-leaf element offsets of W
    const int32_t *yofs;       // per-leaf element offsets of Y
    int32_t nrhs;
    int32_t beta_arg;
};

struct Plan;

// FP64 grouped GEMM (gemm_f64.cu)
cudaError_t launch_gemm_f64(const Task *tasks, const Item *items, int ntasks,
                            const Operands &ops, cudaStream_t stream);

cudaError_t prepare_gemm_f64();  // sets the kernel's shared-memory limit (before any capture)

// Row permutation between the caller's point order and the leaf-blocked tree order
// (permute.cu): dir 0 gathers dst(leaf-blocked) = src[perm rows], dir 1 scatters
// dst[perm rows] (+)= src(leaf-blocked).  The caller-order matrix has element (p, j) at
// p * rs + j * cs; leafofs has nleaf + 1 entries, blockofs nleaf.
cudaError_t launch_permute(const int32_t *perm, const int32_t *leafofs, const int32_t *blockofs, int nleaf,
                           int64_t n, const double *src, double *dst, int64_t rs, int64_t cs, int nrhs,
                           int dir, int accumulate, cudaStream_t stream);

// W and Y of an evaluation in the caller's point order: tree position t of leaf i (t in
// [tofs[i], tofs[i + 1])) is row perm[t]; element (row, j) sits at row * rs + j * cs.
struct CallerOrder {
    const int32_t *perm;
    const int32_t *tofs;
    int64_t w_rs, w_cs, y_rs, y_cs;
};

void set_error(const std::string &msg);

}  // namespace mxb
