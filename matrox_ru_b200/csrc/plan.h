// Plan object behind the mxb_plan_* C-ABI.
#pragma once
#include <cstdint>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"

struct mxb_plan {
    virtual ~mxb_plan() = default;
};
struct mxb_batch {
    virtual ~mxb_batch() = default;
};

namespace mxb {

struct SplitBF16;  // device state of the split-BF16 path (split_bf16.cu)
struct Batch;     // merged launch sequence of several split-BF16 plans (split_bf16.cu)

struct Plan : public mxb_plan {
    ~Plan() override;

    // ---- host structure ----
    int device = 0;
    int precision = MXB_PREC_FP64;
    bool want_adjoint = false;  // split-BF16: also tile the transposed operands (MXB_PLAN_ADJOINT)
    int nleaf = 0, numnodes = 0, is_hss = 0, root = 0;
    std::vector<int> Ddim, slen, lch, rch, lm, parent, depth, height, bfs;
    std::vector<int32_t> VTptr;
    std::vector<int> near_x, near_y, far_x, far_y;
    std::vector<uint64_t> near_off, far_off;
    std::vector<int64_t> leaf_row, skel_row;
    int64_t rows_total = 0, skel_total = 0;
    uint64_t D_len = 0, B_len = 0, VT_len = 0;

    // ---- task lists ----
    std::vector<Item> items;
    std::vector<Task> tasks;
    std::vector<Launch> launches_fwd, launches_adj;

    // ---- device state ----
    double *dD = nullptr, *dB = nullptr, *dVT = nullptr;
    Task *dTasks = nullptr;
    Item *dItems = nullptr;
    int32_t *dOfs = nullptr;  // 4 x nleaf per-leaf offsets (slots: in, out, spare)
    std::vector<int32_t> ofs_host[4];
    double *dWskel = nullptr, *dUskel = nullptr;
    size_t scratch_elems = 0;
    // caller point order (mxb_plan_set_permutation): perm (rows_total entries) followed by
    // the first tree position of every leaf (nleaf + 1 entries)
    int32_t *dTree = nullptr;
    double *dTW = nullptr, *dTY = nullptr;  // leaf-blocked copies for the unfused caller-order path
    size_t order_elems = 0;
    SplitBF16 *bf16 = nullptr;
    int debug_flags = 0;              // test hooks (mxb_plan_set_test_hooks)
    long long debug_wait_cycles = 0;  // 0: default wait limit
    std::vector<void *> allocations;
    uint64_t device_bytes = 0;

    static int create(const mxb_cds_desc &d, int precision, Plan **out);
    int validate(const mxb_cds_desc &d);
    void build_tasks(int tile);
    void add_task(std::vector<Task> &tasks, int16_t c_kind, int64_t c_row, int ldc, int M, int item0,
                  int nitem, int16_t beta, int tile);
    int alloc(void **p, size_t bytes);
    int ensure_scratch(int nrhs);
    int stage_offsets(int slot, const int32_t *ofs, int nrhs, cudaStream_t stream);
    int run(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, const int32_t *wofs,
            const int32_t *yofs, int accumulate, cudaStream_t stream);
    int profile(const double *dW, double *dY, int nrhs, cudaStream_t stream, mxb_op_profile *out, int cap,
                int *nops);
    int set_permutation(const int32_t *perm);
    int run_ordered(bool adjoint, const double *dW, int64_t w_rs, int64_t w_cs, double *dY, int64_t y_rs,
                    int64_t y_cs, int nrhs, int accumulate, cudaStream_t stream);
    int read_workspaces(int nrhs, const int32_t *wsko, double *wskel, const int32_t *usko, double *uskel);
    uint64_t flops(int nrhs) const;

    // evaluation replay: one CUDA graph per (operands, nrhs, accumulate, direction)
    struct GraphEntry {
        const void *launches;
        const double *W;
        double *Y;
        int nrhs, accumulate;
        cudaGraphExec_t exec;
    };
    std::vector<GraphEntry> graphs;
    cudaStream_t capture_stream = nullptr;
    void clear_graphs();
    int enqueue(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, int accumulate,
                cudaStream_t stream);

    // split-BF16 path (split_bf16.cu)
    int setup_split_bf16(const mxb_cds_desc &d);
    void clear_split_graphs();
    int run_split_bf16(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, int accumulate,
                       cudaStream_t stream, const CallerOrder *order = nullptr);
    void free_split_bf16();
};

const char *last_error();
int row_tile_for(int precision);
int split_bf16_launches(const Plan &p);
int split_bf16_prepare();
int batch_create(Plan *const *plans, int count, Batch **out);
int batch_evaluate(Batch *b, const double *const *W, double *const *Y, const int *nrhs, int accumulate,
                   cudaStream_t stream);
int batch_status(Batch *b);
void batch_destroy(Batch *b);
int batch_launches(const Batch *b);
int batch_set_one_launch(Batch *b, int on);
int batch_tuned_widths(const Batch *b, int *widths, int cap);
int split_bf16_status(Plan &p);
Batch *split_bf16_batch(Plan &p);  // the plan's own single-plan batch
int batch_profile(Batch *b, const double *const *W, double *const *Y, const int *nrhs, cudaStream_t stream,
                  mxb_op_profile *out, int cap, int *nops);

}  // namespace mxb
