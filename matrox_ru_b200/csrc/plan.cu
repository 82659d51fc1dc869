// Plan: validated structure, device copy of the CDS and the task lists of every pass.
//
// Schedule of one evaluation (the reference runs the same four phases,
// symGen/HGEMM_gen.h:125-236, but as thousands of separate DGEMM calls):
//   1. leaf up        wskel[v] = P_v W[leaf v]                          (one launch)
//   2. transfer up    wskel[v] = P_v [wskel[l]; wskel[r]]    one launch per height, bottom-up
//   3. far + down     uskel[c] = sum_y B_cy wskel[y] + P_p[:, c]^T uskel[p]
//                                                            one launch per depth, top-down
//   4. near + leaf down  Y[x] (+)= sum_y D_xy W[y] + P_x^T uskel[x]        (one launch)
// Phase 3 fuses the far coupling with the downward transfer and phase 4 fuses the near
// field with the leaf projection, so each skeleton block and each Y block is written
// exactly once per evaluation.  The adjoint reuses phases 1-2 on G and runs phases 3-4
// with every near block and far coupling transposed.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"
#include "plan.h"

namespace mxb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

#define MXB_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return MXB_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

int row_tile_for(int precision);

Plan::~Plan()
{
    clear_graphs();
    if (capture_stream) cudaStreamDestroy(capture_stream);
    free_split_bf16();
    for (void *p : allocations) cudaFree(p);
}

int Plan::alloc(void **p, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? MXB_ERR_NOMEM : MXB_ERR_CUDA;
    }
    allocations.push_back(*p);
    device_bytes += bytes;
    return MXB_OK;
}

// ---------------------------------------------------------------------------------------
// validation of the host structure
// ---------------------------------------------------------------------------------------

static int fail(const std::string &m)
{
    set_error(m);
    return MXB_ERR_STRUCTURE;
}

static int arg_fail(const std::string &m)
{
    set_error(m);
    return MXB_ERR_ARG;
}

int Plan::validate(const mxb_cds_desc &d)
{
    if (d.nleaf < 1 || d.numnodes < 1 || d.ncount < 0 || d.fcount < 0) {
        set_error("nleaf, numnodes must be >= 1 and pair counts >= 0");
        return MXB_ERR_ARG;
    }
    if (!d.D || !d.Dptr || !d.lchildren || !d.rchildren || !d.lm || !d.slen || !d.Ddim ||
        (d.ncount && (!d.npairx || !d.npairy)) || (d.fcount && (!d.fpairx || !d.fpairy || !d.B || !d.Bptr)) ||
        (d.numnodes > 1 && (!d.VT || !d.VTptr))) {
        set_error("null array in CDS description");
        return MXB_ERR_ARG;
    }
    nleaf = d.nleaf;
    numnodes = d.numnodes;
    is_hss = d.is_hss;
    Ddim.assign(d.Ddim, d.Ddim + nleaf);
    slen.assign(d.slen, d.slen + numnodes);
    lch.assign(d.lchildren, d.lchildren + numnodes);
    rch.assign(d.rchildren, d.rchildren + numnodes);
    lm.assign(d.lm, d.lm + numnodes);
    parent.assign(numnodes, -1);
    for (int i = 0; i < nleaf; ++i)
        if (Ddim[i] < 1) return fail("Ddim[" + std::to_string(i) + "] < 1");
    std::vector<int> leafseen(nleaf, 0);
    for (int v = 0; v < numnodes; ++v) {
        if (slen[v] < 0) return fail("negative rank at node " + std::to_string(v));
        const int l = lch[v], r = rch[v];
        if ((l == -1) != (r == -1)) return fail("node " + std::to_string(v) + " has one child");
        if (l == -1) {
            if (lm[v] < 0 || lm[v] >= nleaf) return fail("leaf " + std::to_string(v) + " has no leaf index");
            if (leafseen[lm[v]]++) return fail("leaf index used twice");
        } else {
            if (l < 0 || l >= numnodes || r < 0 || r >= numnodes || l == r || l == v || r == v)
                return fail("child index out of range at node " + std::to_string(v));
            if (parent[l] != -1 || parent[r] != -1) return fail("node with two parents");
            parent[l] = v;
            parent[r] = v;
        }
    }
    for (int i = 0; i < nleaf; ++i)
        if (!leafseen[i]) return fail("leaf index " + std::to_string(i) + " unused");
    root = -1;
    for (int v = 0; v < numnodes; ++v)
        if (parent[v] == -1) {
            if (root != -1) return fail("more than one root");
            root = v;
        }
    if (root == -1) return fail("no root");
    // depth (from root) and height (from leaves); detects cycles by counting visits
    depth.assign(numnodes, -1);
    height.assign(numnodes, 0);
    std::vector<int> order;
    order.reserve(numnodes);
    order.push_back(root);
    depth[root] = 0;
    for (size_t i = 0; i < order.size(); ++i) {
        const int v = order[i];
        if (lch[v] != -1) {
            for (int c : {lch[v], rch[v]}) {
                if (depth[c] != -1) return fail("cycle in tree");
                depth[c] = depth[v] + 1;
                order.push_back(c);
            }
        }
    }
    if ((int)order.size() != numnodes) return fail("tree does not span all nodes");
    for (int i = numnodes - 1; i >= 0; --i) {
        const int v = order[i];
        if (lch[v] != -1) height[v] = 1 + std::max(height[lch[v]], height[rch[v]]);
    }
    bfs = order;

    // ranks of leaves may not exceed their sizes' usefulness but any s >= 0 is allowed;
    // check projection extents
    VT_len = d.VT_len;
    for (int v = 0; v < numnodes; ++v) {
        if (v == root || slen[v] == 0) continue;
        const uint64_t cols = (lch[v] == -1) ? (uint64_t)Ddim[lm[v]] : (uint64_t)slen[lch[v]] + slen[rch[v]];
        if (d.VTptr[v] < 0 || (uint64_t)d.VTptr[v] + (uint64_t)slen[v] * cols > d.VT_len)
            return fail("projection of node " + std::to_string(v) + " exceeds VT");
    }
    if (slen[root] != 0 && lch[root] != -1) {
        // the reference never projects the root (cacheSkeldim starts at node 1)
    }
    VTptr.assign(d.VTptr ? d.VTptr : nullptr, d.VTptr ? d.VTptr + numnodes : nullptr);
    if (VTptr.empty()) VTptr.assign(numnodes, 0);

    near_x.assign(d.npairx, d.npairx + d.ncount);
    near_y.assign(d.npairy, d.npairy + d.ncount);
    near_off.assign(d.Dptr, d.Dptr + d.ncount);
    for (int k = 0; k < d.ncount; ++k) {
        const int x = near_x[k], y = near_y[k];
        if (x < 0 || x >= nleaf || y < 0 || y >= nleaf) return fail("near pair out of range");
        if (near_off[k] + (uint64_t)Ddim[x] * Ddim[y] > d.D_len) return fail("near block exceeds D");
    }
    far_x.assign(d.fpairx, d.fpairx + d.fcount);
    far_y.assign(d.fpairy, d.fpairy + d.fcount);
    far_off.assign(d.Bptr, d.Bptr + d.fcount);
    for (int k = 0; k < d.fcount; ++k) {
        const int x = far_x[k], y = far_y[k];
        if (x < 0 || x >= numnodes || y < 0 || y >= numnodes) return fail("far pair out of range");
        if (x == root || y == root) {
            if (slen[root] != 0) return fail("far pair touches the root");
        }
        if (far_off[k] + (uint64_t)slen[x] * slen[y] > d.B_len) return fail("far block exceeds B");
    }
    D_len = d.D_len;
    B_len = d.B_len;
    rows_total = 0;
    leaf_row.resize(nleaf);
    for (int i = 0; i < nleaf; ++i) {
        leaf_row[i] = rows_total;
        rows_total += Ddim[i];
    }
    skel_row.assign(numnodes, 0);
    skel_total = 0;
    for (int v : bfs) {
        skel_row[v] = skel_total;
        skel_total += slen[v];
    }
    return MXB_OK;
}

// ---------------------------------------------------------------------------------------
// task lists
// ---------------------------------------------------------------------------------------

void Plan::add_task(std::vector<Task> &tasks, int16_t c_kind, int64_t c_row, int ldc, int M,
                    int item0, int nitem, int16_t beta, int tile)
{
    for (int m0 = 0; m0 < M; m0 += tile) {
        Task t{};
        t.c_row = c_row;
        t.ldc = ldc;
        t.M = M;
        t.m0 = m0;
        t.item0 = item0;
        t.nitem = nitem;
        t.c_kind = c_kind;
        t.beta = beta;
        tasks.push_back(t);
    }
}

static Item make_item(int16_t pool, uint64_t a_off, int lda, int K, int trans, int16_t b_kind,
                      int64_t b_row, int ldb)
{
    Item it{};
    it.a_pool = pool;
    it.a_off = a_off;
    it.lda = lda;
    it.K = K;
    it.trans = (int16_t)trans;
    it.b_kind = b_kind;
    it.b_row = b_row;
    it.ldb = ldb;
    return it;
}

void Plan::build_tasks(int tile)
{
    items.clear();
    tasks.clear();
    launches_fwd.clear();
    launches_adj.clear();
    auto begin_launch = [&](std::vector<Launch> &L, int kind, int level) {
        Launch l{};
        l.task0 = (int)tasks.size();
        l.kind = kind;
        l.level = level;
        L.push_back(l);
    };
    auto end_launch = [&](std::vector<Launch> &L) {
        L.back().ntasks = (int)tasks.size() - L.back().task0;
        if (L.back().ntasks == 0) {
            L.pop_back();
            return;
        }
        // longest tasks first: the CTAs of a launch start in task order, so the last wave holds
        // the shortest tasks (each task owns its output tile, so the order changes no result)
        auto cost = [&](const Task &t) {
            int64_t k = 0;
            for (int q = t.item0; q < t.item0 + t.nitem; ++q) k += items[q].K;
            return k;
        };
        std::stable_sort(tasks.begin() + L.back().task0, tasks.end(),
                         [&](const Task &a, const Task &b) { return cost(a) > cost(b); });
    };
    // per-node far lists (forward: pairs (c, y) for output c; adjoint: pairs (x, c))
    std::vector<std::vector<int>> far_out(numnodes), far_in(numnodes);
    for (size_t k = 0; k < far_x.size(); ++k) {
        far_out[far_x[k]].push_back((int)k);
        far_in[far_y[k]].push_back((int)k);
    }
    std::vector<std::vector<int>> near_out(nleaf), near_in(nleaf);
    for (size_t k = 0; k < near_x.size(); ++k) {
        near_out[near_x[k]].push_back((int)k);
        near_in[near_y[k]].push_back((int)k);
    }
    int maxh = 0, maxd = 0;
    for (int v = 0; v < numnodes; ++v) {
        maxh = std::max(maxh, height[v]);
        maxd = std::max(maxd, depth[v]);
    }
    auto projects = [&](int v) { return v != root && slen[v] > 0; };

    // phases 1-2: up-sweep, shared by forward and adjoint
    std::vector<Launch> up;
    for (int h = 0; h <= maxh; ++h) {
        begin_launch(up, MXB_PHASE_UP, h);
        for (int v : bfs) {
            if (height[v] != h || !projects(v)) continue;
            const int s = slen[v];
            const int item0 = (int)items.size();
            if (lch[v] == -1) {
                const int leaf = lm[v];
                items.push_back(make_item(2, (uint64_t)VTptr[v], s, Ddim[leaf], 0, KIND_W, leaf, Ddim[leaf]));
            } else {
                const int l = lch[v], r = rch[v];
                if (slen[l] > 0)
                    items.push_back(make_item(2, (uint64_t)VTptr[v], s, slen[l], 0, KIND_WSKEL, skel_row[l], slen[l]));
                if (slen[r] > 0)
                    items.push_back(make_item(2, (uint64_t)VTptr[v] + (uint64_t)s * slen[l], s, slen[r], 0,
                                              KIND_WSKEL, skel_row[r], slen[r]));
            }
            add_task(tasks, KIND_WSKEL, skel_row[v], s, s, item0, (int)items.size() - item0, 0, tile);
        }
        end_launch(up);
    }
    launches_fwd = up;
    launches_adj = up;

    // phase 3: far + down, top-down by depth
    auto down_item = [&](int c) -> bool {
        const int p = parent[c];
        if (p < 0 || !projects(p) || slen[c] == 0) return false;
        const uint64_t off = (uint64_t)VTptr[p] + (c == rch[p] ? (uint64_t)slen[p] * slen[lch[p]] : 0);
        items.push_back(make_item(2, off, slen[p], slen[p], 1, KIND_USKEL, skel_row[p], slen[p]));
        return true;
    };
    for (int adj = 0; adj < 2; ++adj) {
        std::vector<Launch> &L = adj ? launches_adj : launches_fwd;
        for (int dd = 1; dd <= maxd; ++dd) {
            begin_launch(L, MXB_PHASE_FAR_DOWN, dd);
            for (int c : bfs) {
                if (depth[c] != dd || !projects(c)) continue;
                const int item0 = (int)items.size();
                if (!adj) {
                    for (int k : far_out[c]) {
                        const int y = far_y[k];
                        if (slen[y] == 0) continue;
                        items.push_back(make_item(1, far_off[k], slen[c], slen[y], 0, KIND_WSKEL, skel_row[y], slen[y]));
                    }
                } else {
                    for (int k : far_in[c]) {
                        const int x = far_x[k];
                        if (slen[x] == 0) continue;
                        items.push_back(make_item(1, far_off[k], slen[x], slen[x], 1, KIND_WSKEL, skel_row[x], slen[x]));
                    }
                }
                down_item(c);
                add_task(tasks, KIND_USKEL, skel_row[c], slen[c], slen[c], item0, (int)items.size() - item0, 0, tile);
            }
            end_launch(L);
        }
        // phase 4: near + leaf down
        begin_launch(L, MXB_PHASE_NEAR_LEAF_DOWN, 0);
        for (int v : bfs) {
            if (lch[v] != -1) continue;
            const int x = lm[v];
            const int item0 = (int)items.size();
            if (!adj) {
                for (int k : near_out[x]) {
                    const int y = near_y[k];
                    items.push_back(make_item(0, near_off[k], Ddim[x], Ddim[y], 0, KIND_W, y, Ddim[y]));
                }
            } else {
                for (int k : near_in[x]) {
                    const int xx = near_x[k];
                    items.push_back(make_item(0, near_off[k], Ddim[xx], Ddim[xx], 1, KIND_W, xx, Ddim[xx]));
                }
            }
            if (projects(v)) items.push_back(make_item(2, (uint64_t)VTptr[v], slen[v], slen[v], 1, KIND_USKEL, skel_row[v], slen[v]));
            add_task(tasks, KIND_Y, x, Ddim[x], Ddim[x], item0, (int)items.size() - item0, 2, tile);
        }
        end_launch(L);
    }
}

uint64_t Plan::flops(int nrhs) const
{
    uint64_t f = 0;
    for (int v = 0; v < numnodes; ++v) {
        if (v == root) continue;
        const uint64_t s = (uint64_t)slen[v];
        if (lch[v] == -1) f += 2 * s * nrhs * (uint64_t)Ddim[lm[v]];
        else f += 2 * s * ((uint64_t)slen[lch[v]] + slen[rch[v]]) * nrhs;
    }
    f *= 2;
    for (size_t k = 0; k < near_x.size(); ++k) f += 2ull * Ddim[near_x[k]] * Ddim[near_y[k]] * nrhs;
    for (size_t k = 0; k < far_x.size(); ++k) f += 2ull * slen[far_x[k]] * slen[far_y[k]] * nrhs;
    return f;
}

// ---------------------------------------------------------------------------------------
// creation, scratch, evaluation
// ---------------------------------------------------------------------------------------

int Plan::create(const mxb_cds_desc &d, int prec, Plan **out)
{
    const int flags = prec & ~0xFF;
    prec &= 0xFF;
    if (prec < MXB_PREC_FP64 || prec > MXB_PREC_SPLIT_BF16_X6 || (flags & ~MXB_PLAN_ADJOINT)) {
        set_error("unknown precision mode");
        return MXB_ERR_ARG;
    }
    std::unique_ptr<Plan> p(new Plan());
    p->precision = prec;
    p->want_adjoint = (flags & MXB_PLAN_ADJOINT) && prec != MXB_PREC_FP64;  // FP64 plans always have it
    MXB_CUDA(cudaGetDevice(&p->device));
    int rc = p->validate(d);
    if (rc) return rc;
    p->build_tasks(row_tile_for(prec));
    // FP64 CDS (host or device arrays: cudaMemcpyDefault follows the pointers)
    rc = p->alloc((void **)&p->dD, std::max<uint64_t>(d.D_len, 1) * sizeof(double));
    if (rc) return rc;
    MXB_CUDA(cudaMemcpy(p->dD, d.D, d.D_len * sizeof(double), cudaMemcpyDefault));
    rc = p->alloc((void **)&p->dB, std::max<uint64_t>(d.B_len, 1) * sizeof(double));
    if (rc) return rc;
    if (d.B_len) MXB_CUDA(cudaMemcpy(p->dB, d.B, d.B_len * sizeof(double), cudaMemcpyDefault));
    rc = p->alloc((void **)&p->dVT, std::max<uint64_t>(d.VT_len, 1) * sizeof(double));
    if (rc) return rc;
    if (d.VT_len) MXB_CUDA(cudaMemcpy(p->dVT, d.VT, d.VT_len * sizeof(double), cudaMemcpyDefault));
    rc = p->alloc((void **)&p->dTasks, p->tasks.size() * sizeof(Task));
    if (rc) return rc;
    if (!p->tasks.empty())
        MXB_CUDA(cudaMemcpy(p->dTasks, p->tasks.data(), p->tasks.size() * sizeof(Task), cudaMemcpyHostToDevice));
    rc = p->alloc((void **)&p->dItems, p->items.size() * sizeof(Item));
    if (rc) return rc;
    if (!p->items.empty())
        MXB_CUDA(cudaMemcpy(p->dItems, p->items.data(), p->items.size() * sizeof(Item), cudaMemcpyHostToDevice));
    rc = p->alloc((void **)&p->dOfs, 4 * (size_t)p->nleaf * sizeof(int32_t));
    if (rc) return rc;
    if (prec != MXB_PREC_FP64) {
        rc = p->setup_split_bf16(d);
        if (rc) return rc;
    }
    // The uploads above are synchronous copies from pageable memory, which may return before
    // their DMA has landed; the evaluations that follow run on the caller's streams, which do
    // not wait for the legacy stream.  Wait for every copy here.
    MXB_CUDA(cudaDeviceSynchronize());
    *out = p.release();
    return MXB_OK;
}

void Plan::clear_graphs()
{
    for (GraphEntry &g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
    clear_split_graphs();
}

int Plan::ensure_scratch(int nrhs)
{
    const size_t need = (size_t)std::max<int64_t>(skel_total, 1) * nrhs;
    if (need <= scratch_elems) return MXB_OK;
    clear_graphs();
    if (dWskel) {
        cudaFree(dWskel);
        cudaFree(dUskel);
        allocations.erase(std::remove(allocations.begin(), allocations.end(), (void *)dWskel), allocations.end());
        allocations.erase(std::remove(allocations.begin(), allocations.end(), (void *)dUskel), allocations.end());
        device_bytes -= 2 * scratch_elems * sizeof(double);
        dWskel = dUskel = nullptr;
        scratch_elems = 0;
    }
    int rc = alloc((void **)&dWskel, need * sizeof(double));
    if (rc) return rc;
    rc = alloc((void **)&dUskel, need * sizeof(double));
    if (rc) return rc;
    scratch_elems = need;
    return MXB_OK;
}

// Per-leaf offsets for one call; packed offsets when the caller passes none.
int Plan::stage_offsets(int slot, const int32_t *ofs, int nrhs, cudaStream_t stream)
{
    std::vector<int32_t> &host = ofs_host[slot];
    std::vector<int32_t> want(nleaf);
    if (ofs) {
        std::memcpy(want.data(), ofs, sizeof(int32_t) * nleaf);
        for (int i = 0; i < nleaf; ++i)
            if (want[i] < 0) return fail("negative leaf offset");
    } else {
        for (int i = 0; i < nleaf; ++i) {
            const int64_t o = leaf_row[i] * (int64_t)nrhs;
            if (o > INT32_MAX) return fail("packed leaf offsets overflow int32");
            want[i] = (int32_t)o;
        }
    }
    if (want != host) {
        host = want;
        MXB_CUDA(cudaMemcpyAsync(dOfs + (size_t)slot * nleaf, host.data(), sizeof(int32_t) * nleaf,
                                 cudaMemcpyHostToDevice, stream));
        MXB_CUDA(cudaStreamSynchronize(stream));
    }
    return MXB_OK;
}

int Plan::run(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs,
              const int32_t *wofs, const int32_t *yofs, int accumulate, cudaStream_t stream)
{
    if (nrhs < 1) {
        set_error("nrhs must be >= 1");
        return MXB_ERR_ARG;
    }
    if (!dW || !dY) {
        set_error("null device operand");
        return MXB_ERR_ARG;
    }
    int cur = -1;
    MXB_CUDA(cudaGetDevice(&cur));
    if (cur != device) {
        set_error("plan used on a different device than it was created on");
        return MXB_ERR_ARG;
    }
    int rc = precision == MXB_PREC_FP64 ? ensure_scratch(nrhs) : MXB_OK;  // FP64 skeleton scratch
    if (rc) return rc;
    rc = stage_offsets(0, wofs, nrhs, stream);
    if (rc) return rc;
    rc = stage_offsets(1, yofs, nrhs, stream);
    if (rc) return rc;
    if (precision != MXB_PREC_FP64) return run_split_bf16(L, dW, dY, nrhs, accumulate, stream);
    MXB_CUDA(prepare_gemm_f64());
    static const bool use_graphs = [] {
        const char *e = getenv("MXB_NO_GRAPHS");
        return !(e && *e && *e != '0');
    }();
    if (!use_graphs) return enqueue(L, dW, dY, nrhs, accumulate, stream);
    // replay a captured graph of the whole evaluation: one launch instead of dozens
    GraphEntry *hit = nullptr;
    for (GraphEntry &g : graphs)
        if (g.launches == &L && g.W == dW && g.Y == dY && g.nrhs == nrhs && g.accumulate == accumulate) hit = &g;
    if (!hit) {
        if (!capture_stream) MXB_CUDA(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking));
        MXB_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue(L, dW, dY, nrhs, accumulate, capture_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(capture_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) {
            set_error(std::string("capturing the evaluation graph: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            set_error(std::string("instantiating the evaluation graph: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
        if (graphs.size() >= 8) {
            cudaGraphExecDestroy(graphs.front().exec);
            graphs.erase(graphs.begin());
        }
        graphs.push_back(GraphEntry{&L, dW, dY, nrhs, accumulate, exec});
        hit = &graphs.back();
    }
    MXB_CUDA(cudaGraphLaunch(hit->exec, stream));
    return MXB_OK;
}

// The caller's point order: perm[t] is the row of W / Y holding tree position t (the `lids`
// order of matroxTest-V1/hcds.h:766-788).  Host or device array; checked to be a permutation.
int Plan::set_permutation(const int32_t *perm)
{
    if (!perm) return arg_fail("null permutation");
    const int64_t n = rows_total;
    std::vector<int32_t> h((size_t)n + nleaf + 1);
    MXB_CUDA(cudaMemcpy(h.data(), perm, sizeof(int32_t) * (size_t)n, cudaMemcpyDefault));
    std::vector<char> seen((size_t)n, 0);
    for (int64_t t = 0; t < n; ++t) {
        const int32_t q = h[(size_t)t];
        if (q < 0 || q >= n || seen[(size_t)q]) return arg_fail("perm is not a permutation of the plan's rows");
        seen[(size_t)q] = 1;
    }
    for (int i = 0; i <= nleaf; ++i) h[(size_t)n + i] = (int32_t)(i < nleaf ? leaf_row[i] : n);
    if (!dTree) {
        int rc = alloc((void **)&dTree, h.size() * sizeof(int32_t));
        if (rc) return rc;
    }
    MXB_CUDA(cudaMemcpy(dTree, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    MXB_CUDA(cudaDeviceSynchronize());  // a pageable upload may return before it lands
    return MXB_OK;
}

// dY (+)= K~ dW (or K~^T) with dW / dY in the caller's point order.  Split-BF16 forward
// evaluations gather W's rows inside the launch that splits W into operand tiles and scatter
// Y's rows in the epilogues that write Y: no extra pass over either matrix.  Other paths
// (FP64, the adjoint) permute into leaf-blocked copies, evaluate, and permute back.
int Plan::run_ordered(bool adjoint, const double *dW, int64_t w_rs, int64_t w_cs, double *dY, int64_t y_rs,
                      int64_t y_cs, int nrhs, int accumulate, cudaStream_t stream)
{
    if (!dTree) return arg_fail("no point order set (mxb_plan_set_permutation)");
    if (!dW || !dY || nrhs < 1) return arg_fail("bad caller-order operands");
    const int64_t n = rows_total;
    // distinct elements must not alias: one stride has to step over the whole other extent
    auto separated = [&](int64_t rs, int64_t cs) {
        return rs >= 1 && cs >= 1 && (rs >= (int64_t)nrhs * cs || cs >= n * rs);
    };
    if (!separated(w_rs, w_cs) || !separated(y_rs, y_cs)) return arg_fail("caller-order strides overlap");
    const std::vector<Launch> &L = adjoint ? launches_adj : launches_fwd;
    if (precision != MXB_PREC_FP64 && !adjoint) {
        int cur = -1;
        MXB_CUDA(cudaGetDevice(&cur));
        if (cur != device) return arg_fail("plan used on a different device than it was created on");
        int rc = stage_offsets(0, nullptr, nrhs, stream);
        if (!rc) rc = stage_offsets(1, nullptr, nrhs, stream);
        if (rc) return rc;
        const CallerOrder o{dTree, dTree + n, w_rs, w_cs, y_rs, y_cs};
        return run_split_bf16(L, dW, dY, nrhs, accumulate, stream, &o);
    }
    const size_t need = (size_t)std::max<int64_t>(n, 1) * nrhs;
    if (need > order_elems) {
        for (double **q : {&dTW, &dTY}) {
            if (!*q) continue;
            cudaFree(*q);
            allocations.erase(std::remove(allocations.begin(), allocations.end(), (void *)*q), allocations.end());
            *q = nullptr;
        }
        device_bytes -= 2 * order_elems * sizeof(double);
        order_elems = 0;
        int rc = alloc((void **)&dTW, need * sizeof(double));
        if (!rc) rc = alloc((void **)&dTY, need * sizeof(double));
        if (rc) return rc;
        order_elems = need;
    }
    int rc = stage_offsets(0, nullptr, nrhs, stream);  // packed blocks of the leaf-blocked copies
    if (rc) return rc;
    MXB_CUDA(launch_permute(dTree, dTree + n, dOfs, nleaf, n, dW, dTW, w_rs, w_cs, nrhs, 0, 0, stream));
    rc = run(L, dTW, dTY, nrhs, nullptr, nullptr, 0, stream);
    if (rc) return rc;
    MXB_CUDA(launch_permute(dTree, dTree + n, dOfs + nleaf, nleaf, n, dTY, dY, y_rs, y_cs, nrhs, 1, accumulate,
                            stream));
    return MXB_OK;
}

int Plan::enqueue(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, int accumulate,
                  cudaStream_t stream)
{
    if (precision != MXB_PREC_FP64) return run_split_bf16(L, dW, dY, nrhs, accumulate, stream);
    Operands ops{};
    ops.pool[0] = dD;
    ops.pool[1] = dB;
    ops.pool[2] = dVT;
    ops.W = dW;
    ops.Y = dY;
    ops.wskel = dWskel;
    ops.uskel = dUskel;
    ops.wofs = dOfs;
    ops.yofs = dOfs + nleaf;
    ops.nrhs = nrhs;
    ops.beta_arg = accumulate ? 1 : 0;
    for (const Launch &l : L) {
        cudaError_t e = launch_gemm_f64(dTasks + l.task0, dItems, l.ntasks, ops, stream);
        if (e != cudaSuccess) {
            set_error(std::string("FP64 grouped GEMM launch: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
    }
    return MXB_OK;
}

// Launch-by-launch timing of the forward evaluation (mxb_plan_profile).
int Plan::profile(const double *dW, double *dY, int nrhs, cudaStream_t stream, mxb_op_profile *out, int cap,
                  int *nops)
{
    int rc = run(launches_fwd, dW, dY, nrhs, nullptr, nullptr, 0, stream);  // checks, offsets, graphs, tuning
    if (rc) return rc;
    if (precision != MXB_PREC_FP64) return batch_profile(split_bf16_batch(*this), &dW, &dY, &nrhs, stream, out, cap, nops);
    const std::vector<Launch> &L = launches_fwd;
    const int tile = row_tile_for(precision), ncol = (int)((nrhs + tile - 1) / tile);
    std::vector<cudaEvent_t> ev(L.size() + 1, nullptr);
    for (cudaEvent_t &e : ev)
        if (!rc && cudaEventCreate(&e) != cudaSuccess) {
            set_error("profile: creating CUDA events failed");
            rc = MXB_ERR_CUDA;
        }
    for (int rep = 0; rep < 2 && !rc; ++rep) {
        cudaEventRecord(ev[0], stream);
        for (size_t i = 0; i < L.size() && !rc; ++i) {
            rc = enqueue(std::vector<Launch>{L[i]}, dW, dY, nrhs, 0, stream);
            cudaEventRecord(ev[i + 1], stream);
        }
        if (!rc && cudaStreamSynchronize(stream) != cudaSuccess) {
            set_error("profile: stream synchronisation failed");
            rc = MXB_ERR_CUDA;
        }
    }
    if (nops) *nops = (int)L.size();
    for (size_t i = 0; i < L.size() && !rc && (int)i < cap && out; ++i) {
        const Launch &l = L[i];
        mxb_op_profile &o = out[i];
        o = mxb_op_profile{};
        o.phase = l.kind;
        o.level = l.level;
        o.width = tile;
        o.units = l.ntasks * ncol;
        for (int t = l.task0; t < l.task0 + l.ntasks; ++t) {
            const Task &T = tasks[t];
            const double rows = std::min(tile, T.M - T.m0);
            for (int k = T.item0; k < T.item0 + T.nitem; ++k) {
                o.flops += 2.0 * rows * items[k].K * nrhs;
                o.issued_flops += 2.0 * tile * items[k].K * (double)ncol * tile;
            }
        }
        cudaEventElapsedTime(&o.ms, ev[i], ev[i + 1]);
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

int Plan::read_workspaces(int nrhs, const int32_t *wsko, double *wskel, const int32_t *usko, double *uskel)
{
    if (precision != MXB_PREC_FP64) {
        set_error("skeleton workspaces are kept by FP64 plans only");
        return MXB_ERR_UNSUPPORTED;
    }
    if (!dWskel || scratch_elems < (size_t)skel_total * nrhs) {
        set_error("no evaluation with this nrhs has run on the plan");
        return MXB_ERR_ARG;
    }
    MXB_CUDA(cudaDeviceSynchronize());
    std::vector<double> w((size_t)skel_total * nrhs), u((size_t)skel_total * nrhs);
    MXB_CUDA(cudaMemcpy(w.data(), dWskel, w.size() * sizeof(double), cudaMemcpyDeviceToHost));
    MXB_CUDA(cudaMemcpy(u.data(), dUskel, u.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int v = 0; v < numnodes; ++v) {
        const size_t n = (size_t)slen[v] * nrhs;
        if (!n) continue;
        if (wskel && wsko) std::memcpy(wskel + wsko[v], w.data() + skel_row[v] * nrhs, n * sizeof(double));
        if (uskel && usko) std::memcpy(uskel + usko[v], u.data() + skel_row[v] * nrhs, n * sizeof(double));
    }
    return MXB_OK;
}

}  // namespace mxb
