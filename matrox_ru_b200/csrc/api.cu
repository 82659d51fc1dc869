// C-ABI entry points: the reference-signature drop-ins (host arrays, synchronous) and the
// device-pointer plan API.
#include <algorithm>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"
#include "plan.h"

using namespace mxb;

#define API_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return MXB_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

namespace {

std::mutex g_mu;
int g_precision = MXB_PREC_FP64;
uint32_t g_flags = 0;
int g_shape_nrow = -1, g_shape_frow = -1, g_shape_cdepth = -1;
int g_hss_nleaf = -1, g_hss_cdepth = -1;

// ---- device copy cache of CDSs seen by the drop-ins ----
struct CacheEntry {
    uint64_t key;
    int device;
    int precision;
    std::unique_ptr<Plan> plan;
};
std::list<CacheEntry> g_cache;  // most recent first
constexpr size_t kCacheSlots = 4;

// Per-device state of the drop-ins.  An evaluation runs over column slabs of the right-hand
// sides: slab k's upload (stream `in`), evaluation (`stream`) and download (`out`) overlap with
// the neighbouring slabs', with two W and two Y slab buffers in rotation.
struct DeviceBuffers {
    int device = -1;
    cudaStream_t stream = nullptr, in = nullptr, out = nullptr;
    double *W[2] = {nullptr, nullptr}, *Y[2] = {nullptr, nullptr};
    size_t wcap[2] = {0, 0}, ycap[2] = {0, 0};
    cudaEvent_t uploaded[2] = {}, computed[2] = {}, downloaded[2] = {};
};
DeviceBuffers g_buf[64];

uint64_t fnv(uint64_t h, const void *p, size_t n)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}
template <class T>
uint64_t fnv_arr(uint64_t h, const T *p, size_t n)
{
    return p ? fnv(h, p, n * sizeof(T)) : fnv(h, "null", 4);
}
// sample of a numeric pool: length, first, last and ~4096 evenly spaced values
uint64_t fnv_sample(uint64_t h, const double *p, uint64_t n)
{
    h = fnv(h, &n, sizeof(n));
    if (!p || !n) return h;
    const uint64_t step = std::max<uint64_t>(1, n / 4096);
    for (uint64_t i = 0; i < n; i += step) h = fnv(h, p + i, sizeof(double));
    return fnv(h, p + n - 1, sizeof(double));
}

// every word of a numeric pool: four independent multiply-rotate lanes over 64-bit words
uint64_t hash_full(uint64_t h, const double *p, uint64_t n)
{
    h = fnv(h, &n, sizeof(n));
    if (!p || !n) return h;
    const uint64_t *w = reinterpret_cast<const uint64_t *>(p);
    uint64_t a[4] = {h, h ^ 0x9e3779b97f4a7c15ull, h ^ 0xc2b2ae3d27d4eb4full, h ^ 0x165667b19e3779f9ull};
    uint64_t i = 0;
    for (; i + 4 <= n; i += 4)
        for (int k = 0; k < 4; ++k) {
            a[k] ^= w[i + k];
            a[k] *= 0x9fb21c651e98df25ull;
            a[k] = (a[k] << 29) | (a[k] >> 35);
        }
    for (; i < n; ++i) a[0] = (a[0] ^ w[i]) * 0x9fb21c651e98df25ull;
    return fnv(h, a, sizeof(a));
}

int g_cache_mode = MXB_CACHE_SAMPLED;

uint64_t desc_key(const mxb_cds_desc &d)
{
    uint64_t h = 1469598103934665603ull;
    const void *ptrs[] = {d.D, d.B, d.VT};
    h = fnv(h, ptrs, sizeof(ptrs));
    h = fnv(h, &d.nleaf, sizeof(int32_t) * 3);
    if (g_cache_mode == MXB_CACHE_FULL) {
        h = hash_full(h, d.D, d.D_len);
        h = hash_full(h, d.B, d.B_len);
        h = hash_full(h, d.VT, d.VT_len);
    } else {
        h = fnv_sample(h, d.D, d.D_len);
        h = fnv_sample(h, d.B, d.B_len);
        h = fnv_sample(h, d.VT, d.VT_len);
    }
    h = fnv_arr(h, d.Dptr, d.ncount);
    h = fnv_arr(h, d.Bptr, d.fcount);
    h = fnv_arr(h, d.VTptr, d.numnodes);
    h = fnv_arr(h, d.lchildren, d.numnodes);
    h = fnv_arr(h, d.rchildren, d.numnodes);
    h = fnv_arr(h, d.lm, d.numnodes);
    h = fnv_arr(h, d.slen, d.numnodes);
    h = fnv_arr(h, d.Ddim, d.nleaf);
    h = fnv_arr(h, d.npairx, d.ncount);
    h = fnv_arr(h, d.npairy, d.ncount);
    h = fnv_arr(h, d.fpairx, d.fcount);
    h = fnv_arr(h, d.fpairy, d.fcount);
    return h;
}

int cached_plan(const mxb_cds_desc &d, Plan **out)
{
    int dev = 0;
    API_CUDA(cudaGetDevice(&dev));
    if (g_cache_mode == MXB_CACHE_OFF) g_cache.clear();
    const uint64_t key = desc_key(d);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
        if (it->key == key && it->device == dev && it->precision == g_precision) {
            g_cache.splice(g_cache.begin(), g_cache, it);
            *out = g_cache.front().plan.get();
            return MXB_OK;
        }
    }
    Plan *p = nullptr;
    int rc = Plan::create(d, g_precision, &p);
    if (rc) return rc;
    g_cache.push_front(CacheEntry{key, dev, g_precision, std::unique_ptr<Plan>(p)});
    while (g_cache.size() > kCacheSlots) g_cache.pop_back();
    *out = p;
    return MXB_OK;
}

DeviceBuffers *buffers()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    DeviceBuffers &b = g_buf[dev];
    if (!b.stream) {
        cudaStream_t s[3] = {};
        cudaEvent_t e[6] = {};
        bool ok = true;
        for (cudaStream_t &x : s) ok = ok && cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) == cudaSuccess;
        for (cudaEvent_t &x : e) ok = ok && cudaEventCreateWithFlags(&x, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            for (cudaStream_t x : s)
                if (x) cudaStreamDestroy(x);
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
            return nullptr;
        }
        b.in = s[1];
        b.out = s[2];
        for (int i = 0; i < 2; ++i) {
            b.uploaded[i] = e[i];
            b.computed[i] = e[2 + i];
            b.downloaded[i] = e[4 + i];
        }
        b.device = dev;
        b.stream = s[0];
    }
    return &b;
}

// Columns per slab of a drop-in evaluation: about eight slabs, at least 128 columns each
// (narrower slabs lose tensor-core efficiency), a multiple of 64.  MXB_DROPIN_SLAB=<columns>
// overrides it; MXB_DROPIN_SLAB=0 evaluates all columns as one slab.
int slab_columns(int nrhs)
{
    static const int forced = [] {
        const char *e = getenv("MXB_DROPIN_SLAB");
        return e && *e ? atoi(e) : -1;
    }();
    if (forced == 0) return nrhs;
    if (forced > 0) return std::min(forced, nrhs);
    const int c = ((nrhs + 7) / 8 + 63) / 64 * 64;
    return std::min(nrhs, std::max(128, c));
}

// Copies columns [j0, j0 + cw) of every leaf block between the caller's host array (leaf i's
// block, Ddim[i] x nrhs column-major, at element offset hofs[i]) and a packed device slab
// (leaf i's block, Ddim[i] x cw, at leaf_row[i] * cw).  Runs of leaves with equal sizes and
// evenly spaced host blocks move as one 2-D copy.
cudaError_t copy_slab(const Plan &p, double *host, const int32_t *hofs, double *dev, int j0, int cw, bool to_device,
                      cudaStream_t s)
{
    const int n = p.nleaf;
    for (int i = 0; i < n;) {
        const int m = p.Ddim[i];
        int g = 1;
        const int64_t stride = i + 1 < n ? (int64_t)hofs[i + 1] - hofs[i] : 0;
        if (m > 0 && stride >= (int64_t)m * cw && stride * (int64_t)sizeof(double) < (int64_t)INT32_MAX)
            while (i + g < n && p.Ddim[i + g] == m && (int64_t)hofs[i + g] - hofs[i + g - 1] == stride) ++g;
        if (m > 0) {
            double *h = host + hofs[i] + (size_t)j0 * m;
            double *d = dev + (size_t)p.leaf_row[i] * cw;
            const size_t width = (size_t)m * cw * sizeof(double);
            cudaError_t e;
            if (g == 1)
                e = cudaMemcpyAsync(to_device ? (void *)d : (void *)h, to_device ? (const void *)h : (const void *)d,
                                    width, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, s);
            else if (to_device)
                e = cudaMemcpy2DAsync(d, width, h, (size_t)stride * sizeof(double), width, g, cudaMemcpyHostToDevice, s);
            else
                e = cudaMemcpy2DAsync(h, (size_t)stride * sizeof(double), d, width, width, g, cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) return e;
        }
        i += g;
    }
    return cudaSuccess;
}

int grow(double **p, size_t *cap, size_t elems)
{
    if (elems <= *cap) return MXB_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, std::max<size_t>(elems, 1) * sizeof(double));
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc for drop-in operands: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? MXB_ERR_NOMEM : MXB_ERR_CUDA;
    }
    *cap = elems;
    return MXB_OK;
}

// Flat pair list from the reference's CSR-of-CSR blocking (nblockSet -> nblocks -> pairs);
// the pair index k addresses Dptr / Bptr directly, as in codeGen/H2GEMM.h:395-404.
int flatten_blocked(const int32_t *set, const int32_t *blocks, int nrow, std::vector<int> &ks)
{
    ks.clear();
    if (nrow < 0) {
        set_error("negative block-row count");
        return MXB_ERR_ARG;
    }
    if (nrow == 0) return MXB_OK;
    if (!set || !blocks) {
        set_error("null blocking array");
        return MXB_ERR_ARG;
    }
    for (int i = 0; i < nrow; ++i) {
        if (set[i] > set[i + 1] || set[i] < 0) {
            set_error("blockset not monotone");
            return MXB_ERR_STRUCTURE;
        }
        for (int j = set[i]; j < set[i + 1]; ++j) {
            if (blocks[j] > blocks[j + 1] || blocks[j] < 0) {
                set_error("blocks not monotone");
                return MXB_ERR_STRUCTURE;
            }
            for (int k = blocks[j]; k < blocks[j + 1]; ++k) ks.push_back(k);
        }
    }
    return MXB_OK;
}

struct DropIn {
    // reference arrays
    double *D, *B, *VT;
    uint64_t *Dptr, *Bptr;
    int32_t *VTptr, *lch, *rch, *Ddim, *wptr, *uptr, *wsko, *usko, *lm, *slen;
    double *mrhs, *apres, *wskel, *uskel;
    int32_t nrhs;
    int nleaf, numnodes;
    bool hss;
    std::vector<int32_t> px, py, fx, fy;
    std::vector<uint64_t> dofs, bofs;
};

int run_dropin(DropIn &a)
{
    if (!a.D || !a.VT || !a.Dptr || !a.VTptr || !a.lch || !a.rch || !a.Ddim || !a.wptr || !a.uptr || !a.lm ||
        !a.slen || !a.mrhs || !a.apres) {
        set_error("null argument");
        return MXB_ERR_ARG;
    }
    if (a.nrhs < 1 || a.nleaf < 1 || a.numnodes < 1) {
        set_error("nrhs, nleaf and numnodes must be >= 1");
        return MXB_ERR_ARG;
    }
    // array extents implied by the offsets (the reference passes none)
    uint64_t D_len = 0, B_len = 0, VT_len = 0;
    for (size_t k = 0; k < a.px.size(); ++k) {
        const int x = a.px[k], y = a.py[k];
        if (x < 0 || x >= a.nleaf || y < 0 || y >= a.nleaf) {
            set_error("near pair index out of range");
            return MXB_ERR_STRUCTURE;
        }
        D_len = std::max<uint64_t>(D_len, a.dofs[k] + (uint64_t)a.Ddim[x] * a.Ddim[y]);
    }
    for (size_t k = 0; k < a.fx.size(); ++k) {
        const int x = a.fx[k], y = a.fy[k];
        if (x < 0 || x >= a.numnodes || y < 0 || y >= a.numnodes) {
            set_error("far pair index out of range");
            return MXB_ERR_STRUCTURE;
        }
        B_len = std::max<uint64_t>(B_len, a.bofs[k] + (uint64_t)a.slen[x] * a.slen[y]);
    }
    for (int v = 0; v < a.numnodes; ++v) {
        if (a.slen[v] <= 0) continue;
        const int l = a.lch[v], r = a.rch[v];
        uint64_t cols;
        if (l == -1) {
            if (a.lm[v] < 0 || a.lm[v] >= a.nleaf) {
                set_error("leaf map out of range");
                return MXB_ERR_STRUCTURE;
            }
            cols = (uint64_t)a.Ddim[a.lm[v]];
        } else {
            if (l < 0 || l >= a.numnodes || r < 0 || r >= a.numnodes) {
                set_error("child index out of range");
                return MXB_ERR_STRUCTURE;
            }
            cols = (uint64_t)a.slen[l] + a.slen[r];
        }
        if (a.VTptr[v] < 0) {
            set_error("negative VTptr");
            return MXB_ERR_STRUCTURE;
        }
        VT_len = std::max<uint64_t>(VT_len, (uint64_t)a.VTptr[v] + (uint64_t)a.slen[v] * cols);
    }
    if (!a.fx.empty() && !a.B) {
        set_error("null B with far pairs");
        return MXB_ERR_ARG;
    }
    mxb_cds_desc d{};
    d.nleaf = a.nleaf;
    d.numnodes = a.numnodes;
    d.is_hss = a.hss;
    d.D = a.D;
    d.D_len = D_len;
    d.B = a.B;
    d.B_len = B_len;
    d.VT = a.VT;
    d.VT_len = VT_len;
    d.Dptr = a.dofs.data();
    d.Bptr = a.bofs.data();
    d.VTptr = a.VTptr;
    d.lchildren = a.lch;
    d.rchildren = a.rch;
    d.lm = a.lm;
    d.slen = a.slen;
    d.Ddim = a.Ddim;
    d.npairx = a.px.data();
    d.npairy = a.py.data();
    d.ncount = (int32_t)a.px.size();
    d.fpairx = a.fx.data();
    d.fpairy = a.fy.data();
    d.fcount = (int32_t)a.fx.size();

    std::lock_guard<std::mutex> lock(g_mu);
    Plan *plan = nullptr;
    int rc = cached_plan(d, &plan);
    if (rc) return rc;
    DeviceBuffers *buf = buffers();
    if (!buf) {
        set_error("cannot create the drop-in stream");
        return MXB_ERR_CUDA;
    }
    for (int i = 0; i < a.nleaf; ++i) {
        if (a.wptr[i] < 0 || a.uptr[i] < 0) {
            set_error("negative leaf offset");
            return MXB_ERR_STRUCTURE;
        }
    }
    const bool mirror = (g_flags & MXB_FLAG_MIRROR_WORKSPACES) && plan->precision == MXB_PREC_FP64;
    // Column slabs: the skeleton workspaces of one evaluation cover only its own columns, so
    // mirroring them back needs all columns in one slab.
    const int cw = mirror ? a.nrhs : slab_columns(a.nrhs);
    const int nslab = (a.nrhs + cw - 1) / cw;
    const size_t slab_elems = (size_t)std::max<int64_t>(plan->rows_total, 1) * cw;
    for (int b = 0; b < std::min(nslab, 2); ++b) {
        rc = grow(&buf->W[b], &buf->wcap[b], slab_elems);
        if (rc) return rc;
        rc = grow(&buf->Y[b], &buf->ycap[b], slab_elems);
        if (rc) return rc;
    }
    // H2-b accumulates into apres (near beta = 1), HSS overwrites it
    const bool upload_y = !a.hss && !(g_flags & MXB_FLAG_OUTPUT_IS_ZERO);
    // slab k uses buffers k % 2.  Upload k waits until evaluation k-2 has read W[b] (and, for
    // an uploaded Y, until download k-2 has read Y[b]); evaluation k waits for upload k and for
    // download k-2; download k waits for evaluation k.
    for (int k = 0; k < nslab; ++k) {
        const int b = k & 1, j0 = k * cw, w = std::min(cw, a.nrhs - j0);
        if (k >= 2) {
            API_CUDA(cudaStreamWaitEvent(buf->in, buf->computed[b], 0));
            if (upload_y) API_CUDA(cudaStreamWaitEvent(buf->in, buf->downloaded[b], 0));
        }
        API_CUDA(copy_slab(*plan, a.mrhs, a.wptr, buf->W[b], j0, w, true, buf->in));
        if (upload_y) API_CUDA(copy_slab(*plan, a.apres, a.uptr, buf->Y[b], j0, w, true, buf->in));
        API_CUDA(cudaEventRecord(buf->uploaded[b], buf->in));
        API_CUDA(cudaStreamWaitEvent(buf->stream, buf->uploaded[b], 0));
        if (k >= 2) API_CUDA(cudaStreamWaitEvent(buf->stream, buf->downloaded[b], 0));
        // a Y known to be zero is overwritten instead of accumulated into
        rc = plan->run(plan->launches_fwd, buf->W[b], buf->Y[b], w, nullptr, nullptr, upload_y ? 1 : 0,
                       buf->stream);
        if (rc) {
            cudaDeviceSynchronize();
            return rc;
        }
        API_CUDA(cudaEventRecord(buf->computed[b], buf->stream));
        API_CUDA(cudaStreamWaitEvent(buf->out, buf->computed[b], 0));
        API_CUDA(copy_slab(*plan, a.apres, a.uptr, buf->Y[b], j0, w, false, buf->out));
        API_CUDA(cudaEventRecord(buf->downloaded[b], buf->out));
    }
    API_CUDA(cudaStreamSynchronize(buf->out));
    API_CUDA(cudaStreamSynchronize(buf->stream));
    if (mirror) {
        rc = plan->read_workspaces(a.nrhs, a.wsko, a.wskel, a.usko, a.uskel);
        if (rc) return rc;
    }
    return MXB_OK;
}

void fill_common(DropIn &a, double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                 int32_t *lchildren, int32_t *rchildren, double *mrhs, double *apres, int32_t nrhs,
                 int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel, int32_t *wskeloffset, double *uskel,
                 int32_t *uskeloffset, int32_t *lm, int32_t *slen)
{
    a.D = D;
    a.B = B;
    a.VT = VT;
    a.Dptr = Dptr;
    a.Bptr = Bptr;
    a.VTptr = VTptr;
    a.lch = lchildren;
    a.rch = rchildren;
    a.mrhs = mrhs;
    a.apres = apres;
    a.nrhs = nrhs;
    a.Ddim = Ddim;
    a.wptr = wptr;
    a.uptr = uptr;
    a.wskel = wskel;
    a.wsko = wskeloffset;
    a.uskel = uskel;
    a.usko = uskeloffset;
    a.lm = lm;
    a.slen = slen;
}

// numnodes from a schedule: the coarsened (or plain) level sets list every node but the
// root once, so numnodes = entries + 1 and nleaf = (numnodes + 1) / 2 for a full binary tree.
int sizes_from_schedule(int entries, DropIn &a)
{
    if (entries < 0) {
        set_error("schedule arrays are inconsistent");
        return MXB_ERR_STRUCTURE;
    }
    a.numnodes = entries + 1;
    a.nleaf = (a.numnodes + 1) / 2;
    return MXB_OK;
}

int h2b_common(DropIn &a, int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy,
               int32_t *fblockSet, int32_t *fblocks, int32_t *fpairx, int32_t *fpairy, int nrow, int frow)
{
    std::vector<int> ks;
    int rc = flatten_blocked(nblockSet, nblocks, nrow, ks);
    if (rc) return rc;
    if (!ks.empty() && (!npairx || !npairy)) {
        set_error("null near pair arrays");
        return MXB_ERR_ARG;
    }
    a.hss = false;
    for (int k : ks) {
        a.px.push_back(npairx[k]);
        a.py.push_back(npairy[k]);
        a.dofs.push_back(a.Dptr[k]);
    }
    rc = flatten_blocked(fblockSet, fblocks, frow, ks);
    if (rc) return rc;
    if (!ks.empty() && (!fpairx || !fpairy || !a.Bptr)) {
        set_error("null far pair arrays");
        return MXB_ERR_ARG;
    }
    for (int k : ks) {
        a.fx.push_back(fpairx[k]);
        a.fy.push_back(fpairy[k]);
        a.bofs.push_back(a.Bptr[k]);
    }
    return run_dropin(a);
}

int hss_common(DropIn &a, int ncount, int fcount)
{
    a.hss = true;
    if (ncount != a.nleaf || fcount != a.numnodes - 1) {
        set_error("HSS ncount / fcount do not match the level sets (ncount = leaves, fcount = numnodes - 1)");
        return MXB_ERR_STRUCTURE;
    }
    for (int i = 0; i < ncount; ++i) {
        a.px.push_back(i);
        a.py.push_back(i);
        a.dofs.push_back(a.Dptr[i]);
    }
    if (fcount > 0 && !a.Bptr) {
        set_error("null Bptr");
        return MXB_ERR_ARG;
    }
    for (int i = 1; i < fcount + 1; ++i) {
        a.fx.push_back(i);
        a.fy.push_back((i & 1) == 0 ? i - 1 : i + 1);
        a.bofs.push_back(a.Bptr[i - 1]);
    }
    return run_dropin(a);
}

int coarse_entries(const int32_t *wpart, const int32_t *clevelset, int cdepth)
{
    if (!wpart || !clevelset || cdepth < 0) return -1;
    return wpart[clevelset[cdepth]] - wpart[clevelset[0]];
}

}  // namespace

extern "C" {

const char *mxb_last_error(void) { return mxb::last_error(); }
const char *mxb_version(void) { return "matrox_b200 0.1 (sm_100a)"; }

int32_t mxb_set_precision(int32_t mode)
{
    if (mode < MXB_PREC_FP64 || mode > MXB_PREC_SPLIT_BF16_X6) {
        set_error("unknown precision mode");
        return MXB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_precision = mode;
    return MXB_OK;
}

int32_t mxb_set_flags(uint32_t flags)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_flags = flags;
    return MXB_OK;
}

int32_t mxb_cache_invalidate(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_cache.clear();
    return MXB_OK;
}

int32_t mxb_cache_set_mode(int32_t mode)
{
    if (mode != MXB_CACHE_SAMPLED && mode != MXB_CACHE_FULL && mode != MXB_CACHE_OFF) {
        set_error("mxb_cache_set_mode: mode must be MXB_CACHE_SAMPLED, MXB_CACHE_FULL or MXB_CACHE_OFF");
        return MXB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_cache_mode = mode;
    g_cache.clear();
    return MXB_OK;
}

int32_t CBHGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy, int32_t *fblockSet,
                int32_t *fblocks, int32_t *fpairx, int32_t *fpairy, int32_t ncount, int32_t fcount,
                int32_t *wpart, int32_t *clevelset, int cdepth)
{
    (void)levelset;
    (void)idx;
    DropIn a{};
    fill_common(a, D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
                wskeloffset, uskel, uskeloffset, lm, slen);
    int rc = sizes_from_schedule(coarse_entries(wpart, clevelset, cdepth), a);
    if (rc) return rc;
    return h2b_common(a, nblockSet, nblocks, npairx, npairy, fblockSet, fblocks, fpairx, fpairy, ncount, fcount);
}

int32_t lowH2GEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                  int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                  double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                  int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy, int32_t *fblockSet,
                  int32_t *fblocks, int32_t *fpairx, int32_t *fpairy, int32_t ncount, int32_t fcount,
                  int32_t *wpart, int32_t *clevelset, int cdepth)
{
    return CBHGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres, nrhs, Ddim, wptr,
                   uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen, nblockSet, nblocks, npairx, npairy,
                   fblockSet, fblocks, fpairx, fpairy, ncount, fcount, wpart, clevelset, cdepth);
}

int32_t blockGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                  int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                  double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                  int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy, int32_t *fblockSet,
                  int32_t *fblocks, int32_t *fpairx, int32_t *fpairy, int32_t ncount, int32_t fcount,
                  int32_t depth)
{
    (void)idx;
    DropIn a{};
    fill_common(a, D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
                wskeloffset, uskel, uskeloffset, lm, slen);
    if (!levelset || depth < 0) {
        set_error("null levelset");
        return MXB_ERR_ARG;
    }
    int rc = sizes_from_schedule(levelset[depth] - levelset[0], a);
    if (rc) return rc;
    return h2b_common(a, nblockSet, nblocks, npairx, npairy, fblockSet, fblocks, fpairx, fpairy, ncount, fcount);
}

int32_t mxb_hgemm_set_shape(int32_t nrow, int32_t frow, int32_t cdepth)
{
    if (nrow < 0 || frow < 0 || cdepth < 0) {
        set_error("negative shape");
        return MXB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_shape_nrow = nrow;
    g_shape_frow = frow;
    g_shape_cdepth = cdepth;
    return MXB_OK;
}

int32_t HGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
              int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
              double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
              int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
              int32_t *nblockSet, int32_t *nblocks, int32_t *npairx, int32_t *npairy, int32_t *fblockSet,
              int32_t *fblocks, int32_t *fpairx, int32_t *fpairy, int32_t *wpart, int32_t *clevelset)
{
    int nrow, frow, cdepth;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        nrow = g_shape_nrow;
        frow = g_shape_frow;
        cdepth = g_shape_cdepth;
    }
    if (nrow < 0) {
        set_error("HGEMM: call mxb_hgemm_set_shape first (the generated code bakes these sizes in)");
        return MXB_ERR_ARG;
    }
    return CBHGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres, nrhs, Ddim, wptr,
                   uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen, nblockSet, nblocks, npairx, npairy,
                   fblockSet, fblocks, fpairx, fpairy, nrow, frow, wpart, clevelset, cdepth);
}

int32_t parHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                   int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                   double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                   int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t *wpart, int32_t *clevelset, int ncount, int fcount, int cdepth)
{
    (void)levelset;
    (void)idx;
    DropIn a{};
    fill_common(a, D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
                wskeloffset, uskel, uskeloffset, lm, slen);
    int rc = sizes_from_schedule(coarse_entries(wpart, clevelset, cdepth), a);
    if (rc) return rc;
    return hss_common(a, ncount, fcount);
}

int32_t lowHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                   int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                   double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                   int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t *wpart, int32_t *clevelset, int ncount, int fcount, int cdepth)
{
    return parHSSGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres, nrhs, Ddim,
                      wptr, uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, ncount, fcount,
                      cdepth);
}

int32_t seqHSSGEMM(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                   int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                   double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                   int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                   int32_t ncount, int32_t fcount, int32_t depth)
{
    (void)idx;
    DropIn a{};
    fill_common(a, D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, mrhs, apres, nrhs, Ddim, wptr, uptr, wskel,
                wskeloffset, uskel, uskeloffset, lm, slen);
    if (!levelset || depth < 0) {
        set_error("null levelset");
        return MXB_ERR_ARG;
    }
    int rc = sizes_from_schedule(levelset[depth] - levelset[0], a);
    if (rc) return rc;
    return hss_common(a, ncount, fcount);
}

int32_t mxb_hgemm_hss_set_shape(int32_t nleaf, int32_t cdepth)
{
    if (nleaf < 1 || cdepth < 0) {
        set_error("bad HSS shape");
        return MXB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_hss_nleaf = nleaf;
    g_hss_cdepth = cdepth;
    return MXB_OK;
}

int32_t HGEMM_HSS(double *D, double *B, double *VT, uint64_t *Dptr, uint64_t *Bptr, int32_t *VTptr,
                  int32_t *lchildren, int32_t *rchildren, int32_t *levelset, int32_t *idx, double *mrhs,
                  double *apres, int32_t nrhs, int32_t *Ddim, int32_t *wptr, int32_t *uptr, double *wskel,
                  int32_t *wskeloffset, double *uskel, int32_t *uskeloffset, int32_t *lm, int32_t *slen,
                  int32_t *wpart, int32_t *clevelset)
{
    int nleaf, cdepth;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        nleaf = g_hss_nleaf;
        cdepth = g_hss_cdepth;
    }
    if (nleaf < 1) {
        set_error("HGEMM_HSS: call mxb_hgemm_hss_set_shape first");
        return MXB_ERR_ARG;
    }
    return parHSSGEMM(D, B, VT, Dptr, Bptr, VTptr, lchildren, rchildren, levelset, idx, mrhs, apres, nrhs, Ddim,
                      wptr, uptr, wskel, wskeloffset, uskel, uskeloffset, lm, slen, wpart, clevelset, nleaf,
                      2 * nleaf - 2, cdepth);
}

// ---- permutation -----------------------------------------------------------------------

int32_t mxb_permute_rows(const int32_t *d_perm, const int32_t *d_leafofs, const int32_t *d_blockofs,
                         int32_t nleaf, int64_t n, const double *src, double *dst, int64_t row_stride,
                         int64_t col_stride, int32_t nrhs, int32_t direction, int32_t accumulate, void *stream)
{
    if (!d_perm || !d_leafofs || !d_blockofs || !src || !dst || nleaf < 1 || n < 0 || nrhs < 0 ||
        (direction != 0 && direction != 1)) {
        set_error("mxb_permute_rows: bad argument");
        return MXB_ERR_ARG;
    }
    API_CUDA(launch_permute(d_perm, d_leafofs, d_blockofs, nleaf, n, src, dst, row_stride, col_stride, nrhs,
                            direction, accumulate, (cudaStream_t)stream));
    return MXB_OK;
}

static int host_permute(const int32_t *perm, const int32_t *leafofs, const int32_t *blockofs, int32_t nleaf,
                        const double *src, int64_t n, int64_t ld, int32_t nrhs, double *dst, int dir)
{
    if (!perm || !leafofs || !blockofs || !src || !dst || nleaf < 1 || n < 0 || nrhs < 1 || ld < n) {
        set_error("transform: bad argument");
        return MXB_ERR_ARG;
    }
    if (leafofs[0] != 0 || leafofs[nleaf] != n) {
        set_error("transform: leaf offsets must cover [0, n)");
        return MXB_ERR_STRUCTURE;
    }
    size_t blk_ext = 0;
    for (int i = 0; i < nleaf; ++i)
        blk_ext = std::max<size_t>(blk_ext, (size_t)blockofs[i] + (size_t)(leafofs[i + 1] - leafofs[i]) * nrhs);
    for (int64_t t = 0; t < n; ++t)
        if (perm[t] < 0 || perm[t] >= n) {
            set_error("transform: permutation entry out of range");
            return MXB_ERR_STRUCTURE;
        }
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceBuffers *buf = buffers();
    if (!buf) return MXB_ERR_CUDA;
    cudaStream_t s = buf->stream;
    const size_t mat = (size_t)ld * nrhs;
    int32_t *di = nullptr;
    double *dm = nullptr, *db = nullptr;
    const size_t ni = (size_t)n + 2 * ((size_t)nleaf + 1);
    API_CUDA(cudaMalloc(&di, ni * sizeof(int32_t)));
    cudaError_t e = cudaMalloc(&dm, mat * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&db, std::max<size_t>(blk_ext, 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(di, perm, n * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(di + n, leafofs, (nleaf + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(di + n + nleaf + 1, blockofs, nleaf * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        if (dir == 0) {
            e = cudaMemcpyAsync(dm, src, mat * sizeof(double), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess)
                e = launch_permute(di, di + n, di + n + nleaf + 1, nleaf, n, dm, db, 1, ld, nrhs, 0, 0, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dst, db, blk_ext * sizeof(double), cudaMemcpyDeviceToHost, s);
        } else {
            e = cudaMemcpyAsync(db, src, blk_ext * sizeof(double), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dm, dst, mat * sizeof(double), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess)
                e = launch_permute(di, di + n, di + n + nleaf + 1, nleaf, n, db, dm, 1, ld, nrhs, 1, 0, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dst, dm, mat * sizeof(double), cudaMemcpyDeviceToHost, s);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(di);
    cudaFree(dm);
    cudaFree(db);
    if (e != cudaSuccess) {
        set_error(std::string("transform: ") + cudaGetErrorString(e));
        return MXB_ERR_CUDA;
    }
    return MXB_OK;
}

int32_t mxb_transform(const int32_t *perm, const int32_t *leafofs, const int32_t *wptr, int32_t nleaf,
                      const double *W, int64_t n, int64_t ldw, int32_t nrhs, double *TW)
{
    return host_permute(perm, leafofs, wptr, nleaf, W, n, ldw, nrhs, TW, 0);
}

int32_t mxb_untransform(const int32_t *perm, const int32_t *leafofs, const int32_t *uptr, int32_t nleaf,
                        const double *TY, int64_t n, int64_t ldy, int32_t nrhs, double *Y)
{
    return host_permute(perm, leafofs, uptr, nleaf, TY, n, ldy, nrhs, Y, 1);
}

// ---- plan API ------------------------------------------------------------------------------

int32_t mxb_plan_create(const mxb_cds_desc *desc, int32_t precision, mxb_plan **out)
{
    if (!desc || !out) {
        set_error("null argument");
        return MXB_ERR_ARG;
    }
    Plan *p = nullptr;
    int rc = Plan::create(*desc, precision, &p);
    if (rc) return rc;
    *out = p;
    return MXB_OK;
}

int32_t mxb_plan_destroy(mxb_plan *plan)
{
    delete static_cast<Plan *>(plan);
    return MXB_OK;
}

int32_t mxb_plan_evaluate(mxb_plan *plan, const double *dW, double *dY, int32_t nrhs, const int32_t *wptr,
                          const int32_t *uptr, int32_t accumulate, void *stream)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    Plan *p = static_cast<Plan *>(plan);
    return p->run(p->launches_fwd, dW, dY, nrhs, wptr, uptr, accumulate, (cudaStream_t)stream);
}

int32_t mxb_plan_adjoint(mxb_plan *plan, const double *dG, double *dGW, int32_t nrhs, const int32_t *gptr,
                         const int32_t *gwptr, int32_t accumulate, void *stream)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    Plan *p = static_cast<Plan *>(plan);
    return p->run(p->launches_adj, dG, dGW, nrhs, gptr, gwptr, accumulate, (cudaStream_t)stream);
}

int32_t mxb_plan_set_permutation(mxb_plan *plan, const int32_t *perm)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    return static_cast<Plan *>(plan)->set_permutation(perm);
}

int32_t mxb_plan_evaluate_ordered(mxb_plan *plan, const double *dW, int64_t w_rs, int64_t w_cs, double *dY,
                                  int64_t y_rs, int64_t y_cs, int32_t nrhs, int32_t accumulate, void *stream)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    return static_cast<Plan *>(plan)->run_ordered(false, dW, w_rs, w_cs, dY, y_rs, y_cs, nrhs, accumulate,
                                                  (cudaStream_t)stream);
}

int32_t mxb_plan_adjoint_ordered(mxb_plan *plan, const double *dG, int64_t g_rs, int64_t g_cs, double *dGW,
                                 int64_t gw_rs, int64_t gw_cs, int32_t nrhs, int32_t accumulate, void *stream)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    return static_cast<Plan *>(plan)->run_ordered(true, dG, g_rs, g_cs, dGW, gw_rs, gw_cs, nrhs, accumulate,
                                                  (cudaStream_t)stream);
}

int32_t mxb_plan_flops(const mxb_plan *plan, int32_t nrhs, uint64_t *flops)
{
    if (!plan || !flops || nrhs < 0) {
        set_error("bad argument");
        return MXB_ERR_ARG;
    }
    *flops = static_cast<const Plan *>(plan)->flops(nrhs);
    return MXB_OK;
}

int32_t mxb_plan_info(const mxb_plan *plan, uint64_t *device_bytes, int32_t *launches, int32_t *precision)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    const Plan *p = static_cast<const Plan *>(plan);
    if (device_bytes) *device_bytes = p->device_bytes;
    if (launches)
        *launches = p->precision != MXB_PREC_FP64 ? (int32_t)split_bf16_launches(*p)
                                                        : (int32_t)p->launches_fwd.size();
    if (precision) *precision = p->precision;
    return MXB_OK;
}

int32_t mxb_batch_create(mxb_plan *const *plans, int32_t count, mxb_batch **out)
{
    if (!plans || count < 1 || !out) {
        set_error("mxb_batch_create: bad argument");
        return MXB_ERR_ARG;
    }
    std::vector<Plan *> ps(count);
    for (int i = 0; i < count; ++i) {
        ps[i] = static_cast<Plan *>(plans[i]);
        if (!ps[i]) {
            set_error("mxb_batch_create: null plan");
            return MXB_ERR_ARG;
        }
    }
    Batch *b = nullptr;
    int rc = batch_create(ps.data(), count, &b);
    if (rc) return rc;
    *out = reinterpret_cast<mxb_batch *>(static_cast<mxb_batch *>(reinterpret_cast<mxb_batch *>(b)));
    return MXB_OK;
}

int32_t mxb_batch_evaluate(mxb_batch *batch, const double *const *dW, double *const *dY, const int32_t *nrhs,
                           int32_t accumulate, void *stream)
{
    return batch_evaluate(reinterpret_cast<Batch *>(batch), dW, dY, nrhs, accumulate, (cudaStream_t)stream);
}

int32_t mxb_plan_profile(mxb_plan *plan, const double *dW, double *dY, int32_t nrhs, void *stream,
                         mxb_op_profile *out, int32_t cap, int32_t *nops)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    int n = 0;
    const int rc = static_cast<Plan *>(plan)->profile(dW, dY, nrhs, (cudaStream_t)stream, out, cap, &n);
    if (nops) *nops = n;
    return rc;
}

int32_t mxb_batch_profile(mxb_batch *batch, const double *const *dW, double *const *dY, const int32_t *nrhs,
                          void *stream, mxb_op_profile *out, int32_t cap, int32_t *nops)
{
    int n = 0;
    const int rc = batch_profile(reinterpret_cast<Batch *>(batch), dW, dY, nrhs, (cudaStream_t)stream, out, cap, &n);
    if (nops) *nops = n;
    return rc;
}

int32_t mxb_batch_status(mxb_batch *batch) { return batch_status(reinterpret_cast<Batch *>(batch)); }

int32_t mxb_batch_info(const mxb_batch *batch, int32_t *launches, int32_t *widths, int32_t cap, int32_t *nwidths)
{
    if (!batch) {
        set_error("null batch");
        return MXB_ERR_ARG;
    }
    const Batch *b = reinterpret_cast<const Batch *>(batch);
    if (launches) *launches = batch_launches(b);
    const int n = widths && cap > 0 ? batch_tuned_widths(b, widths, cap) : 0;
    if (nwidths) *nwidths = n;
    return MXB_OK;
}

int32_t mxb_batch_set_launch_mode(mxb_batch *batch, int32_t mode)
{
    if (!batch || (mode != MXB_BATCH_LEVEL_LAUNCHES && mode != MXB_BATCH_ONE_LAUNCH)) {
        set_error("mxb_batch_set_launch_mode: null batch or unknown mode");
        return MXB_ERR_ARG;
    }
    return batch_set_one_launch(reinterpret_cast<Batch *>(batch), mode == MXB_BATCH_ONE_LAUNCH);
}

int32_t mxb_batch_destroy(mxb_batch *batch)
{
    batch_destroy(reinterpret_cast<Batch *>(batch));
    return MXB_OK;
}

int32_t mxb_plan_set_test_hooks(mxb_plan *plan, int32_t flags, int64_t wait_cycles)
{
    if (!plan || wait_cycles < 0) {
        set_error("bad argument");
        return MXB_ERR_ARG;
    }
    Plan *p = static_cast<Plan *>(plan);
    if (p->precision == MXB_PREC_FP64 && flags) {
        set_error("test hooks apply to split-BF16 plans");
        return MXB_ERR_UNSUPPORTED;
    }
    p->debug_flags = flags;
    p->debug_wait_cycles = wait_cycles;
    p->clear_graphs();  // hooks are baked into captured graphs
    return MXB_OK;
}

int32_t mxb_plan_status(mxb_plan *plan)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    Plan *p = static_cast<Plan *>(plan);
    API_CUDA(cudaDeviceSynchronize());
    return split_bf16_status(*p);
}

int32_t mxb_plan_read_workspaces(mxb_plan *plan, int32_t nrhs, const int32_t *wskeloffset, double *wskel,
                                 const int32_t *uskeloffset, double *uskel)
{
    if (!plan) {
        set_error("null plan");
        return MXB_ERR_ARG;
    }
    return static_cast<Plan *>(plan)->read_workspaces(nrhs, wskeloffset, wskel, uskeloffset, uskel);
}

}  // extern "C"
