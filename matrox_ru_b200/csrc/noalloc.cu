// Evaluation entry point for callers that are not allowed to allocate device memory.
//
// Some hosts own every byte of device memory: a framework that hands the GPU to its own
// pooling allocator (a library cudaMalloc would sit outside the pool, fragment it or push
// the process over a fixed memory budget), or a steady-state pipeline that must never call
// cudaMalloc / cudaFree because those calls can synchronise the whole device.  Such callers
// keep the CDS, W and Y in memory they allocated themselves and need an evaluation that
// allocates nothing.  mxb_evaluate_noalloc is that entry point: the same FP64 grouped-GEMM
// kernel as mxb_plan_evaluate, with its task lists, per-leaf offsets and skeleton
// workspaces placed in one statically sized device array that lives in this file.
#include <mutex>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"
#include "plan.h"

namespace mxb {
namespace {

// Shared by every call on a device; each GPU that loads the library holds it until exit.
constexpr size_t kScratchBytes = MXB_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// In host code g_noalloc_scratch names a host-side stand-in, not device memory: the device
// address comes from cudaGetSymbolAddress, looked up once per device with that device
// current (the first call on each device does this).
std::mutex g_mu;
void *g_scratch_addr[128];

int scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("mxb_evaluate_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return MXB_ERR_CUDA;
    }
    if (dev < 0 || dev >= 128) {
        set_error("mxb_evaluate_noalloc: device index out of range");
        return MXB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("mxb_evaluate_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return MXB_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The kernels read D, B, VT and W and write Y directly, so each must be memory of the current
// device (or managed memory).  A host pointer here -- e.g. a descriptor built for
// mxb_plan_create, whose pools are host arrays -- is rejected before anything is launched.
int check_device_pointer(const void *ptr, const char *what)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    cudaPointerAttributes a{};
    if (e == cudaSuccess) e = cudaPointerGetAttributes(&a, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("mxb_evaluate_noalloc: ") + what + ": cudaPointerGetAttributes: " +
                  cudaGetErrorString(e));
        return MXB_ERR_ARG;
    }
    const bool ok = a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
    if (!ok) {
        set_error(std::string("mxb_evaluate_noalloc: ") + what + " must be device memory of the current device "
                  "(this entry point reads the CDS pools, W and Y in place)");
        return MXB_ERR_ARG;
    }
    return MXB_OK;
}

}  // namespace
}  // namespace mxb

using namespace mxb;

extern "C" int32_t mxb_evaluate_noalloc(const mxb_cds_desc *desc, const double *dW, double *dY, int32_t nrhs,
                                        int32_t accumulate, void *stream)
{
    if (!desc || !dW || !dY || nrhs < 1) {
        set_error("mxb_evaluate_noalloc: null argument or nrhs < 1");
        return MXB_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // The task lists are staged from host vectors that this call frees on return; a capturing
    // stream would record copies that read them after they are gone.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(s, &cap);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("mxb_evaluate_noalloc: cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
        return MXB_ERR_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("mxb_evaluate_noalloc: the stream is capturing; this entry point copies each call's task lists "
                  "from temporary host memory and is called outside stream capture");
        return MXB_ERR_UNSUPPORTED;
    }
    int rc = MXB_OK;
    if (desc->D_len && (rc = check_device_pointer(desc->D, "desc->D"))) return rc;
    if (desc->B_len && (rc = check_device_pointer(desc->B, "desc->B"))) return rc;
    if (desc->VT_len && (rc = check_device_pointer(desc->VT, "desc->VT"))) return rc;
    if ((rc = check_device_pointer(dW, "dW"))) return rc;
    if ((rc = check_device_pointer(dY, "dY"))) return rc;
    // host-side structure and task lists only: this Plan never touches device memory
    Plan p;
    rc = p.validate(*desc);
    if (rc) return rc;
    p.build_tasks(row_tile_for(MXB_PREC_FP64));

    const size_t tasks_b = p.tasks.size() * sizeof(Task);
    const size_t items_b = p.items.size() * sizeof(Item);
    const size_t ofs_b = (size_t)p.nleaf * sizeof(int32_t);
    const size_t skel_b = (size_t)p.skel_total * (size_t)nrhs * sizeof(double);
    const size_t off_items = align256(tasks_b);
    const size_t off_ofs = off_items + align256(items_b);
    const size_t off_w = off_ofs + align256(ofs_b);
    const size_t off_u = off_w + align256(skel_b);
    const size_t need = off_u + skel_b;
    if (need > kScratchBytes) {
        set_error("mxb_evaluate_noalloc: this CDS with nrhs = " + std::to_string(nrhs) + " needs " +
                  std::to_string(need) + " bytes of scratch (task lists + skeleton workspaces), more than the " +
                  std::to_string(kScratchBytes) + " bytes of MXB_NOALLOC_SCRATCH_BYTES; use mxb_plan_evaluate "
                  "or fewer right-hand sides per call");
        return MXB_ERR_UNSUPPORTED;
    }
    std::vector<int32_t> ofs(p.nleaf);
    for (int i = 0; i < p.nleaf; ++i) {
        const int64_t o = p.leaf_row[i] * (int64_t)nrhs;
        if (o > INT32_MAX) {
            set_error("mxb_evaluate_noalloc: packed leaf offsets overflow int32");
            return MXB_ERR_ARG;
        }
        ofs[i] = (int32_t)o;
    }
    void *base = nullptr;
    rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char *b = static_cast<unsigned char *>(base);
    // pageable sources: each copy has consumed its host buffer when the call returns (the
    // copies may therefore block the host until the stream reaches them)
    cudaError_t e = cudaSuccess;
    if (tasks_b) e = cudaMemcpyAsync(b, p.tasks.data(), tasks_b, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && items_b) e = cudaMemcpyAsync(b + off_items, p.items.data(), items_b, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + off_ofs, ofs.data(), ofs_b, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        set_error(std::string("mxb_evaluate_noalloc: staging task lists: ") + cudaGetErrorString(e));
        return MXB_ERR_CUDA;
    }
    Operands ops{};
    ops.pool[0] = desc->D;
    ops.pool[1] = desc->B;
    ops.pool[2] = desc->VT;
    ops.W = dW;
    ops.Y = dY;
    ops.wskel = reinterpret_cast<double *>(b + off_w);
    ops.uskel = reinterpret_cast<double *>(b + off_u);
    ops.wofs = reinterpret_cast<const int32_t *>(b + off_ofs);
    ops.yofs = ops.wofs;
    ops.nrhs = nrhs;
    ops.beta_arg = accumulate ? 1 : 0;
    const Task *dtasks = reinterpret_cast<const Task *>(b);
    const Item *ditems = reinterpret_cast<const Item *>(b + off_items);
    for (const Launch &l : p.launches_fwd) {
        e = launch_gemm_f64(dtasks + l.task0, ditems, l.ntasks, ops, s);
        if (e != cudaSuccess) {
            set_error(std::string("mxb_evaluate_noalloc: launch: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
    }
    return MXB_OK;
}
