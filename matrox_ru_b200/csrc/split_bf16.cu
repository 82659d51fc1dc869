// Split-BF16 evaluation path on the 5th-generation tensor cores (tcgen05).
//
// Precision scheme (per north-star: BF16 tensor-core products with split operands, FP32
// accumulation, FP32-accurate transfers, FP64 final Y):
//   near D_xy W_y and far B_xy wskel_y : both operands split into bf16 hi + mid, three
//        products hi*hi + hi*mid + mid*hi ("bf16x3"), FP32 accumulation in TMEM.  Splitting
//        only W leaves the CDS operand at 8 bits (~2e-3 relative error); splitting both
//        gives ~5e-6.
//   transfers (leaf / internal projections up and down): hi + mid + lo (24 bits), six
//        products ("bf16x6"), which matches an FP32 SGEMM's error (~3e-7).
//   Y: FP64, accumulated from the FP32 tile in the epilogue.
//
// Data layout: every operand lives in HBM already in the shared-memory tile format
// (128 rows x 64 K bf16, K-major, 128-byte swizzle; parts of one tile contiguous), so each
// pipeline stage is filled by a few 1-D bulk copies (cp.async.bulk) on an mbarrier -- no
// tensor maps, no per-element address math in the main loop.  The CDS operands (D, B, the
// projections and their transposes) are tiled once when the plan is created; W and the
// skeleton vectors are tiled per evaluation by split kernels (HBM-bound passes).
//
// GEMM kernel: one CTA per (task row tile, 128|256 right-hand sides), 10 warps:
//   warp 8 lane 0 : producer -- bulk copies of the A and B part tiles of each K step
//   warp 9 lane 0 : MMA issuer -- tcgen05.mma M=128, N=BN, K=16, 3 or 6 per 16-K slice,
//                   one fresh TMEM accumulator (of two) per 64-deep K tile
//   warps 0-7     : drain every K tile's accumulator into round-to-nearest FP32 registers
//                   (tcgen05.ld), then store rows with coalesced writes
// Every wait is bounded (tc::WAIT_CYCLES); a CTA that times out raises MXB_ERR_TIMEOUT in
// the plan's error word, drains its own copies and MMAs, frees its TMEM and exits.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"
#include "plan.h"
#include "tc_common.cuh"

namespace mxb {

int row_tile_for(int precision) { return precision != MXB_PREC_FP64 ? 128 : 64; }

namespace {

using tc::TILE_BYTES;

struct TcItem {
    uint64_t a_off;   // byte offset of A's tile (0, 0) in the launch's A pool
    int64_t b_base;   // K-tile base of the B operand's node / leaf in the B buffer
    int32_t KT;       // K tiles of this item
    int32_t pad;
};

struct SplitJob {     // one leaf block of W or one skeleton block -> tiled parts
    int64_t src_row;  // leaf index (W) or skeleton row offset
    int64_t dst_kt;   // K-tile base in the destination buffer
    int32_t ld, K, KT, pad;
};

struct PoolJob {      // one CDS matrix -> tiled parts (plan creation)
    uint64_t src_off;  // element offset in the FP64 pool
    uint64_t dst_off;  // byte offset of tile (0, 0)
    int32_t src_pool, ld, R, K, RT, KT, trans, parts;
};

// Output of a tensor-core task.
enum OutKind : int16_t {
    OUT_Y = 0,      // FP64 Y block (leaf-blocked, caller's offsets)
    OUT_F32 = 1,    // FP32 skeleton block (a far result the down launch adds to)
    OUT_TILES = 2,  // skeleton block written as 3-part bf16 operand tiles for the next launches
};

struct TcTask {
    int64_t c_row;   // leaf index (OUT_Y) or skeleton row offset (FP32 block)
    int64_t out_kt;  // K-tile base of the node in the tile buffer (OUT_TILES)
    int32_t ldc;
    int32_t M;       // rows of the whole output block
    int32_t m0;      // first row of this task's 128-row tile
    int32_t item0;
    int32_t nitem;
    int16_t out_kind;
    int16_t beta;    // 0 overwrite, 1 accumulate (OUT_TILES: add the FP32 block), 2 launch arg
};

struct TcArgs {
    const uint8_t *a_pool;
    const uint8_t *b_pool;
    uint8_t *t_pool;  // tile buffer of OUT_TILES tasks
    double *Y;
    const int32_t *yofs;
    float *skel;      // FP32 skeleton blocks (written by OUT_F32, added by OUT_TILES with beta)
    int *err;
    int NT;         // 128-column tiles per node in the B buffers (even)
    int nrhs;
    int beta_arg;
    long long wait_cycles;  // limit of every wait in the kernel
    int stall_test;         // test hook: CTA 0 withholds its first stage, so a wait runs out
};

// ---------------------------------------------------------------------------------------
// tiling kernels
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ void store_parts(uint8_t *tile0, int parts, int r, int c, const __nv_bfloat16 (&h)[8],
                                            const __nv_bfloat16 (&m)[8], const __nv_bfloat16 (&l)[8])
{
    const uint32_t o = tc::swizzled_offset(r, c * 8);
    uint4 vh, vm, vl;
    memcpy(&vh, h, 16);
    memcpy(&vm, m, 16);
    memcpy(&vl, l, 16);
    *reinterpret_cast<uint4 *>(tile0 + o) = vh;
    *reinterpret_cast<uint4 *>(tile0 + TILE_BYTES + o) = vm;
    if (parts > 2) *reinterpret_cast<uint4 *>(tile0 + 2 * TILE_BYTES + o) = vl;
}

// CDS matrix -> tiled parts.  op(A)(r, k) = trans ? src[k + r ld] : src[r + k ld].
__global__ void __launch_bounds__(256) tile_pool_kernel(const PoolJob *__restrict__ jobs, const double *p0,
                                                        const double *p1, const double *p2, uint8_t *dst)
{
    const PoolJob j = jobs[blockIdx.x];
    const int kt = blockIdx.y, rt = blockIdx.z;
    if (kt >= j.KT || rt >= j.RT) return;
    const double *src = (j.src_pool == 0 ? p0 : (j.src_pool == 1 ? p1 : p2)) + j.src_off;
    uint8_t *tile0 = dst + j.dst_off + ((size_t)rt * j.KT + kt) * (size_t)j.parts * TILE_BYTES;
    for (int i = 0; i < 4; ++i) {
        const int idx = threadIdx.x + i * 256;
        const int r = j.trans ? idx / 8 : idx % 128;
        const int c = j.trans ? idx % 8 : idx / 128;
        const int gr = rt * 128 + r;
        __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int gk = kt * 64 + c * 8 + e;
            double x = 0.0;
            if (gr < j.R && gk < j.K) x = j.trans ? src[gk + (size_t)gr * j.ld] : src[gr + (size_t)gk * j.ld];
            tc::split3(x, h[e], m[e], l[e]);
        }
        store_parts(tile0, j.parts, r, c, h, m, l);
    }
}

// W (FP64, leaf-blocked) or a skeleton block (FP32) -> B-operand tiles with 3 parts.
// B(n, k) = src[k + n ld]; rows n >= nrhs and k >= K are zero.
template <typename T>
__global__ void __launch_bounds__(256) split_b_kernel(const SplitJob *__restrict__ jobs, const T *__restrict__ base,
                                                      const int32_t *__restrict__ ofs, int nrhs, int NT,
                                                      uint8_t *__restrict__ dst)
{
    const SplitJob j = jobs[blockIdx.x];
    const int kt = blockIdx.y, nt = blockIdx.z;
    if (kt >= j.KT) return;
    const T *src = base + (ofs ? (int64_t)ofs[j.src_row] : j.src_row * (int64_t)nrhs);
    uint8_t *tile0 = dst + ((size_t)j.dst_kt * NT + (size_t)nt * j.KT + kt) * 3 * (size_t)TILE_BYTES;
    for (int i = 0; i < 4; ++i) {
        const int idx = threadIdx.x + i * 256;
        const int c = idx % 8, r = idx / 8;
        const int n = nt * 128 + r;
        __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int k = kt * 64 + c * 8 + e;
            T x = T(0);
            if (n < nrhs && k < j.K) x = src[k + (size_t)n * j.ld];
            tc::split3(x, h[e], m[e], l[e]);
        }
        store_parts(tile0, 3, r, c, h, m, l);
    }
}

// ---------------------------------------------------------------------------------------
// tcgen05 grouped GEMM
// ---------------------------------------------------------------------------------------

// 8 x 8 transpose inside each group of 8 lanes: lane 8g + i ends with x[j] = the value lane
// 8g + j held in x[i] (three butterfly stages of block swaps).
__device__ __forceinline__ void transpose8(float (&x)[8], int lane)
{
#pragma unroll
    for (int s = 1; s < 8; s <<= 1) {
        const bool up = (lane & s) != 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if ((i & s) == 0) {
                const float send = up ? x[i] : x[i + s];
                const float recv = __shfl_xor_sync(0xffffffffu, send, s);
                if (up) x[i] = recv;
                else x[i + s] = recv;
            }
        }
    }
}

template <int P, int BN>
struct TcCfg {
    static constexpr int STAGES = 2;
    static constexpr int HALVES = BN / 128;
    static constexpr int A_BYTES = P * TILE_BYTES;
    static constexpr int B_BYTES = HALVES * P * TILE_BYTES;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
    static constexpr int NPROD = P == 2 ? 3 : 6;
    static constexpr int EPI_WARPS = 8;          // two per TMEM lane quarter, one per column half
    static constexpr int THREADS = (EPI_WARPS + 2) * 32;
    static constexpr int COLS = BN / 2;          // accumulator columns per epilogue thread
    static constexpr int TMEM_COLS = 2 * BN;     // two accumulator buffers
};

// Tensor-core FP32 accumulation is not round-to-nearest: its error grows with the number of
// MMAs chained into one accumulator (measured ~4e-5 relative after 8192-deep chains).  So
// each 64-deep K tile gets a fresh TMEM accumulator (two buffers, alternating), and the
// epilogue warps add every tile's partial sums into per-thread FP32 registers with ordinary
// round-to-nearest adds while the tensor core already works on the next tile.
//
// Persistent: one CTA per SM walks the work units u = blockIdx.x, blockIdx.x + gridDim.x, ...
// (unit = task x column tile).  The three roles walk the same sequence, so one global K-tile
// counter drives every stage and accumulator phase; TMEM and the barriers are set up once,
// and the epilogue of one unit overlaps the MMAs of the next.
template <int P, int BN>
__global__ void __launch_bounds__(TcCfg<P, BN>::THREADS, 1)
tc_gemm_kernel(const TcTask *__restrict__ tasks, const TcItem *__restrict__ items, int nunits, TcArgs args)
{
    using C = TcCfg<P, BN>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    uint64_t *empty = full + C::STAGES;
    uint64_t *accf = empty + C::STAGES;  // accumulator buffer b holds a finished K tile
    uint64_t *acce = accf + 2;           // accumulator buffer b has been drained
    uint64_t *doneb = acce + 2;          // every MMA this CTA issued has completed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(doneb + 1);
    volatile int *abort_word = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncol = (args.nrhs + BN - 1) / BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accf[b], 1);
            tc::mbar_init(&acce[b], C::EPI_WARPS);
        }
        tc::mbar_init(doneb, 1);
        *abort_word = 0;
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == C::EPI_WARPS) {
        if (lane == 0) {
            // ---------------- producer ----------------
            uint32_t g = 0;  // global K-tile counter of this CTA
            uint32_t filled[C::STAGES];  // rounds filled per stage (drained before exit)
#pragma unroll
            for (int s = 0; s < C::STAGES; ++s) filled[s] = 0;
            for (int u = blockIdx.x; u < nunits && !*abort_word; u += gridDim.x) {
                const TcTask t = tasks[u / ncol];
                const int col = u % ncol;
                const TcItem *ti = items + t.item0;
                const int mt = t.m0 / 128;
                for (int q = 0; q < t.nitem && !*abort_word; ++q) {
                    const TcItem it = ti[q];
                    for (int kt = 0; kt < it.KT; ++kt, ++g) {
                        const int s = g % C::STAGES;
                        const uint32_t round = g / C::STAGES;
                        if (!tc::mbar_wait(&empty[s], (round & 1) ^ 1, abort_word, args.wait_cycles)) {
                            *abort_word = 1;
                            break;
                        }
                        if (args.stall_test && blockIdx.x == 0 && g == 0) continue;  // never filled
                        uint8_t *sa = smem + s * C::STAGE;
                        uint8_t *sb = sa + C::A_BYTES;
                        tc::mbar_expect_tx(&full[s], C::STAGE);
                        const uint8_t *ga =
                            args.a_pool + it.a_off + ((size_t)mt * it.KT + kt) * (size_t)P * TILE_BYTES;
                        tc::bulk_g2s(sa, ga, C::A_BYTES, &full[s]);
#pragma unroll
                        for (int hh = 0; hh < C::HALVES; ++hh) {
                            const size_t nt = (size_t)col * C::HALVES + hh;
                            const uint8_t *gb = args.b_pool +
                                                ((size_t)it.b_base * args.NT + nt * it.KT + kt) * 3 * (size_t)TILE_BYTES;
#pragma unroll
                            for (int p = 0; p < P; ++p)
                                tc::bulk_g2s(sb + (p * C::HALVES + hh) * TILE_BYTES, gb + (size_t)p * TILE_BYTES,
                                             TILE_BYTES, &full[s]);
                        }
                        filled[s] = round + 1;
                    }
                }
            }
            // every stage this thread filled must have landed before the CTA may exit
#pragma unroll
            for (int s = 0; s < C::STAGES; ++s) {
                if (!filled[s]) continue;
                volatile int never = 0;
                tc::mbar_wait(&full[s], (filled[s] - 1) & 1, &never, args.wait_cycles);
            }
        }
    } else if (warp == C::EPI_WARPS + 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, BN);
            constexpr int PA[6] = {0, 0, 1, 0, 1, 2};
            constexpr int PB[6] = {0, 1, 0, 2, 1, 0};
            uint32_t g = 0;
            bool any = false;
            for (int u = blockIdx.x; u < nunits && !*abort_word; u += gridDim.x) {
                const TcTask t = tasks[u / ncol];
                int ktiles = 0;
                for (int q = 0; q < t.nitem; ++q) ktiles += items[t.item0 + q].KT;
                for (int i = 0; i < ktiles; ++i, ++g) {
                    const int s = g % C::STAGES;
                    const uint32_t round = g / C::STAGES;
                    const int b = g & 1;
                    const uint32_t use = g >> 1;
                    if (!tc::mbar_wait(&acce[b], (use & 1) ^ 1, abort_word, args.wait_cycles) ||
                        !tc::mbar_wait(&full[s], round & 1, abort_word, args.wait_cycles)) {
                        *abort_word = 1;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t sa = tc::smem_u32(smem + s * C::STAGE);
                    const uint32_t sb = sa + C::A_BYTES;
                    const uint32_t dst = tmem + (uint32_t)(b * BN);
                    uint32_t accum = 0;
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks) {
#pragma unroll
                        for (int j = 0; j < C::NPROD; ++j) {
                            const uint64_t ad = tc::smem_desc_sw128(sa + PA[j] * TILE_BYTES + ks * 32);
                            const uint64_t bd = tc::smem_desc_sw128(sb + PB[j] * C::HALVES * TILE_BYTES + ks * 32);
                            tc::mma_bf16(dst, ad, bd, IDESC, accum);
                            accum = 1;
                        }
                    }
                    tc::mma_commit(&empty[s]);
                    tc::mma_commit(&accf[b]);
                    any = true;
                }
            }
            if (any) tc::mma_commit(doneb);
            else tc::mbar_expect_tx(doneb, 0);  // nothing issued: complete the barrier's phase now
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        uint32_t g = 0;
        for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
            const TcTask t = tasks[u / ncol];
            const int col = u % ncol;
            int ktiles = 0;
            for (int q = 0; q < t.nitem; ++q) ktiles += items[t.item0 + q].KT;
            float acc[C::COLS];
#pragma unroll
            for (int e = 0; e < C::COLS; ++e) acc[e] = 0.f;
            bool ok = !*abort_word;
            for (int i = 0; i < ktiles && ok; ++i, ++g) {
                const int b = g & 1;
                const uint32_t use = g >> 1;
                if (!tc::mbar_wait(&accf[b], use & 1, abort_word, args.wait_cycles)) {
                    *abort_word = 1;
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
#pragma unroll
                for (int c0 = 0; c0 < C::COLS; c0 += 32) {
                    float v[32];
                    tc::tmem_ld32(tmem + lane_base + (uint32_t)(b * BN + half * C::COLS + c0), v);
#pragma unroll
                    for (int e = 0; e < 32; ++e) acc[c0 + e] += v[e];
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tc::smem_u32(&acce[b])) : "memory");
            }
            if (!ok || *abort_word) break;
            const int r = t.m0 + quarter * 32 + lane;
            const int beta = t.beta == 2 ? args.beta_arg : t.beta;
            const int col0 = col * BN + half * C::COLS;
            // accumulating outputs: all old values of a 16-column chunk are loaded before any
            // store, so the loads overlap instead of waiting on each other
            if (t.out_kind == OUT_Y) {
                if (r < t.M) {
                    double *Yb = args.Y + args.yofs[t.c_row] + r;
#pragma unroll
                    for (int c0 = 0; c0 < C::COLS; c0 += 16) {
                        double old[16];
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int cc = col0 + c0 + e;
                            old[e] = (beta && cc < args.nrhs) ? Yb[(size_t)cc * t.ldc] : 0.0;
                        }
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int cc = col0 + c0 + e;
                            if (cc < args.nrhs) Yb[(size_t)cc * t.ldc] = old[e] + (double)acc[c0 + e];
                        }
                    }
                }
            } else if (t.out_kind == OUT_F32) {
                if (r < t.M) {
                    float *Sb = args.skel + t.c_row * (int64_t)args.nrhs + r;
#pragma unroll
                    for (int e = 0; e < C::COLS; ++e) {
                        const int cc = col0 + e;
                        if (cc < args.nrhs) Sb[(size_t)cc * t.ldc] = acc[e];
                    }
                }
            } else {
                // OUT_TILES: (optionally) add the FP32 far result, then write this row's values
                // as 3-part bf16 operand tiles.  The lane holds one K index; a transpose in
                // groups of 8 lanes gives it 8 consecutive K of one column: one 16-byte chunk
                // per part.  Rows past M carry zeros (A is zero-padded); rows past the node's
                // K tiles are not written.
                if (beta && r < t.M) {
                    const float *Sb = args.skel + t.c_row * (int64_t)args.nrhs + r;
#pragma unroll
                    for (int c0 = 0; c0 < C::COLS; c0 += 16) {
                        float old[16];
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int cc = col0 + c0 + e;
                            old[e] = cc < args.nrhs ? Sb[(size_t)cc * t.ldc] : 0.f;
                        }
#pragma unroll
                        for (int e = 0; e < 16; ++e) acc[c0 + e] += old[e];
                    }
                }
                const int KTv = (t.M + 63) / 64;
                const int k0 = t.m0 + quarter * 32 + (lane & ~7);
                const bool k_ok = k0 < KTv * 64;
                const int kt = k0 >> 6;
                const uint32_t kin = (uint32_t)(k0 & 63);
#pragma unroll
                for (int g8 = 0; g8 < C::COLS / 8; ++g8) {
                    float x[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) x[j] = acc[8 * g8 + j];
                    transpose8(x, lane);
                    const int n = col0 + 8 * g8 + (lane & 7);
                    __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) tc::split3(x[j], h[j], m[j], l[j]);
                    if (k_ok) {
                        uint8_t *tile0 = args.t_pool +
                                         ((size_t)t.out_kt * args.NT + (size_t)(n >> 7) * KTv + kt) * 3 * (size_t)TILE_BYTES;
                        store_parts(tile0, 3, n & 127, (int)(kin >> 3), h, m, l);
                    }
                }
            }
        }
    }
    __syncwarp();
    __syncthreads();
    // all MMAs must be complete before TMEM is released (bounded, also after an abort)
    if (threadIdx.x == 0) {
        volatile int never = 0;
        if (!tc::mbar_wait(doneb, 0, &never, args.wait_cycles)) *abort_word = 1;
    }
    __syncthreads();
    if (*abort_word && threadIdx.x == 0) atomicExch(args.err, MXB_ERR_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, C::TMEM_COLS);
}

int g_sm_count[128];

template <int P, int BN>
cudaError_t launch_tc(const TcTask *tasks, const TcItem *items, int ntasks, const TcArgs &a, cudaStream_t s)
{
    if (ntasks <= 0) return cudaSuccess;
    using C = TcCfg<P, BN>;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    if (!g_sm_count[dev]) {
        e = cudaDeviceGetAttribute(&g_sm_count[dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    static bool configured[128];
    if (!configured[dev]) {
        e = cudaFuncSetAttribute(tc_gemm_kernel<P, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    const int nunits = ntasks * ((a.nrhs + BN - 1) / BN);
    const int grid = std::min(nunits, g_sm_count[dev]);
    tc_gemm_kernel<P, BN><<<grid, C::THREADS, C::SMEM, s>>>(tasks, items, nunits, a);
    return cudaGetLastError();
}

enum OpKind { OP_SPLIT_W, OP_SPLIT_WSKEL, OP_SPLIT_USKEL, OP_TC2, OP_TC3 };
enum APool { POOL_NEAR, POOL_FAR, POOL_VU3, POOL_VD3, NPOOL };
enum BBuf { BUF_W, BUF_WSKEL, BUF_USKEL };

struct Op {
    int kind, first, count, max_kt;
    int a_pool, b_buf, t_buf;  // A pool, B buffer, tile buffer written by OUT_TILES tasks
};

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

struct SplitBF16 {
    uint8_t *pool[NPOOL] = {};
    size_t pool_bytes[NPOOL] = {};
    TcTask *dTasks = nullptr;
    TcItem *dItems = nullptr;
    SplitJob *dJobs = nullptr;
    int *dErr = nullptr;
    std::vector<Op> ops;
    std::vector<TcTask> tasks;
    std::vector<TcItem> items;
    std::vector<SplitJob> jobs;
    std::vector<int64_t> leaf_kt, node_kt;  // K-tile bases
    int64_t leaf_kt_total = 0, node_kt_total = 0;
    int nt_cap = 0, nrhs_cap = 0;
    uint8_t *Wt = nullptr, *wT = nullptr, *uT = nullptr;
    float *u32 = nullptr;  // FP32 far results awaiting the down launch
};

int Plan::setup_split_bf16(const mxb_cds_desc &)
{
    SplitBF16 *S = new SplitBF16();
    bf16 = S;
    // bf16x3 (2 stored parts) or bf16x6 (3 parts) for the near field and the far couplings
    const int near_parts = precision == MXB_PREC_SPLIT_BF16_X6 ? 3 : 2;
    const int far_parts = precision == MXB_PREC_SPLIT_BF16 ? 2 : 3;
    auto KT = [](int64_t k) { return (int32_t)ceil_div(std::max<int64_t>(k, 0), 64); };
    auto RT = [](int64_t r) { return (int32_t)ceil_div(std::max<int64_t>(r, 0), 128); };
    auto projects = [&](int v) { return v != root && slen[v] > 0; };

    // ---- K-tile bases of the B operands (per-evaluation buffers) ----
    S->leaf_kt.resize(nleaf);
    for (int i = 0; i < nleaf; ++i) {
        S->leaf_kt[i] = S->leaf_kt_total;
        S->leaf_kt_total += KT(Ddim[i]);
    }
    S->node_kt.assign(numnodes, 0);
    for (int v : bfs) {
        S->node_kt[v] = S->node_kt_total;
        S->node_kt_total += KT(slen[v]);
    }

    // ---- CDS pools: tiling jobs ----
    std::vector<PoolJob> pj[NPOOL];
    auto add_pool = [&](int pool, int src_pool, uint64_t src_off, int ld, int R, int K, int trans, int parts) {
        PoolJob j{};
        j.src_pool = src_pool;
        j.src_off = src_off;
        j.ld = ld;
        j.R = R;
        j.K = K;
        j.RT = RT(R);
        j.KT = KT(K);
        j.trans = trans;
        j.parts = parts;
        j.dst_off = S->pool_bytes[pool];
        S->pool_bytes[pool] += (size_t)j.RT * j.KT * parts * TILE_BYTES;
        pj[pool].push_back(j);
        return j.dst_off;
    };
    std::vector<uint64_t> near_a(near_x.size()), far_a(far_x.size());
    for (size_t k = 0; k < near_x.size(); ++k)
        near_a[k] = add_pool(POOL_NEAR, 0, near_off[k], Ddim[near_x[k]], Ddim[near_x[k]], Ddim[near_y[k]], 0, near_parts);
    for (size_t k = 0; k < far_x.size(); ++k)
        far_a[k] = add_pool(POOL_FAR, 1, far_off[k], slen[far_x[k]], slen[far_x[k]], slen[far_y[k]], 0, far_parts);
    std::vector<uint64_t> up_a(numnodes), up_b(numnodes), down_a(numnodes);
    for (int v = 0; v < numnodes; ++v) {
        if (!projects(v)) continue;
        const int s = slen[v];
        if (lch[v] == -1) {
            up_a[v] = add_pool(POOL_VU3, 2, (uint64_t)VTptr[v], s, s, Ddim[lm[v]], 0, 3);
            down_a[v] = add_pool(POOL_VD3, 2, (uint64_t)VTptr[v], s, Ddim[lm[v]], s, 1, 3);  // leaf down: P_v^T
        } else {
            const int l = lch[v], r = rch[v];
            up_a[v] = add_pool(POOL_VU3, 2, (uint64_t)VTptr[v], s, s, slen[l], 0, 3);
            up_b[v] = add_pool(POOL_VU3, 2, (uint64_t)VTptr[v] + (uint64_t)s * slen[l], s, s, slen[r], 0, 3);
        }
    }
    // down slices: child c of projecting parent p: op(A) = P_p[:, part of c]^T (s_c x s_p)
    std::vector<uint64_t> down_child(numnodes);
    for (int c = 0; c < numnodes; ++c) {
        const int p = parent[c];
        if (p < 0 || !projects(p) || !projects(c)) continue;
        const uint64_t off = (uint64_t)VTptr[p] + (c == rch[p] ? (uint64_t)slen[p] * slen[lch[p]] : 0);
        down_child[c] = add_pool(POOL_VD3, 2, off, slen[p], slen[c], slen[p], 1, 3);
    }
    for (int pidx = 0; pidx < NPOOL; ++pidx) {
        int rc = alloc((void **)&S->pool[pidx], std::max<size_t>(S->pool_bytes[pidx], 16));
        if (rc) return rc;
        if (pj[pidx].empty()) continue;
        PoolJob *dj = nullptr;
        rc = alloc((void **)&dj, pj[pidx].size() * sizeof(PoolJob));
        if (rc) return rc;
        cudaError_t e = cudaMemcpy(dj, pj[pidx].data(), pj[pidx].size() * sizeof(PoolJob), cudaMemcpyHostToDevice);
        int maxkt = 1, maxrt = 1;
        for (auto &j : pj[pidx]) {
            maxkt = std::max(maxkt, j.KT);
            maxrt = std::max(maxrt, j.RT);
        }
        if (e == cudaSuccess) {
            tile_pool_kernel<<<dim3((unsigned)pj[pidx].size(), maxkt, maxrt), 256>>>(dj, dD, dB, dVT, S->pool[pidx]);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error(std::string("tiling the CDS for the split-BF16 path: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
    }

    // ---- task lists and op sequence (forward) ----
    int maxh = 0, maxd = 0;
    for (int v = 0; v < numnodes; ++v) {
        maxh = std::max(maxh, height[v]);
        maxd = std::max(maxd, depth[v]);
    }
    auto begin_op = [&](int kind, int a_pool, int b_buf, int t_buf) {
        Op o{};
        o.kind = kind;
        o.a_pool = a_pool;
        o.b_buf = b_buf;
        o.t_buf = t_buf;
        o.first = (kind <= OP_SPLIT_USKEL) ? (int)S->jobs.size() : (int)S->tasks.size();
        S->ops.push_back(o);
    };
    auto end_op = [&]() {
        Op &o = S->ops.back();
        if (o.kind >= OP_TC2) {
            // longest tasks first: balances the persistent kernel's static round-robin
            auto cost = [&](const TcTask &t) {
                int k = 0;
                for (int q = 0; q < t.nitem; ++q) k += S->items[t.item0 + q].KT;
                return k;
            };
            std::stable_sort(S->tasks.begin() + o.first, S->tasks.end(),
                             [&](const TcTask &a, const TcTask &b) { return cost(a) > cost(b); });
        }
        o.count = ((o.kind <= OP_SPLIT_USKEL) ? (int)S->jobs.size() : (int)S->tasks.size()) - o.first;
        o.max_kt = 1;
        if (o.kind <= OP_SPLIT_USKEL)
            for (int j = o.first; j < o.first + o.count; ++j) o.max_kt = std::max(o.max_kt, S->jobs[j].KT);
        if (o.count == 0) S->ops.pop_back();
    };
    auto add_tasks = [&](int16_t out_kind, int64_t c_row, int64_t out_kt, int ldc, int M, int item0,
                         int16_t beta) {
        for (int m0 = 0; m0 < M; m0 += 128) {
            TcTask t{};
            t.c_row = c_row;
            t.out_kt = out_kt;
            t.ldc = ldc;
            t.M = M;
            t.m0 = m0;
            t.item0 = item0;
            t.nitem = (int)S->items.size() - item0;
            t.out_kind = out_kind;
            t.beta = beta;
            S->tasks.push_back(t);
        }
    };
    auto item = [&](uint64_t a_off, int64_t b_base, int K) {
        TcItem it{};
        it.a_off = a_off;
        it.b_base = b_base;
        it.KT = KT(K);
        if (it.KT > 0) S->items.push_back(it);
    };
    auto split_job = [&](int64_t src_row, int64_t dst_kt, int ld, int K) {
        SplitJob j{};
        j.src_row = src_row;
        j.dst_kt = dst_kt;
        j.ld = ld;
        j.K = K;
        j.KT = KT(K);
        if (j.KT > 0) S->jobs.push_back(j);
    };

    // W -> tiles
    begin_op(OP_SPLIT_W, -1, BUF_W, -1);
    for (int i = 0; i < nleaf; ++i) split_job(i, S->leaf_kt[i], Ddim[i], Ddim[i]);
    end_op();
    // up-sweep by height: the epilogue writes wskel directly as operand tiles
    for (int h = 0; h <= maxh; ++h) {
        begin_op(OP_TC3, POOL_VU3, h == 0 ? BUF_W : BUF_WSKEL, BUF_WSKEL);
        for (int v : bfs) {
            if (height[v] != h || !projects(v)) continue;
            const int item0 = (int)S->items.size();
            if (lch[v] == -1) {
                item(up_a[v], S->leaf_kt[lm[v]], Ddim[lm[v]]);
            } else {
                if (slen[lch[v]] > 0) item(up_a[v], S->node_kt[lch[v]], slen[lch[v]]);
                if (slen[rch[v]] > 0) item(up_b[v], S->node_kt[rch[v]], slen[rch[v]]);
            }
            add_tasks(OUT_TILES, skel_row[v], S->node_kt[v], slen[v], slen[v], item0, 0);
        }
        end_op();
    }
    // far + down by depth: a node whose parent projects keeps its far result in FP32 for the
    // down launch, which adds its own product and writes uskel tiles; other nodes' far
    // results become tiles directly
    auto has_down = [&](int c) { return parent[c] >= 0 && projects(parent[c]); };
    std::vector<std::vector<int>> far_out(numnodes);
    for (size_t k = 0; k < far_x.size(); ++k) far_out[far_x[k]].push_back((int)k);
    for (int dd = 1; dd <= maxd; ++dd) {
        begin_op(far_parts == 2 ? OP_TC2 : OP_TC3, POOL_FAR, BUF_WSKEL, BUF_USKEL);
        for (int c : bfs) {
            if (depth[c] != dd || !projects(c)) continue;
            const int item0 = (int)S->items.size();
            for (int k : far_out[c])
                if (slen[far_y[k]] > 0) item(far_a[k], S->node_kt[far_y[k]], slen[far_y[k]]);
            add_tasks(has_down(c) ? OUT_F32 : OUT_TILES, skel_row[c], S->node_kt[c], slen[c], slen[c], item0, 0);
        }
        end_op();
        begin_op(OP_TC3, POOL_VD3, BUF_USKEL, BUF_USKEL);
        for (int c : bfs) {
            if (depth[c] != dd || !projects(c) || !has_down(c)) continue;
            const int item0 = (int)S->items.size();
            item(down_child[c], S->node_kt[parent[c]], slen[parent[c]]);
            add_tasks(OUT_TILES, skel_row[c], S->node_kt[c], slen[c], slen[c], item0, 1);
        }
        end_op();
    }
    // near (Y (+)= D W) then leaf down (Y += P^T uskel)
    std::vector<std::vector<int>> near_out(nleaf);
    for (size_t k = 0; k < near_x.size(); ++k) near_out[near_x[k]].push_back((int)k);
    begin_op(near_parts == 2 ? OP_TC2 : OP_TC3, POOL_NEAR, BUF_W, -1);
    for (int v : bfs) {
        if (lch[v] != -1) continue;
        const int x = lm[v];
        const int item0 = (int)S->items.size();
        for (int k : near_out[x]) item(near_a[k], S->leaf_kt[near_y[k]], Ddim[near_y[k]]);
        add_tasks(OUT_Y, x, 0, Ddim[x], Ddim[x], item0, 2);
    }
    end_op();
    begin_op(OP_TC3, POOL_VD3, BUF_USKEL, -1);
    for (int v : bfs) {
        if (lch[v] != -1 || !projects(v)) continue;
        const int item0 = (int)S->items.size();
        item(down_a[v], S->node_kt[v], slen[v]);
        add_tasks(OUT_Y, lm[v], 0, Ddim[lm[v]], Ddim[lm[v]], item0, 1);
    }
    end_op();

    int rc = alloc((void **)&S->dTasks, std::max<size_t>(S->tasks.size(), 1) * sizeof(TcTask));
    if (!rc) rc = alloc((void **)&S->dItems, std::max<size_t>(S->items.size(), 1) * sizeof(TcItem));
    if (!rc) rc = alloc((void **)&S->dJobs, std::max<size_t>(S->jobs.size(), 1) * sizeof(SplitJob));
    if (!rc) rc = alloc((void **)&S->dErr, sizeof(int));
    if (rc) return rc;
    cudaError_t e = cudaMemcpy(S->dTasks, S->tasks.data(), S->tasks.size() * sizeof(TcTask), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !S->items.empty())
        e = cudaMemcpy(S->dItems, S->items.data(), S->items.size() * sizeof(TcItem), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !S->jobs.empty())
        e = cudaMemcpy(S->dJobs, S->jobs.data(), S->jobs.size() * sizeof(SplitJob), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(S->dErr, 0, sizeof(int));
    if (e != cudaSuccess) {
        set_error(std::string("uploading split-BF16 task lists: ") + cudaGetErrorString(e));
        return MXB_ERR_CUDA;
    }
    return MXB_OK;
}

static int split_buffers(Plan &p, SplitBF16 &S, int nrhs)
{
    const int NT = 2 * (int)ceil_div(nrhs, 256);  // even: BN = 256 launches read tile pairs
    if (NT <= S.nt_cap && nrhs <= S.nrhs_cap) return MXB_OK;
    auto release = [&](void *q) {
        if (!q) return;
        cudaFree(q);
        p.allocations.erase(std::remove(p.allocations.begin(), p.allocations.end(), q), p.allocations.end());
    };
    release(S.Wt);
    release(S.wT);
    release(S.uT);
    release(S.u32);
    S.Wt = S.wT = S.uT = nullptr;
    S.u32 = nullptr;
    const size_t tile3 = 3 * (size_t)TILE_BYTES;
    int rc = p.alloc((void **)&S.Wt, std::max<int64_t>(S.leaf_kt_total, 1) * NT * tile3);
    if (!rc) rc = p.alloc((void **)&S.wT, std::max<int64_t>(S.node_kt_total, 1) * NT * tile3);
    if (!rc) rc = p.alloc((void **)&S.uT, std::max<int64_t>(S.node_kt_total, 1) * NT * tile3);
    if (!rc) rc = p.alloc((void **)&S.u32, std::max<int64_t>(p.skel_total, 1) * (size_t)nrhs * sizeof(float));
    if (rc) return rc;
    S.nt_cap = NT;
    S.nrhs_cap = nrhs;
    return MXB_OK;
}

int Plan::prepare_split_bf16(int nrhs, bool *reallocated)
{
    const int nt_before = bf16->nt_cap, n_before = bf16->nrhs_cap;
    int rc = split_buffers(*this, *bf16, nrhs);
    if (rc) return rc;
    *reallocated = bf16->nt_cap != nt_before || bf16->nrhs_cap != n_before;
    return split_bf16_prepare();
}

int Plan::run_split_bf16(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, int accumulate,
                         cudaStream_t stream)
{
    if (&L == &launches_adj) {
        set_error("the adjoint runs in FP64 mode only (create an FP64 plan for mxb_plan_adjoint)");
        return MXB_ERR_UNSUPPORTED;
    }
    SplitBF16 &S = *bf16;
    const int NT = S.nt_cap;
    cudaError_t e = cudaSuccess;
    bool first_tc = true;
    for (const Op &o : S.ops) {
        switch (o.kind) {
        case OP_SPLIT_W:
            split_b_kernel<double><<<dim3(o.count, o.max_kt, NT), 256, 0, stream>>>(S.dJobs + o.first, dW, dOfs,
                                                                                  nrhs, NT, S.Wt);
            break;
        default: {
            TcArgs a{};
            a.a_pool = S.pool[o.a_pool];
            a.b_pool = o.b_buf == BUF_W ? S.Wt : (o.b_buf == BUF_WSKEL ? S.wT : S.uT);
            a.t_pool = o.t_buf == BUF_WSKEL ? S.wT : S.uT;
            a.Y = dY;
            a.yofs = dOfs + nleaf;
            a.err = S.dErr;
            a.NT = NT;
            a.nrhs = nrhs;
            a.skel = S.u32;
            a.beta_arg = accumulate ? 1 : 0;
            a.wait_cycles = debug_wait_cycles > 0 ? debug_wait_cycles : tc::WAIT_CYCLES;
            a.stall_test = (debug_flags & MXB_DEBUG_STALL_ONE_WAIT) && first_tc;
            first_tc = false;
            if (o.kind == OP_TC2) e = launch_tc<2, 256>(S.dTasks + o.first, S.dItems, o.count, a, stream);
            else e = launch_tc<3, 128>(S.dTasks + o.first, S.dItems, o.count, a, stream);
            break;
        }
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            set_error(std::string("split-BF16 launch: ") + cudaGetErrorString(e));
            return MXB_ERR_CUDA;
        }
    }
    return MXB_OK;
}

int split_bf16_prepare()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return MXB_ERR_CUDA;
    if (!g_sm_count[dev] && cudaDeviceGetAttribute(&g_sm_count[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return MXB_ERR_CUDA;
    if (cudaFuncSetAttribute(tc_gemm_kernel<2, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<2, 256>::SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(tc_gemm_kernel<3, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<3, 128>::SMEM) != cudaSuccess) {
        set_error("configuring the tensor-core kernels' shared memory failed");
        return MXB_ERR_CUDA;
    }
    return MXB_OK;
}

int split_bf16_launches(const Plan &p) { return p.bf16 ? (int)p.bf16->ops.size() : 0; }

int split_bf16_status(Plan &p)
{
    if (!p.bf16) return MXB_OK;
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, p.bf16->dErr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error(std::string("reading the error word: ") + cudaGetErrorString(e));
        return MXB_ERR_CUDA;
    }
    if (h) {
        cudaMemset(p.bf16->dErr, 0, sizeof(int));
        set_error("a tensor-core kernel wait timed out (MXB_ERR_TIMEOUT)");
        return h;
    }
    return MXB_OK;
}

void Plan::free_split_bf16()
{
    delete bf16;
    bf16 = nullptr;
}

}  // namespace mxb
