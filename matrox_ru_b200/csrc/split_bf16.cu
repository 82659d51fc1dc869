// Split-BF16 evaluation path on the 5th-generation tensor cores (tcgen05).
//
// Precision scheme (BF16 tensor-core products with split operands, FP32 accumulation,
// FP32-accurate transfers, FP64 final Y):
//   near D_xy W_y and far B_xy wskel_y : both operands split into bf16 hi + mid, three
//        products hi*hi + hi*mid + mid*hi ("bf16x3"), FP32 accumulation.  Splitting only W
//        leaves the CDS operand at 8 bits (~2e-3 relative error); splitting both gives ~5e-6.
//   transfers (leaf / internal projections up and down): hi + mid + lo (24 bits), six
//        products ("bf16x6"), which matches an FP32 SGEMM's error (~3e-7).
//   Y: FP64, accumulated from the FP32 tile in the epilogue.
//
// Data layout: every operand lives in HBM already in the shared-memory tile format
// (128 rows x 64 K bf16, K-major, 128-byte swizzle; the parts of one tile contiguous), so a
// pipeline stage is filled by a few 1-D bulk copies (cp.async.bulk) on an mbarrier -- no
// tensor maps, no per-element address math in the main loop.  The CDS operands (D, B, the
// projections and their transposes) are tiled once when the plan is created; W is tiled per
// evaluation by a split kernel, and the skeleton vectors are written as tiles directly by the
// GEMM epilogue.
//
// GEMM kernel (persistent, one CTA per SM, 10 warps), walking a list of work units
// (task row tile x BN right-hand sides; BN = 64, 128 or 256, picked by the autotuner):
//   warp 8 lane 0 : producer -- bulk copies of the A and B part tiles of each K step
//   warp 9 lane 0 : MMA issuer -- tcgen05.mma M=128, N=BN, K=16, 3 or 6 per 16-K slice, one
//                   fresh TMEM accumulator (of two) per 64-deep K tile
//   warps 0-7     : drain every K tile's accumulator into round-to-nearest FP32 registers
//                   (tcgen05.ld), then write Y (FP64), an FP32 block, or operand tiles
// A task carries the index of its plan, so one launch can serve many H-matrices (batches).
// Every wait is bounded; a CTA that times out raises MXB_ERR_TIMEOUT in the error word,
// drains its own copies and MMAs, frees its TMEM and exits.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <queue>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"
#include "plan.h"
#include "tc_common.cuh"

#define MXB_CUDA_OR(call)                                                                 \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return MXB_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

namespace mxb {

int row_tile_for(int precision) { return precision != MXB_PREC_FP64 ? 128 : 64; }

namespace {

using tc::TILE_BYTES;

// POOL_NEART / POOL_FART: the near blocks and far couplings transposed (plans with the adjoint)
enum APool { POOL_NEAR, POOL_FAR, POOL_VU3, POOL_VD3, POOL_NEART, POOL_FART, NPOOL };
enum BBuf { BUF_W, BUF_WSKEL, BUF_USKEL, NBUF };

struct TcItem {
    uint64_t a_off;   // byte offset of A's tile (0, 0) in the plan's A pool `a_pool`
    int64_t b_base;   // K-tile base of the B operand's node / leaf in the B buffer `b_buf`
    int32_t KT;       // K tiles of this item
    int32_t K;        // K before padding to whole tiles (flop accounting)
    int16_t a_pool;   // APool of A
    int16_t b_buf;    // BBuf of B
    int32_t pad;
};
static_assert(sizeof(TcItem) == 32, "TcItem layout");

// Output of a tensor-core task.
enum OutKind : int16_t {
    OUT_Y = 0,      // FP64 Y block (leaf-blocked, caller's offsets)
    OUT_F32 = 1,    // FP32 skeleton block (a far result the down launch adds to)
    OUT_TILES = 2,  // skeleton block written as 3-part bf16 operand tiles for the next launches
    OUT_SPLIT = 3,  // no product: one leaf's W block split into 3-part operand tiles (c_row:
                    // leaf, out_kt: its K-tile base, M: its points; a unit's col: 128-column tile)
};

struct TcTask {
    int64_t c_row;   // leaf index (OUT_Y) or skeleton row offset (FP32 block)
    int64_t out_kt;  // K-tile base of the node in the tile buffer (OUT_TILES)
    int32_t ldc;
    int32_t M;       // rows of the whole output block
    int32_t m0;      // first row of this task's 128-row tile
    int32_t item0;
    int32_t nitem;
    int32_t plan;    // index into the launch's plan table
    int16_t out_kind;
    int16_t beta;    // 0 overwrite, 1 accumulate (OUT_TILES: add the FP32 block), 2 plan's arg
    int32_t t_buf;   // BBuf that OUT_TILES writes
};

struct TcUnit {
    int32_t task;
    int32_t col;     // column tile: right-hand sides [col * BN, col * BN + BN)
    int32_t ktiles;  // K tiles of the task (sum over its items)
    int32_t chain;   // chained launches: parts << 28 | level << 20 | units of the level before
                     // (parts 2 or 3: the unit's operand parts when they differ from the launch's)
    // Dataflow launches (LaunchArgs::deps): the unit loads its B tiles once the node counters
    // dep0 / dep1 (-1: none) have counted need0 / need1 finished units (need0 | need1 << 16),
    // and counts itself into counter `sig` (-1: none) once its output is written.
    int32_t dep0, dep1;
    int32_t need;
    int32_t sig;
};
static_assert(sizeof(TcUnit) == 32, "TcUnit layout");

struct SplitJob {     // one leaf block of W -> B-operand tiles
    int64_t src_row;  // leaf index
    int64_t dst_kt;   // K-tile base in the W tile buffer
    int32_t ld, K, KT, plan;
};

struct PoolJob {      // one CDS matrix -> tiled parts (plan creation)
    uint64_t src_off;  // element offset in the FP64 pool
    uint64_t dst_off;  // byte offset of tile (0, 0)
    int32_t src_pool, ld, R, K, RT, KT, trans, parts;
};

// Per-plan pointers of one evaluation (device table indexed by TcTask::plan / SplitJob::plan).
struct PlanArgs {
    const uint8_t *pool[NPOOL];
    uint8_t *buf[NBUF];  // W tiles, wskel tiles, uskel tiles
    const double *W;
    double *Y;
    const int32_t *wofs;
    const int32_t *yofs;
    float *skel;         // FP32 far results awaiting the down launch
    // caller point order (null: leaf-blocked W / Y at wofs / yofs): tree position t of leaf
    // i (t from tofs[i]) is row perm[t]; element (row, j) of W at row * w_rs + j * w_cs
    const int32_t *w_perm;
    const int32_t *y_perm;
    const int32_t *tofs;
    int64_t w_rs, w_cs, y_rs, y_cs;
    int32_t NT;          // 128-column tiles per node in the B buffers (even)
    int32_t nrhs;
    int32_t beta_arg;
    int32_t pad;
};

// Tree levels one tensor-core launch may chain (consecutive ops of one product count and tile,
// e.g. the up-sweep heights): the units of level j wait on the device until every unit of
// level j - 1 has been written.
constexpr int MAX_CHAIN = 24;
// Tile-code flag (above MXB_TILE_PAIR): the op runs in the launch of the op before it.
constexpr int TILE_CHAIN = 1 << 13;

struct LaunchArgs {
    const PlanArgs *plans;
    const TcTask *tasks;
    const TcItem *items;
    const TcUnit *units;
    int *next_unit;         // work-unit counter of this launch, zero at launch
    int *err;
    long long wait_cycles;  // limit of every wait in the kernel
    int nunits;
    int stall_test;         // test hook: CTA 0 withholds its first stage, so a wait runs out
    int kchain;             // K tiles accumulated per TMEM accumulator fill (1 or 2)
    int nlevels;            // chained levels (1: none); a unit's level is in TcUnit::chain
    int *level_done;        // per level: epilogue warps done with a unit of it (zero at launch)
    int stall_level;        // test hook: level 0 never reports done, so level 1's waits run out
    // profiling of chained launches (null otherwise): [0] the earliest CTA start, [1 + j] the
    // time the last unit of level j was written (%globaltimer, ns)
    unsigned long long *level_ns;
    // dataflow launches (null otherwise): per-node completion counters, zero at launch; units
    // wait for the nodes whose tiles they read instead of for whole levels (TcUnit::dep0/dep1)
    int *deps;
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

// W (FP64, leaf-blocked) -> B-operand tiles with 3 parts, for every plan of the launch.
// B(n, k) = W[k + n ld]; rows n >= nrhs and k >= K are zero.  ORD: the evaluation reads W in
// the caller's point order (PlanArgs::w_perm), a separate instantiation so the leaf-blocked
// one keeps its small footprint.
template <bool ORD>
__global__ void __launch_bounds__(256) split_w_kernel(const SplitJob *__restrict__ jobs,
                                                      const PlanArgs *__restrict__ plans)
{
    const SplitJob j = jobs[blockIdx.x];
    const PlanArgs *pa = plans + j.plan;
    const int kt = blockIdx.y, nt = blockIdx.z;
    if (kt >= j.KT || nt >= pa->NT) return;
    const int nrhs = pa->nrhs;
    uint8_t *tile0 = pa->buf[BUF_W] + ((size_t)j.dst_kt * pa->NT + (size_t)nt * j.KT + kt) * 3 * (size_t)TILE_BYTES;
    if (ORD && pa->w_perm) {
        // caller point order: gather rows perm[t] of W through shared memory, 32 K indices
        // (rows of W) at a time across all 128 columns of the tile.  Lanes run along a row, so
        // a row-major W is read in 1 KiB runs; the split then reads the staged values back in
        // the tile order of the path below (chunks 4 h .. 4 h + 3 of every tile row).
        __shared__ double stage[32][129];  // [K index][column]
        const int32_t *rows = pa->w_perm + pa->tofs[j.src_row];
        const int64_t rs = pa->w_rs, cs = pa->w_cs;
        const int n = nt * 128 + (threadIdx.x & 127);
        const double *wc = pa->W + (int64_t)n * cs;
        for (int h = 0; h < 2; ++h) {
            // this thread's 16 K indices: kk = threadIdx.x / 128 + 2 i; its column: threadIdx.x % 128
            int64_t rofs[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int k = kt * 64 + h * 32 + (threadIdx.x >> 7) + 2 * i;
                rofs[i] = k < j.K ? (int64_t)rows[k] * rs : -1;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i)
                stage[(threadIdx.x >> 7) + 2 * i][threadIdx.x & 127] = (n < nrhs && rofs[i] >= 0) ? wc[rofs[i]] : 0.0;
            __syncthreads();
            for (int q = threadIdx.x; q < 128 * 4; q += 256) {
                const int c = q & 3, rr = q >> 2;
                __nv_bfloat16 hi[8], mi[8], lo[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) tc::split3(stage[c * 8 + e][rr], hi[e], mi[e], lo[e]);
                store_parts(tile0, 3, rr, h * 4 + c, hi, mi, lo);
            }
            __syncthreads();
        }
        return;
    }
    const double *src = pa->W + pa->wofs[j.src_row];
    for (int i = 0; i < 4; ++i) {
        const int idx = threadIdx.x + i * 256;
        const int c = idx % 8, r = idx / 8;
        const int n = nt * 128 + r;
        __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int k = kt * 64 + c * 8 + e;
            double x = 0.0;
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

// Launch shape.  PAIR: a cluster of two CTAs (one per SM) computes a 256-row x BN tile with
// tcgen05.mma.cta_group::2; each CTA stages its own 128 rows of A and half of the BN rows of
// B, so a pair moves a third less operand data per flop than two single CTAs and has room for
// a deeper pipeline.
template <int P, int BN, int STAGES_, bool PAIR = false>
struct TcCfg {
    static constexpr int STAGES = STAGES_;
    static constexpr int B_ROWS = PAIR ? BN / 2 : BN;      // B rows (output columns) staged per CTA
    static constexpr int B_ROWS_BYTES = B_ROWS * 128;      // one part of the staged B operand
    static constexpr int A_BYTES = P * TILE_BYTES;
    static constexpr int B_BYTES = P * B_ROWS_BYTES;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int SMEM = STAGES * STAGE + 1024 + 1024;  // + alignment, barriers, unit ring
    static constexpr int NPROD = P == 2 ? 3 : 6;
    static constexpr int EPI_WARPS = 8;          // two per TMEM lane quarter, one per column half
    static constexpr int RING = 16;              // work units published ahead of the readers
    // readers of a ring slot: MMA issuer and epilogue warps (+ the odd CTA's producer, relay
    // and epilogue warps in a pair)
    static constexpr int RING_READERS = PAIR ? 2 * (1 + EPI_WARPS) + 1 : 1 + EPI_WARPS;
    static constexpr int THREADS = (EPI_WARPS + 2) * 32;
    // level-count increments per unit: one per epilogue warp (of both CTAs of a pair)
    static constexpr int UNIT_WRITERS = EPI_WARPS * (PAIR ? 2 : 1);
    static constexpr int COLS = BN / 2;          // accumulator columns per epilogue thread
    // old values loaded ahead of the stores in the epilogue's read-modify-writes (fewer where
    // 128 accumulators already fill the registers)
    static constexpr int RMW = COLS >= 128 ? 8 : 16;
    static constexpr int NACC = BN >= 256 ? 2 : 4;  // TMEM accumulator buffers (512 columns at most)
    static constexpr int TMEM_COLS = NACC * BN;
    static constexpr int M_MMA = PAIR ? 256 : 128;
    static_assert(SMEM <= 232448, "shared memory");
    static_assert(B_ROWS % 64 == 0, "B rows per CTA");
};

// Tensor-core FP32 accumulation is not round-to-nearest: its error grows with the number of
// MMAs chained into one accumulator (measured ~4e-5 relative after 8192-deep chains).  So
// every 64-deep K tile (bf16x6 launches) or pair of K tiles (bf16x3 launches, whose split
// error is ten times larger) gets a fresh TMEM accumulator (2 or 4 buffers in rotation), and the
// epilogue warps add every tile's partial sums into per-thread FP32 registers with ordinary
// round-to-nearest adds while the tensor core already works on the next tiles.
//
// Persistent with dynamic scheduling: the producer thread of a CTA (of the even CTA of a pair)
// claims work units from the launch's counter in list order (longest first) and publishes each
// unit in a ring in shared memory (in both CTAs of a pair); every role reads the ring, so all
// roles walk the same sequence, and one K-tile counter drives every stage and accumulator
// phase.  TMEM and the barriers are set up once, and the epilogue of one unit overlaps the
// MMAs of the next.  A unit of -1 ends the sequence.
//
// In a pair the even CTA issues the MMAs.  The odd CTA's MMA-warp thread relays "my stage has
// landed" to the even CTA's pfull barrier, its epilogue warps arrive on the even CTA's acce
// barrier, and the even CTA's commits arrive on both CTAs' barriers.  A failed wait in either
// CTA sets both CTAs' abort words.
template <int P, int BN, int STAGES_, bool PAIR, bool ORD>
__global__ void __launch_bounds__(TcCfg<P, BN, STAGES_, PAIR>::THREADS, 1) tc_gemm_kernel(LaunchArgs la)
{
    using C = TcCfg<P, BN, STAGES_, PAIR>;
    constexpr int NB = C::STAGES;  // full / empty / pair barriers: one per stage
    constexpr int RING = C::RING;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    uint64_t *empty = full + NB;
    uint64_t *pfull = empty + NB;  // pair: the odd CTA's copy of the stage has landed
    uint64_t *accf = pfull + NB;   // accumulator buffer b holds a finished K tile
    uint64_t *acce = accf + C::NACC;      // accumulator buffer b has been drained
    uint64_t *doneb = acce + C::NACC;     // every MMA of this CTA (pair) has completed
    uint64_t *ufull = doneb + 1;          // ring slot i holds a unit
    uint64_t *uempty = ufull + RING;      // every reader of ring slot i has taken its unit
    volatile int *ring = reinterpret_cast<volatile int *>(uempty + RING);
    volatile int *ring_kt = ring + RING;  // K tiles of the unit in ring slot i
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(const_cast<int *>(ring_kt) + RING);
    volatile int *abort_word = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = PAIR ? tc::cluster_ctarank() : 0u;
    const bool issuer = rank == 0;
    auto raise_abort = [&]() {
        *abort_word = 1;
        if constexpr (PAIR) tc::st_remote_u32(tc::peer_smem((const void *)abort_word, rank ^ 1u), 1u);
    };
    // waits on barriers that the other CTA of a pair completes take cluster-scope acquire
    auto wait_x = [&](uint64_t *bar, uint32_t parity, volatile int *ab) {
        if constexpr (PAIR) return tc::mbar_wait_cluster(bar, parity, ab, la.wait_cycles);
        else return tc::mbar_wait(bar, parity, ab, la.wait_cycles);
    };
    auto arrive_local = [&](uint64_t *bar) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tc::smem_u32(bar)) : "memory");
    };
    // Next unit of the ring for a reader (one thread): waits for slot `slot`, takes the unit,
    // its K-tile count and its operand parts (published as ktiles | parts << 24, so the MMA
    // issuer needs no global load per unit), and releases the slot to the producer (in the
    // even CTA of a pair).  -2: a wait gave up.
    auto take_unit = [&](uint32_t &slot, int &ktiles, int *parts = nullptr) -> int {
        const int i = (int)(slot % RING);
        const uint32_t parity = (slot / RING) & 1u;
        ++slot;
        int u = -2;
        if (wait_x(&ufull[i], parity, abort_word)) {
            u = ring[i];
            const int v = ring_kt[i];
            ktiles = v & 0xFFFFFF;
            if (parts) *parts = v >> 24;
        }
        if constexpr (PAIR) {
            if (rank == 1) tc::mbar_arrive_remote(tc::peer_smem(&uempty[i], 0));
            else arrive_local(&uempty[i]);
        } else {
            arrive_local(&uempty[i]);
        }
        return u;
    };

    // Operand parts of a unit (2: bf16x3 products, 3: bf16x6) and K tiles per accumulator fill:
    // the launch's, or the unit's own in launches that mix both (those run with P = 3 stages).
    auto unit_parts = [&](int32_t chain) { const int c = (chain >> 28) & 3; return c ? c : P; };
    auto unit_kchain = [&](int parts) { return parts == P ? la.kchain : (parts == 2 ? 2 : 1); };

    if (threadIdx.x == 0) {
        for (int s = 0; s < NB; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
            tc::mbar_init(&pfull[s], 1);
        }
        for (int b = 0; b < C::NACC; ++b) {
            tc::mbar_init(&accf[b], 1);
            tc::mbar_init(&acce[b], C::EPI_WARPS * (PAIR ? 2 : 1));
        }
        tc::mbar_init(doneb, 1);
        for (int i = 0; i < RING; ++i) {
            tc::mbar_init(&ufull[i], 1);
            tc::mbar_init(&uempty[i], C::RING_READERS);
        }
        *abort_word = 0;

        tc::fence_mbar_init();
    }
    if (warp == 0) {
        if constexpr (PAIR) tc::tmem_alloc_pair(tmem_slot, C::TMEM_COLS);
        else tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
    }
    tc::fence_before_sync();
    __syncthreads();
    if constexpr (PAIR) tc::cluster_sync();  // both CTAs' barriers and TMEM exist
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    if (la.level_ns && threadIdx.x == 0) atomicMin(la.level_ns, tc::globaltimer_ns());

    if (warp == C::EPI_WARPS) {
        if (lane == 0) {
            // ---------------- producer ----------------
            uint32_t g = 0;               // K-tile counter of this CTA
            uint32_t slot = 0;            // ring counter
            int waited = 0;               // last chained level waited for
            uint32_t filled[C::STAGES];   // rounds filled per stage (drained before exit)
#pragma unroll
            for (int s = 0; s < C::STAGES; ++s) filled[s] = 0;
            bool stop = false;
            // Lookahead (the claiming CTA): the next unit is claimed, and its unit and task
            // records are loaded, while the current unit's copies are issued -- one dependent step
            // per K tile -- so a new unit does not start with a chain of global round trips
            // (claim, unit record, task record).  A CTA holds at most two claimed units, which it
            // runs in claim order.
            int nu = -1;
            TcUnit nun{};
            TcTask ntk{};
            int nstate = 0;  // 0: nothing claimed, 1: claimed, 2: unit record loaded, 3: task loaded
            auto advance = [&]() {
                if (nstate == 0) {
                    nu = atomicAdd(la.next_unit, 1);
                } else if (nstate == 1) {
                    if (nu >= la.nunits) nu = -1;
                    if (nu >= 0) nun = la.units[nu];
                } else if (nstate == 2) {
                    if (nu >= 0) ntk = la.tasks[nun.task];
                }
                ++nstate;
            };
            while (!stop && !*abort_word) {
                int u, kt_unit = 0;
                TcUnit un{};
                TcTask t{};
                if (!PAIR || issuer) {
                    // take the claimed unit and publish it to every reader
                    while (nstate < 3) advance();
                    u = nu;
                    un = nun;
                    t = ntk;
                    nstate = 0;
                    int kt_pub = 0;
                    if (u >= 0) {
                        kt_unit = un.ktiles;
                        kt_pub = un.ktiles | (unit_parts(un.chain) << 24);
                    }
                    const int i = (int)(slot % RING);
                    const uint32_t round = slot / RING;
                    ++slot;
                    if (!wait_x(&uempty[i], (round & 1) ^ 1, abort_word)) {
                        raise_abort();
                        break;
                    }
                    ring[i] = u;
                    ring_kt[i] = kt_pub;
                    if constexpr (PAIR) {
                        tc::st_remote_u32(tc::peer_smem((const void *)&ring[i], 1), (uint32_t)u);
                        tc::st_remote_u32(tc::peer_smem((const void *)&ring_kt[i], 1), (uint32_t)kt_pub);
                        tc::mbar_arrive_remote(tc::peer_smem(&ufull[i], 1));
                    }
                    arrive_local(&ufull[i]);
                } else {
                    u = take_unit(slot, kt_unit);
                    if (u == -2) {
                        raise_abort();
                        break;
                    }
                    if (u >= 0) {
                        un = la.units[u];
                        t = la.tasks[un.task];
                    }
                }
                if (u < 0) break;
                if (la.nlevels > 1) {
                    // a unit of a chained level reads what the previous level wrote: wait until
                    // every epilogue warp has finished every unit of that level
                    const int lvl = (un.chain >> 20) & 0xFF;
                    if (lvl > waited) {
                        if (!tc::wait_counter(la.level_done + lvl - 1, (un.chain & 0xFFFFF) * C::UNIT_WRITERS,
                                              abort_word, la.wait_cycles)) {
                            raise_abort();
                            break;
                        }
                        waited = lvl;
                    }
                }
                if (la.deps) {
                    // dataflow: the nodes whose tiles this unit reads have written them for this
                    // column tile (every one of their units, every epilogue warp)
                    bool ok = un.dep0 < 0 || tc::wait_counter(la.deps + un.dep0, (un.need & 0xFFFF) * C::UNIT_WRITERS,
                                                              abort_word, la.wait_cycles);
                    if (ok && un.dep1 >= 0)
                        ok = tc::wait_counter(la.deps + un.dep1, (un.need >> 16) * C::UNIT_WRITERS, abort_word,
                                              la.wait_cycles);
                    if (!ok) {
                        raise_abort();
                        break;
                    }
                }
                const PlanArgs *pa = la.plans + t.plan;
                const int NT = pa->NT;
                const int cb = un.col * BN + (int)rank * C::B_ROWS;  // first B row staged here
                const TcItem *ti = la.items + t.item0;
                const int mt = t.m0 / 128 + (int)rank;
                // the odd CTA's rows may lie past the block: its A tile does not exist, and the
                // MMA rows it feeds are never stored
                const bool a_ok = !PAIR || issuer || t.m0 + 128 < t.M;
                const int up = unit_parts(un.chain);
                const uint32_t tx = (a_ok ? (uint32_t)up * TILE_BYTES : 0u) + (uint32_t)up * C::B_ROWS_BYTES;
                TcItem it_next{};
                if (t.nitem > 0) it_next = ti[0];
                for (int q = 0; q < t.nitem && !stop; ++q) {
                    const TcItem it = it_next;
                    if (q + 1 < t.nitem) it_next = ti[q + 1];  // loaded while this item's copies go out
                    const uint8_t *a_pool = pa->pool[it.a_pool];
                    const uint8_t *b_pool = pa->buf[it.b_buf];
                    for (int kt = 0; kt < it.KT; ++kt, ++g) {
                        const int s = g % C::STAGES;
                        const uint32_t round = g / C::STAGES;
                        if (!wait_x(&empty[s], (round & 1) ^ 1, abort_word)) {
                            raise_abort();
                            stop = true;
                            break;
                        }
                        if (la.stall_test && blockIdx.x == 0 && g == 0) continue;  // never filled
                        uint8_t *sa = smem + s * C::STAGE;
                        uint8_t *sb = sa + C::A_BYTES;
                        tc::mbar_expect_tx(&full[s], tx);
                        if (a_ok) {
                            const uint8_t *ga = a_pool + it.a_off + ((size_t)mt * it.KT + kt) * (size_t)up * TILE_BYTES;
                            tc::bulk_g2s(sa, ga, (uint32_t)up * TILE_BYTES, &full[s]);
                        }
                        if (C::B_ROWS >= 128) {
#pragma unroll
                            for (int hh = 0; hh < C::B_ROWS / 128; ++hh) {
                                const size_t nt = (size_t)(cb >> 7) + hh;
                                const uint8_t *gb =
                                    b_pool + ((size_t)it.b_base * NT + nt * it.KT + kt) * 3 * (size_t)TILE_BYTES;
#pragma unroll
                                for (int p = 0; p < P; ++p)
                                    if (p < up)
                                        tc::bulk_g2s(sb + p * C::B_ROWS_BYTES + hh * TILE_BYTES,
                                                     gb + (size_t)p * TILE_BYTES, TILE_BYTES, &full[s]);
                            }
                        } else {
                            // B_ROWS rows starting at row cb % 128 of a 128-row tile: contiguous, and
                            // the swizzle phase (row % 8) is unchanged by the 64-row offset
                            const uint8_t *gb = b_pool +
                                                ((size_t)it.b_base * NT + (size_t)(cb >> 7) * it.KT + kt) * 3 *
                                                    (size_t)TILE_BYTES +
                                                (size_t)(cb & 127) * 128;
#pragma unroll
                            for (int p = 0; p < P; ++p)
                                if (p < up)
                                    tc::bulk_g2s(sb + p * C::B_ROWS_BYTES, gb + (size_t)p * TILE_BYTES, C::B_ROWS_BYTES,
                                                 &full[s]);
                        }
                        filled[s] = round + 1;
                        if ((!PAIR || issuer) && nstate < 3) advance();
                    }
                }
            }
            // every stage this thread filled must have landed before the CTA may exit
#pragma unroll
            for (int s = 0; s < C::STAGES; ++s) {
                if (!filled[s]) continue;
                volatile int never = 0;
                tc::mbar_wait(&full[s], (filled[s] - 1) & 1, &never, la.wait_cycles);
            }
        }
    } else if (warp == C::EPI_WARPS + 1) {
        if (lane == 0 && issuer) {
            // ---------------- MMA issuer ----------------
            constexpr uint32_t IDESC = tc::idesc_bf16_f32(C::M_MMA, BN);
            constexpr int PA[6] = {0, 0, 1, 0, 1, 2};
            constexpr int PB[6] = {0, 1, 0, 2, 1, 0};
            uint32_t g = 0;     // K-tile (stage) counter
            uint32_t ga = 0;    // accumulator-fill counter
            uint32_t slot = 0;  // ring counter
            bool any = false, stop = false;
            while (!stop) {
                int ktiles = 0, up = P;
                const int u = take_unit(slot, ktiles, &up);
                if (u < 0) {
                    if (u == -2) raise_abort();
                    break;
                }
                const int nprod = up == 2 ? 3 : 6;
                const int kc = unit_kchain(up);
                for (int i = 0; i < ktiles; ++i, ++g) {
                    const int s = g % C::STAGES;
                    const uint32_t round = g / C::STAGES;
                    const int b = ga % C::NACC;
                    const uint32_t use = ga / C::NACC;
                    const bool first = i % kc == 0;
                    const bool last = i % kc == kc - 1 || i == ktiles - 1;
                    if ((first && !wait_x(&acce[b], (use & 1) ^ 1, abort_word)) ||
                        !tc::mbar_wait(&full[s], round & 1, abort_word, la.wait_cycles) ||
                        (PAIR && !wait_x(&pfull[s], round & 1, abort_word))) {
                        raise_abort();
                        stop = true;
                        break;
                    }
                    tc::fence_after_sync();
                    // descriptors of the stage's part tiles; a byte offset o within the stage adds
                    // o >> 4 to the start-address field (shared addresses stay below 2^18)
                    const uint32_t sa = tc::smem_u32(smem + s * C::STAGE);
                    const uint64_t da = tc::smem_desc_sw128(sa), db = tc::smem_desc_sw128(sa + C::A_BYTES);
                    const uint32_t dst = tmem + (uint32_t)(b * BN);
                    // the products of one K tile, fully unrolled for each product count (no
                    // run-time loop bound between the MMAs)
                    auto issue = [&](auto np) {
                        uint32_t accum = first ? 0u : 1u;
#pragma unroll
                        for (int ks = 0; ks < 4; ++ks) {
#pragma unroll
                            for (int j = 0; j < decltype(np)::value; ++j) {
                                const uint64_t ad = da + (uint64_t)((PA[j] * TILE_BYTES + ks * 32) >> 4);
                                const uint64_t bd = db + (uint64_t)((PB[j] * C::B_ROWS_BYTES + ks * 32) >> 4);
                                if constexpr (PAIR) tc::mma_bf16_pair(dst, ad, bd, IDESC, accum);
                                else tc::mma_bf16(dst, ad, bd, IDESC, accum);
                                accum = 1;
                            }
                        }
                    };
                    if (C::NPROD == 3 || nprod == 3) issue(std::integral_constant<int, 3>{});
                    else issue(std::integral_constant<int, 6>{});
                    if constexpr (PAIR) {
                        tc::mma_commit_pair(&empty[s]);
                        if (last) tc::mma_commit_pair(&accf[b]);
                    } else {
                        tc::mma_commit(&empty[s]);
                        if (last) tc::mma_commit(&accf[b]);
                    }
                    if (last) ++ga;
                    any = true;
                }
            }
            if (any) {
                if constexpr (PAIR) tc::mma_commit_pair(doneb);
                else tc::mma_commit(doneb);
            } else {
                tc::mbar_expect_tx(doneb, 0);  // nothing issued: complete the barrier's phase now
                if constexpr (PAIR) tc::mbar_arrive_remote(tc::peer_smem(doneb, 1));
            }
        } else if (lane == 0 && PAIR) {
            // ---------------- relay (odd CTA of a pair) ----------------
            uint32_t g = 0, slot = 0;
            bool stop = false;
            while (!stop) {
                int ktiles = 0;
                const int u = take_unit(slot, ktiles);
                if (u < 0) {
                    if (u == -2) raise_abort();
                    break;
                }
                for (int i = 0; i < ktiles; ++i, ++g) {
                    const int s = g % C::STAGES;
                    const uint32_t round = g / C::STAGES;
                    if (!tc::mbar_wait(&full[s], round & 1, abort_word, la.wait_cycles)) {
                        raise_abort();
                        stop = true;
                        break;
                    }
                    tc::mbar_arrive_remote(tc::peer_smem(&pfull[s], 0));
                }
            }
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        const uint32_t acce0 = PAIR ? tc::peer_smem(&acce[0], 0) : tc::smem_u32(&acce[0]);
        uint32_t g = 0, slot = 0;
        int ewaited = 0;  // last chained level this warp acquired
        // Chained launches: this warp's finished units of level pend_level not yet counted.  They
        // are counted (after one fence for all their stores) when the warp takes its first unit
        // of a later level, or at the end: one fence and one atomic per level and warp.
        int pend_level = 0, pend = 0;
        auto flush = [&]() {
            if (!pend) return;
            asm volatile("fence.proxy.async.global;\n" ::: "memory");
            __threadfence();
            __syncwarp();
            if (lane == 0) {
                if (!(la.stall_level && pend_level == 0)) atomicAdd(la.level_done + pend_level, pend);
                if (la.level_ns) atomicMax(la.level_ns + 1 + pend_level, tc::globaltimer_ns());
            }
            pend = 0;
        };
        for (;;) {
            int u = 0, ktiles = 0;
            if (lane == 0) u = take_unit(slot, ktiles);
            u = __shfl_sync(0xffffffffu, u, 0);
            ktiles = __shfl_sync(0xffffffffu, ktiles, 0);
            if (u < 0) {
                if (u == -2 && lane == 0) raise_abort();
                if (u == -1) flush();
                break;
            }
            const TcUnit un = la.units[u];
            if (la.nlevels > 1 && ((un.chain >> 20) & 0xFF) != pend_level) {
                flush();
                pend_level = (un.chain >> 20) & 0xFF;
            }
            const TcTask t = la.tasks[un.task];
            const int kc = unit_kchain(unit_parts(un.chain));
            const int fills = (ktiles + kc - 1) / kc;
            if (la.nlevels > 1 && ((un.chain >> 20) & 0xFF) > ewaited) {
                // the old values this unit reads back (Y, the far result) may come from an
                // earlier level of this launch: acquire that level's completion here too (the
                // producer's wait covers only its bulk copies), once per level and warp.  Lane 0
                // waits; then every lane takes its own acquire of the completed count.
                const int lvl = (un.chain >> 20) & 0xFF;
                ewaited = lvl;
                const int *ctr = la.level_done + lvl - 1;
                int done = 1;
                if (lane == 0)
                    done = tc::wait_counter(ctr, (un.chain & 0xFFFFF) * C::UNIT_WRITERS, abort_word, la.wait_cycles);
                done = __shfl_sync(0xffffffffu, done, 0);
                if (!done) {
                    if (lane == 0) raise_abort();
                    break;
                }
                tc::acquire_counter(ctr);
            }
            {
                // The output phase reads old values (Y, the far result) with a few loads in
                // flight per thread: ask L2 for them now, so the unit's MMAs cover the DRAM
                // latency.  Lane j takes columns j, j + 32, ... of its warp's 32-row segment
                // (128 bytes of FP32, 256 of FP64 per column).
                const PlanArgs *pa = la.plans + t.plan;
                const int r0 = t.m0 + (int)rank * 128 + quarter * 32;
                const int c0 = un.col * BN + half * C::COLS;
                const int beta = t.beta == 2 ? pa->beta_arg : t.beta;
                const int nrhs = pa->nrhs;
                const char *f32 = nullptr, *f64 = nullptr;
                if (ORD && t.out_kind == OUT_Y && beta && pa->y_perm) {
                    // caller point order: each lane asks for its own row's columns when they
                    // are contiguous (one 128-byte line per 16 columns)
                    const int rl = r0 + lane;
                    if (rl < t.M && pa->y_cs == 1) {
                        const char *q = reinterpret_cast<const char *>(
                            pa->Y + (int64_t)pa->y_perm[pa->tofs[t.c_row] + rl] * pa->y_rs + c0);
                        const int ncol = min(C::COLS, nrhs - c0);
                        for (int j = 0; j < ncol; j += 16) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(q + j * 8));
                    }
                } else if (t.out_kind == OUT_Y && beta) {
                    f64 = reinterpret_cast<const char *>(pa->Y + pa->yofs[t.c_row] + r0);
                } else if (t.out_kind == OUT_TILES && beta) {
                    f32 = reinterpret_cast<const char *>(pa->skel + t.c_row * (int64_t)nrhs + r0);
                }
                if (r0 < t.M && (f32 || f64)) {
                    for (int j = lane; j < C::COLS; j += 32) {
                        const int cc = c0 + j;
                        if (cc >= nrhs) break;
                        if (f32) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(f32 + (size_t)cc * t.ldc * 4));
                        if (f64) {  // rows r0 and r0 + 16 (only where they exist)
                            const char *q = f64 + (size_t)cc * t.ldc * 8;
                            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(q));
                            if (r0 + 16 < t.M) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(q + 128));
                        }
                    }
                }
            }
            float acc[C::COLS];
#pragma unroll
            for (int e = 0; e < C::COLS; ++e) acc[e] = 0.f;
            bool ok = !*abort_word;
            for (int i = 0; i < fills && ok; ++i, ++g) {
                const int b = g % C::NACC;
                const uint32_t use = g / C::NACC;
                if (!wait_x(&accf[b], use & 1, abort_word)) {
                    raise_abort();
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                // 64 columns per load where the registers allow (one wait per 64 columns keeps
                // the drain short); 128-column halves load 16 at a time to stay clear of spills
                constexpr int LB = C::COLS == 64 ? 64 : (C::COLS >= 128 ? 16 : 32);
#pragma unroll
                for (int c0 = 0; c0 < C::COLS; c0 += LB) {
                    float v[LB];
                    const uint32_t ta = tmem + lane_base + (uint32_t)(b * BN + half * C::COLS + c0);
                    if constexpr (LB == 64) tc::tmem_ld64(ta, v);
                    else if constexpr (LB == 32) tc::tmem_ld32(ta, v);
                    else tc::tmem_ld16(ta, v);
#pragma unroll
                    for (int e = 0; e < LB; ++e) acc[c0 + e] += v[e];
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    if constexpr (PAIR) tc::mbar_arrive_remote(acce0 + (uint32_t)(b * 8));
                    else asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(acce0 + (uint32_t)(b * 8))
                                      : "memory");
                }
            }
            if (!ok || *abort_word) break;
            const PlanArgs *pa = la.plans + t.plan;
            const int nrhs = pa->nrhs;
            const int r = t.m0 + (int)rank * 128 + quarter * 32 + lane;
            const int beta = t.beta == 2 ? pa->beta_arg : t.beta;
            const int col0 = un.col * BN + half * C::COLS;
            // accumulating outputs: all old values of a 16-column chunk are loaded before any
            // store, so the loads overlap instead of waiting on each other
            if (ORD && t.out_kind == OUT_Y && pa->y_perm) {
                // caller point order: row t of the leaf goes to row perm[t] of Y.  An 8 x 8
                // transpose inside each group of 8 lanes gives every lane one column of 8
                // consecutive tree rows, so each access covers 8 columns (64 bytes) of a row, 4
                // rows per warp instruction, instead of 32 rows.  All lanes take part in the
                // shuffles; rows past M are masked at the accesses.
                const int rg = t.m0 + (int)rank * 128 + quarter * 32 + (lane & ~7);  // group's first row
                const int rows_ok = t.M - rg;  // rows rg + j with j < rows_ok exist
                // lane 8g + i holds the element offset of caller row perm[rg + i]; the others
                // shuffle it
                const int64_t roff =
                    (lane & 7) < rows_ok ? (int64_t)pa->y_perm[pa->tofs[t.c_row] + rg + (lane & 7)] * pa->y_rs : 0;
                const int64_t ycs = pa->y_cs;
                double *ycol = pa->Y + (int64_t)(col0 + (lane & 7)) * ycs;  // advances 8 columns a group
                // per batch: GB column groups x JB rows of old values in flight (fewer where 128
                // accumulators already fill the registers)
                constexpr int GB = C::COLS >= 128 ? 1 : 2;
                constexpr int JB = C::COLS >= 128 ? 4 : 8;
#pragma unroll
                for (int g8 = 0; g8 < C::COLS / 8; g8 += GB) {
                    float x[GB][8];
#pragma unroll
                    for (int gb = 0; gb < GB; ++gb) {
#pragma unroll
                        for (int j = 0; j < 8; ++j) x[gb][j] = acc[8 * (g8 + gb) + j];
                        transpose8(x[gb], lane);  // x[gb][j]: row rg + j, column col0 + 8 (g8 + gb) + (lane & 7)
                    }
#pragma unroll
                    for (int j0 = 0; j0 < 8; j0 += JB) {
                        int64_t ro[JB];
                        double old[GB][JB];
#pragma unroll
                        for (int j = 0; j < JB; ++j) ro[j] = __shfl_sync(0xffffffffu, roff, (lane & ~7) | (j0 + j));
#pragma unroll
                        for (int gb = 0; gb < GB; ++gb) {
                            const bool col_ok = col0 + 8 * (g8 + gb) + (lane & 7) < nrhs;
#pragma unroll
                            for (int j = 0; j < JB; ++j)
                                old[gb][j] = (beta && col_ok && j0 + j < rows_ok) ? ycol[ro[j] + 8 * gb * ycs] : 0.0;
                        }
#pragma unroll
                        for (int gb = 0; gb < GB; ++gb) {
                            const bool col_ok = col0 + 8 * (g8 + gb) + (lane & 7) < nrhs;
#pragma unroll
                            for (int j = 0; j < JB; ++j)
                                if (col_ok && j0 + j < rows_ok) ycol[ro[j] + 8 * gb * ycs] = old[gb][j] + (double)x[gb][j0 + j];
                        }
                    }
                    ycol += 8 * GB * ycs;
                }
            } else if (t.out_kind == OUT_Y) {
                if (r < t.M) {
                    double *Yb = pa->Y + pa->yofs[t.c_row] + r;
#pragma unroll
                    for (int c0 = 0; c0 < C::COLS; c0 += C::RMW) {
                        double old[C::RMW];
#pragma unroll
                        for (int e = 0; e < C::RMW; ++e) {
                            const int cc = col0 + c0 + e;
                            old[e] = (beta && cc < nrhs) ? Yb[(size_t)cc * t.ldc] : 0.0;
                        }
#pragma unroll
                        for (int e = 0; e < C::RMW; ++e) {
                            const int cc = col0 + c0 + e;
                            if (cc < nrhs) Yb[(size_t)cc * t.ldc] = old[e] + (double)acc[c0 + e];
                        }
                    }
                }
            } else if (t.out_kind == OUT_F32) {
                if (r < t.M) {
                    float *Sb = pa->skel + t.c_row * (int64_t)nrhs + r;
#pragma unroll
                    for (int e = 0; e < C::COLS; ++e) {
                        const int cc = col0 + e;
                        if (cc < nrhs) Sb[(size_t)cc * t.ldc] = acc[e];
                    }
                }
            } else if (t.out_kind == OUT_SPLIT) {
                // no product: split one 128-column tile of a leaf's W block (FP64, leaf-blocked)
                // into 3-part operand tiles, every K tile of the leaf, as split_w_kernel does.
                // Columns past nrhs and points past M are zero.
                const int nt = un.col;
                const int KTv = (t.M + 63) / 64;
                const double *src = pa->W + pa->wofs[t.c_row];
                uint8_t *base = pa->buf[t.t_buf] + ((size_t)t.out_kt * pa->NT + (size_t)nt * KTv) * 3 * (size_t)TILE_BYTES;
                const int tid = threadIdx.x;  // the epilogue warps are warps 0 .. EPI_WARPS - 1
                constexpr int PER = 1024 / (C::EPI_WARPS * 32);  // 16-byte chunks per thread and K tile
                for (int kt = 0; kt < KTv; ++kt) {
                    // all of the thread's loads of the K tile in flight before any split
                    double x[PER][8];
#pragma unroll
                    for (int i = 0; i < PER; ++i) {
                        const int idx = tid + i * C::EPI_WARPS * 32;
                        const int c = idx % 8, n = nt * 128 + idx / 8;
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const int k = kt * 64 + c * 8 + e;
                            x[i][e] = (n < nrhs && k < t.M) ? src[k + (size_t)n * t.ldc] : 0.0;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < PER; ++i) {
                        const int idx = tid + i * C::EPI_WARPS * 32;
                        __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e) tc::split3(x[i][e], h[e], m[e], l[e]);
                        store_parts(base + (size_t)kt * 3 * TILE_BYTES, 3, idx / 8, idx % 8, h, m, l);
                    }
                }
            } else {
                // OUT_TILES: (optionally) add the FP32 far result, then write this row's values
                // as 3-part bf16 operand tiles.  The lane holds one K index; a transpose in
                // groups of 8 lanes gives it 8 consecutive K of one column: one 16-byte chunk
                // per part.  Rows past M carry zeros (A is zero-padded); rows past the node's
                // K tiles are not written.
                if (beta && r < t.M) {
                    const float *Sb = pa->skel + t.c_row * (int64_t)nrhs + r;
#pragma unroll
                    for (int c0 = 0; c0 < C::COLS; c0 += C::RMW) {
                        float old[C::RMW];
#pragma unroll
                        for (int e = 0; e < C::RMW; ++e) {
                            const int cc = col0 + c0 + e;
                            old[e] = cc < nrhs ? Sb[(size_t)cc * t.ldc] : 0.f;
                        }
#pragma unroll
                        for (int e = 0; e < C::RMW; ++e) acc[c0 + e] += old[e];
                    }
                }
                const int KTv = (t.M + 63) / 64;
                const int k0 = t.m0 + (int)rank * 128 + quarter * 32 + (lane & ~7);
                const bool k_ok = k0 < KTv * 64;
                const int kt = k0 >> 6;
                const uint32_t kin = (uint32_t)(k0 & 63);
                uint8_t *tbuf = pa->buf[t.t_buf];
                const int NT = pa->NT;
#pragma unroll
                for (int g8 = 0; g8 < C::COLS / 8; ++g8) {
                    float x[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) x[j] = acc[8 * g8 + j];
                    transpose8(x, lane);
                    const int n = col0 + 8 * g8 + (lane & 7);
                    uint4 vh, vm, vl;
                    tc::split3x8(x, vh, vm, vl);
                    if (k_ok) {
                        uint8_t *tile0 = tbuf + ((size_t)t.out_kt * NT + (size_t)(n >> 7) * KTv + kt) * 3 *
                                                    (size_t)TILE_BYTES;
                        const uint32_t o = tc::swizzled_offset(n & 127, (int)kin);
                        *reinterpret_cast<uint4 *>(tile0 + o) = vh;
                        *reinterpret_cast<uint4 *>(tile0 + TILE_BYTES + o) = vm;
                        *reinterpret_cast<uint4 *>(tile0 + 2 * TILE_BYTES + o) = vl;
                    }
                }
            }
            if (la.nlevels > 1) ++pend;  // counted when the warp moves past this level
            if (la.deps && un.sig >= 0) {
                // dataflow: this warp's part of the unit is written; count it for the units
                // that read it (the test hook keeps the units without inputs from counting)
                asm volatile("fence.proxy.async.global;\n" ::: "memory");
                __threadfence();
                __syncwarp();
                if (lane == 0 && !(la.stall_level && un.dep0 < 0)) atomicAdd(la.deps + un.sig, 1);
            }
        }
    }
    __syncwarp();
    __syncthreads();
    // all MMAs must be complete before TMEM is released (bounded, also after an abort)
    if (threadIdx.x == 0) {
        volatile int never = 0;
        if (!wait_x(doneb, 0, &never)) *abort_word = 1;
    }
    __syncthreads();
    if constexpr (PAIR) tc::cluster_sync();  // no traffic between the two CTAs after this point
    if (*abort_word && threadIdx.x == 0) atomicExch(la.err, MXB_ERR_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        if constexpr (PAIR) tc::tmem_dealloc_pair(tmem, C::TMEM_COLS);
        else tc::tmem_dealloc(tmem, C::TMEM_COLS);
    }
}

int g_sm_count[128];

int sm_count()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return 148;
    if (!g_sm_count[dev] && cudaDeviceGetAttribute(&g_sm_count[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return g_sm_count[dev];
}

template <int P, int BN, int S, bool PAIR, bool ORD>
cudaError_t configure_tc()
{
    static bool done[128];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(tc_gemm_kernel<P, BN, S, PAIR, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<P, BN, S, PAIR>::SMEM);
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

template <int P, int BN, int S, bool PAIR, bool ORD>
cudaError_t launch_tc_cfg(const LaunchArgs &a, cudaStream_t s)
{
    using C = TcCfg<P, BN, S, PAIR>;
    if (a.nunits <= 0) return cudaSuccess;
    cudaError_t e = configure_tc<P, BN, S, PAIR, ORD>();
    if (e != cudaSuccess) return e;
    if constexpr (!PAIR) {
        const int grid = std::min(a.nunits, sm_count());
        tc_gemm_kernel<P, BN, S, false, ORD><<<grid, C::THREADS, C::SMEM, s>>>(a);
        return cudaGetLastError();
    } else {
        const int pairs = std::min(a.nunits, std::max(1, sm_count() / 2));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(2 * pairs), 1, 1);
        cfg.blockDim = dim3(C::THREADS, 1, 1);
        cfg.dynamicSmemBytes = C::SMEM;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, tc_gemm_kernel<P, BN, S, true, ORD>, a);
    }
}

// Column-tile widths per product count; pipeline depth fills ~192-216 KiB of shared memory.
// A pair stages half of B per CTA, which buys a deeper pipeline at the same width.
template <bool ORD>
cudaError_t launch_tc_ord(int P, int BN, bool pair, const LaunchArgs &a, cudaStream_t s)
{
    if (pair) {
        if (P == 2)
            return BN == 256 ? launch_tc_cfg<2, 256, 3, true, ORD>(a, s) : launch_tc_cfg<2, 128, 4, true, ORD>(a, s);
        return BN == 256 ? launch_tc_cfg<3, 256, 2, true, ORD>(a, s) : launch_tc_cfg<3, 128, 3, true, ORD>(a, s);
    }
    if (P == 2) {
        if (BN == 256) return launch_tc_cfg<2, 256, 2, false, ORD>(a, s);
        if (BN == 128) return launch_tc_cfg<2, 128, 3, false, ORD>(a, s);
        return launch_tc_cfg<2, 64, 4, false, ORD>(a, s);
    }
    if (BN == 128) return launch_tc_cfg<3, 128, 2, false, ORD>(a, s);
    return launch_tc_cfg<3, 64, 3, false, ORD>(a, s);
}

// ord: the launch writes Y in the caller's point order (the instantiation with the scatter
// epilogue); every other launch runs the leaf-blocked one.
cudaError_t launch_tc(int P, int BN, bool pair, bool ord, const LaunchArgs &a, cudaStream_t s)
{
    return ord ? launch_tc_ord<true>(P, BN, pair, a, s) : launch_tc_ord<false>(P, BN, pair, a, s);
}

template <bool ORD>
cudaError_t configure_all_tc_ord()
{
    cudaError_t e = configure_tc<2, 256, 2, false, ORD>();
    if (e == cudaSuccess) e = configure_tc<2, 128, 3, false, ORD>();
    if (e == cudaSuccess) e = configure_tc<2, 64, 4, false, ORD>();
    if (e == cudaSuccess) e = configure_tc<3, 128, 2, false, ORD>();
    if (e == cudaSuccess) e = configure_tc<3, 64, 3, false, ORD>();
    if (e == cudaSuccess) e = configure_tc<2, 256, 3, true, ORD>();
    if (e == cudaSuccess) e = configure_tc<2, 128, 4, true, ORD>();
    if (e == cudaSuccess) e = configure_tc<3, 256, 2, true, ORD>();
    if (e == cudaSuccess) e = configure_tc<3, 128, 3, true, ORD>();
    return e;
}

cudaError_t configure_all_tc()
{
    cudaError_t e = configure_all_tc_ord<false>();
    return e == cudaSuccess ? configure_all_tc_ord<true>() : e;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Tile code of a tensor-core launch: column-tile width, plus MXB_TILE_PAIR when the launch
// runs on CTA pairs (256-row tiles).
int tile_width(int code) { return code & (MXB_TILE_PAIR - 1); }
bool tile_pair(int code) { return (code & MXB_TILE_PAIR) != 0; }

// Position of an op in the evaluation sequence; ops of different plans with the same key run
// in one launch.  W split, up-sweep by height, then the far couplings of every depth (they read
// only the finished up-sweep) together with the near field when both use the same product
// count, the downward transfers by depth, the near field otherwise, then leaf down.  Phase
// values are the MXB_PHASE_* codes of the profiling API.
enum OpPhase { PH_SPLITW = 0, PH_UP = 1, PH_FAR = 2, PH_DOWN = 3, PH_NEAR = 4, PH_LEAFDOWN = 5, PH_FARNEAR = 8 };
// The product count is part of the key of the coupling ops, so plans of different split modes
// (e.g. bf16x3 and bf16x6 far couplings) share a batch: their couplings run in separate
// launches of the same stage of the sequence.
int64_t op_key(int phase, int level, int P)
{
    switch (phase) {
    case PH_SPLITW: return 0;
    case PH_UP: return 1 + level;
    case PH_FAR:
    case PH_FARNEAR: return 1000000 + P;
    case PH_DOWN: return 2000000 + (int64_t)level;
    case PH_NEAR: return 3000000 + P;
    default: return 4000000;
    }
}

struct Op {             // one op of one plan
    int64_t key;
    int phase, level, P;
    int first, count;   // range in the plan's tasks (TC) or jobs (W split)
};

int batch_fail(const std::string &m, int code = MXB_ERR_ARG)
{
    set_error(m);
    return code;
}

}  // namespace

struct SplitBF16 {
    uint8_t *pool[NPOOL] = {};
    size_t pool_bytes[NPOOL] = {};
    std::vector<Op> ops;
    std::vector<Op> ops_adj;  // the transposed traversal (plans created with MXB_PLAN_ADJOINT)
    std::vector<TcTask> tasks;
    std::vector<TcItem> items;
    std::vector<SplitJob> jobs;
    std::vector<int64_t> leaf_kt, node_kt;  // K-tile bases
    int64_t leaf_kt_total = 0, node_kt_total = 0;
    int nt_cap = 0, nrhs_cap = 0;
    int buf_gen = 0;  // counts reallocations of the buffers below (graphs hold their addresses)
    uint8_t *Wt = nullptr, *wT = nullptr, *uT = nullptr;
    float *u32 = nullptr;  // FP32 far results awaiting the down launch
    int *dErr = nullptr;
    Batch *self = nullptr;      // the single-plan batch used by mxb_plan_evaluate
    Batch *self_adj = nullptr;  // the same for mxb_plan_adjoint
};

// ---------------------------------------------------------------------------------------
// batch: merged launch sequence of several split-BF16 plans
// ---------------------------------------------------------------------------------------

struct Batch : public mxb_batch {
    std::vector<Plan *> plans;
    struct MOp {
        int64_t key;
        int phase, level, P;
        int first, count;  // range in the merged tasks or jobs
        int max_kt;
        int max_m;         // tallest output block (pairs only pay off above 128 rows)
        bool writes_y;     // some task writes Y (the launch scatters rows in caller order)
    };
    std::vector<MOp> ops;
    std::vector<TcTask> tasks;
    std::vector<TcItem> items;
    // One-launch mode: the W split and every tensor-core op run as the levels of a single
    // launch of the kernel with 3-part stages (OUT_SPLIT tasks at [split_task0, + split_tasks)).
    bool one_launch = false;
    int split_task0 = 0, split_tasks = 0;
    unsigned long long *level_ns = nullptr;  // while profiling a one-launch evaluation
    std::vector<SplitJob> jobs;
    TcTask *dTasks = nullptr;
    TcItem *dItems = nullptr;
    SplitJob *dJobs = nullptr;
    int *dNext = nullptr;  // work-unit counter per op
    int *dLevel = nullptr; // per op: epilogue warps done with its units (chained launches)
    std::vector<void *> allocations;
    struct Entry {                     // one captured evaluation
        std::vector<const double *> W;
        std::vector<double *> Y;
        std::vector<int> nrhs;
        int accumulate = 0;
        int debug_flags = 0;
        std::vector<int> bn;           // column-tile width per op (0 for the W split)
        std::vector<CallerOrder> order;  // per plan, when W / Y are in the caller's point order
        PlanArgs *dPlans = nullptr;
        TcUnit *dUnits = nullptr;
        std::vector<int> unit_first, unit_count;
        // dataflow launches: per op, whether its chained launch waits on node counters (the
        // counters of every such launch in one array, zeroed before each evaluation)
        std::vector<char> dataflow;
        int *dDeps = nullptr;
        int ndeps = 0;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<Entry> entries;
    std::map<std::vector<int>, std::vector<int>> tuned;  // nrhs signature -> bn per op
    // buffer generation of each plan when the entries were captured: another batch of the same
    // plan (its own single-plan batch, its adjoint's, a user batch) may have reallocated them
    std::vector<int> buf_gens;
    cudaStream_t capture_stream = nullptr;
    int device = 0;

    ~Batch() override
    {
        clear();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        for (void *p : allocations) cudaFree(p);
    }
    static void release(Entry &e)
    {
        if (e.exec) cudaGraphExecDestroy(e.exec);
        if (e.dPlans) cudaFree(e.dPlans);
        if (e.dUnits) cudaFree(e.dUnits);
        if (e.dDeps) cudaFree(e.dDeps);
        e.exec = nullptr;
        e.dPlans = nullptr;
        e.dUnits = nullptr;
        e.dDeps = nullptr;
        e.ndeps = 0;
    }
    void clear()
    {
        for (Entry &e : entries) release(e);
        entries.clear();
    }
    int build(const std::vector<Plan *> &ps, bool adjoint = false);
    int evaluate(const double *const *W, double *const *Y, const int *nrhs, int accumulate, cudaStream_t stream,
                 int debug_flags, long long wait_cycles, const CallerOrder *order = nullptr);
    int enqueue(Entry &e, cudaStream_t stream, int debug_flags, long long wait_cycles, const std::vector<int> &bn,
                int only_op = -1);
    int units_for(Entry &e, const std::vector<int> &bn, cudaStream_t stream);
    int dataflow_units(const Entry &e, size_t k, size_t end, const std::vector<int> &bn, std::vector<TcUnit> &units,
                       int &ndeps) const;
    void chain_all(std::vector<int> &bn) const;
    int tune(Entry &e, std::vector<PlanArgs> pa, std::vector<int> &bn, cudaStream_t stream, long long wait_cycles);
    int tune_one_launch(Entry &e, std::vector<PlanArgs> pa, std::vector<int> &bn, cudaStream_t stream,
                        long long wait_cycles);
    Entry *find(const double *const *W, double *const *Y, const std::vector<int> &nr, int accumulate,
                int debug_flags, const CallerOrder *order = nullptr);
    int profile(const double *const *W, double *const *Y, const int *nrhs, cudaStream_t stream, mxb_op_profile *out,
                int cap, int *nops);
};

int Batch::build(const std::vector<Plan *> &ps, bool adjoint)
{
    if (ps.empty()) return batch_fail("empty batch");
    plans = ps;
    MXB_CUDA_OR(cudaGetDevice(&device));
    for (Plan *p : ps) {
        // any mix of split modes: the ops whose product counts differ run in separate launches
        if (!p || !p->bf16) return batch_fail("batches take split-BF16 plans");
        if (p->device != device) return batch_fail("all plans of a batch must live on the current device");
    }
    // merge ops by key, in key order; tasks and jobs get their plan index and offsets
    std::map<int64_t, std::vector<std::pair<int, const Op *>>> by_key;
    for (int pi = 0; pi < (int)ps.size(); ++pi) {
        if (adjoint && ps[pi]->bf16->ops_adj.empty()) return batch_fail("the plan has no split-BF16 adjoint");
        for (const Op &o : adjoint ? ps[pi]->bf16->ops_adj : ps[pi]->bf16->ops) by_key[o.key].push_back({pi, &o});
    }
    for (auto &kv : by_key) {
        MOp m{};
        m.key = kv.first;
        const Op *o0 = kv.second[0].second;
        m.phase = o0->phase;
        m.level = o0->level;
        m.P = o0->P;
        m.max_kt = 1;
        m.max_m = 0;
        if (m.phase == PH_SPLITW) {
            m.first = (int)jobs.size();
            for (auto &po : kv.second) {
                const SplitBF16 &S = *ps[po.first]->bf16;
                for (int j = po.second->first; j < po.second->first + po.second->count; ++j) {
                    SplitJob sj = S.jobs[j];
                    sj.plan = po.first;
                    m.max_kt = std::max(m.max_kt, sj.KT);
                    jobs.push_back(sj);
                }
            }
            m.count = (int)jobs.size() - m.first;
        } else {
            m.first = (int)tasks.size();
            for (auto &po : kv.second) {
                const SplitBF16 &S = *ps[po.first]->bf16;
                if (po.second->P != m.P) return batch_fail("plans disagree on a launch's product count");
                for (int j = po.second->first; j < po.second->first + po.second->count; ++j) {
                    TcTask t = S.tasks[j];
                    const int item0 = (int)items.size();
                    for (int q = 0; q < t.nitem; ++q) items.push_back(S.items[t.item0 + q]);
                    t.item0 = item0;
                    t.plan = po.first;
                    m.max_m = std::max(m.max_m, t.M);
                    m.writes_y |= t.out_kind == OUT_Y;
                    tasks.push_back(t);
                }
            }
            m.count = (int)tasks.size() - m.first;
            // longest tasks first: the kernel's CTAs claim units in this order (list scheduling)
            auto cost = [&](const TcTask &t) {
                int k = 0;
                for (int q = 0; q < t.nitem; ++q) k += items[t.item0 + q].KT;
                return k;
            };
            std::stable_sort(tasks.begin() + m.first, tasks.end(),
                             [&](const TcTask &a, const TcTask &b) { return cost(a) > cost(b); });
        }
        if (m.count > 0) ops.push_back(m);
    }
    // the W split as tasks of the tensor-core kernel, for the one-launch mode
    split_task0 = (int)tasks.size();
    for (const MOp &m : ops) {
        if (m.phase != PH_SPLITW) continue;
        for (int j = m.first; j < m.first + m.count; ++j) {
            const SplitJob &sj = jobs[j];
            TcTask t{};
            t.c_row = sj.src_row;
            t.out_kt = sj.dst_kt;
            t.ldc = sj.ld;
            t.M = sj.K;
            t.plan = sj.plan;
            t.out_kind = OUT_SPLIT;
            t.t_buf = BUF_W;
            tasks.push_back(t);
        }
    }
    split_tasks = (int)tasks.size() - split_task0;
    auto up = [&](void **dst, const void *src, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(dst, std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) return batch_fail(std::string("batch allocation: ") + cudaGetErrorString(e), MXB_ERR_NOMEM);
        allocations.push_back(*dst);
        if (bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return batch_fail(std::string("batch upload: ") + cudaGetErrorString(e), MXB_ERR_CUDA);
        return MXB_OK;
    };
    int rc = up((void **)&dTasks, tasks.data(), tasks.size() * sizeof(TcTask));
    if (!rc) rc = up((void **)&dItems, items.data(), items.size() * sizeof(TcItem));
    if (!rc) rc = up((void **)&dJobs, jobs.data(), jobs.size() * sizeof(SplitJob));
    if (!rc) {
        cudaError_t e = cudaMalloc(&dNext, 2 * std::max<size_t>(ops.size(), 1) * sizeof(int));
        if (e != cudaSuccess) return batch_fail(std::string("batch allocation: ") + cudaGetErrorString(e), MXB_ERR_NOMEM);
        allocations.push_back(dNext);
        dLevel = dNext + std::max<size_t>(ops.size(), 1);
    }
    // synchronous copies from pageable memory may return before their DMA lands, and the
    // evaluations run on streams that do not wait for the legacy stream
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = batch_fail("batch upload: synchronisation failed", MXB_ERR_CUDA);
    return rc;
}

// Runs of consecutive up-sweep ops, and of down-sweep ops with leaf down, that share a product
// count and a tile; "family" 1 and 2, 0 for every other op.
int chain_family(int phase) { return phase == PH_UP ? 1 : (phase == PH_DOWN || phase == PH_LEAFDOWN) ? 2 : 0; }

void Batch::chain_all(std::vector<int> &bn) const
{
    for (size_t k = 0; k < ops.size();) {
        const int fam = chain_family(ops[k].phase);
        size_t j = k + 1;
        while (fam && j < ops.size() && chain_family(ops[j].phase) == fam && ops[j].P == ops[k].P &&
               (bn[j] & ~TILE_CHAIN) == (bn[k] & ~TILE_CHAIN) && j - k < (size_t)MAX_CHAIN)
            ++j;
        for (size_t q = k + 1; q < j; ++q) bn[q] |= TILE_CHAIN;
        k = j;
    }
}

// Bytes of A tiles per group of coupling tasks in the unit order (0: longest task first, all
// column tiles of a task together).  MXB_UNIT_GROUP_MB overrides the default.
int64_t unit_group_bytes()
{
    static const int64_t v = [] {
        const char *e = getenv("MXB_UNIT_GROUP_MB");
        return (int64_t)((e && *e) ? atof(e) : 0.0) * (1 << 20);
    }();
    return v;
}

// MXB_TC_DATAFLOW=0 keeps chained launches on level barriers (read when an evaluation graph is
// built).
bool dataflow_enabled()
{
    const char *e = getenv("MXB_TC_DATAFLOW");
    return !(e && *e == '0');
}

// A node of a chained sweep: the tasks of one output block (its row tiles).
struct DfNode {
    int plan = 0, level = 0;
    int64_t key = 0;         // tile K base of the output (OUT_TILES) or leaf index (OUT_Y)
    std::vector<int> tasks;  // tasks that carry units (row tiles; the even one of a pair)
    std::vector<int> dep;    // nodes whose output tiles this node reads
    std::vector<int> cons;   // nodes that read this node's output tiles
    int ncol = 0, kt = 0, ctr = -1, order = 0, unplaced = 0;
    double ready = 0, finish = 0;
};

// The dataflow order of a run's nodes (their dep lists filled): depth-first order over the tree,
// counters from `ndeps` on, and the list-scheduling simulation that emits the units (the scheme
// is described at Batch::dataflow_units).  unit_node, if given, receives the node of every emitted unit.
// Returns 1, 0 where the dependencies are not a tree (nothing emitted), or an error code.
int dataflow_schedule(std::vector<DfNode> &nodes, int workers, std::vector<TcUnit> &units, int &ndeps,
                      std::vector<int> *unit_node = nullptr)
{
    for (const DfNode &nd : nodes)
        if (nd.tasks.empty() || nd.dep.size() > 2 || nd.tasks.size() > 0xFFFF) return 0;
    for (DfNode &nd : nodes) nd.cons.clear();
    for (int n = 0; n < (int)nodes.size(); ++n)
        for (int wn : nodes[n].dep) {
            if (wn < 0 || wn >= (int)nodes.size() || wn == n) return 0;
            nodes[wn].cons.push_back(n);
        }
    bool in_tree = true, out_tree = true;
    for (const DfNode &nd : nodes) {
        in_tree &= nd.cons.size() <= 1;
        out_tree &= nd.dep.size() <= 1;
    }
    if (!in_tree && !out_tree) return 0;

    // depth-first order: children before parents (up sweep), parents before children (down)
    auto tree_less = [&](int a, int b) {
        return std::tie(nodes[a].plan, nodes[a].level, nodes[a].key) < std::tie(nodes[b].plan, nodes[b].level, nodes[b].key);
    };
    int next = 0;
    std::vector<int> roots;
    for (int n = 0; n < (int)nodes.size(); ++n)
        if (in_tree ? nodes[n].cons.empty() : nodes[n].dep.empty()) roots.push_back(n);
    std::sort(roots.begin(), roots.end(), tree_less);
    std::vector<char> seen(nodes.size(), 0);
    bool cyclic = false;
    std::function<void(int)> visit = [&](int n) {
        if (seen[n]) {
            cyclic = true;
            return;
        }
        seen[n] = 1;
        std::vector<int> ch = in_tree ? nodes[n].dep : nodes[n].cons;
        std::sort(ch.begin(), ch.end(), tree_less);
        if (!in_tree) nodes[n].order = next++;
        for (int c : ch) visit(c);
        if (in_tree) nodes[n].order = next++;
    };
    for (int r : roots) visit(r);
    if (cyclic || next != (int)nodes.size()) return 0;

    for (DfNode &nd : nodes)
        if (!nd.cons.empty()) {
            nd.ctr = ndeps;
            ndeps += nd.ncol;
        }

    // list scheduling (simulated, time in K tiles): one worker per CTA (pair), which claims its
    // next unit once it has issued the last loads of the current one, i.e. about STAGES K
    // tiles before the current unit's MMAs end -- a unit claimed before its inputs are written
    // holds its CTA until they are
    struct Cta {
        double claim, mma_free;
        bool operator>(const Cta &o) const { return claim > o.claim; }
    };
    std::priority_queue<Cta, std::vector<Cta>, std::greater<Cta>> ctas;
    for (int i = 0; i < std::max(1, workers); ++i) ctas.push(Cta{0.0, 0.0});
    constexpr double STAGES_KT = 2.0;
    auto later_order = [&](int a, int b) { return nodes[a].order > nodes[b].order; };
    auto later_ready = [&](int a, int b) { return nodes[a].ready > nodes[b].ready; };
    std::priority_queue<int, std::vector<int>, decltype(later_order)> ready(later_order);
    std::priority_queue<int, std::vector<int>, decltype(later_ready)> waiting(later_ready);
    for (int n = 0; n < (int)nodes.size(); ++n) {
        nodes[n].ready = nodes[n].finish = 0;
        nodes[n].unplaced = (int)nodes[n].dep.size();
        if (!nodes[n].unplaced) waiting.push(n);
    }
    for (size_t placed = 0; placed < nodes.size(); ++placed) {
        const double now = ctas.top().claim;
        while (!waiting.empty() && nodes[waiting.top()].ready <= now) {
            ready.push(waiting.top());
            waiting.pop();
        }
        int g;
        if (!ready.empty()) {
            g = ready.top();
            ready.pop();
        } else if (!waiting.empty()) {
            g = waiting.top();  // nothing ready: the node whose inputs finish first
            waiting.pop();
        } else {
            return batch_fail("dataflow schedule: a node's inputs are never written");
        }
        DfNode &nd = nodes[g];
        int need = 0;
        for (size_t d = 0; d < nd.dep.size(); ++d) need |= (int)nodes[nd.dep[d]].tasks.size() << (16 * d);
        for (int c = 0; c < nd.ncol; ++c)
            for (int t : nd.tasks) {
                Cta w = ctas.top();
                ctas.pop();
                const double load = std::max(w.claim, nd.ready);  // the producer waits for inputs
                const double mma = std::max(load + 1.0, w.mma_free);
                w.mma_free = mma + nd.kt;
                w.claim = std::max(load, mma + std::max(0.0, nd.kt - STAGES_KT));
                ctas.push(w);
                nd.finish = std::max(nd.finish, mma + nd.kt + 1.0);
                TcUnit u{};
                u.task = t;
                u.col = c;
                u.ktiles = nd.kt;
                u.chain = 0;
                u.dep0 = nd.dep.size() > 0 ? nodes[nd.dep[0]].ctr + c : -1;
                u.dep1 = nd.dep.size() > 1 ? nodes[nd.dep[1]].ctr + c : -1;
                u.need = need;
                u.sig = nd.ctr >= 0 ? nd.ctr + c : -1;
                units.push_back(u);
                if (unit_node) unit_node->push_back(g);
            }
        for (int cn : nd.cons) {
            DfNode &cd = nodes[cn];
            cd.ready = std::max(cd.ready, nd.finish);
            if (--cd.unplaced == 0) waiting.push(cn);
        }
    }
    return 1;
}

// Dataflow schedule of a chained run of sweep ops [k, end): the up-sweep heights, or the
// down-sweep depths with leaf down.  A node (the tasks of one output block: its row tiles)
// depends on the nodes of earlier levels of the run whose output tiles its items read, and
// each of its units waits, for its own column tile only, until those nodes' units have written
// them -- instead of waiting for the whole level before.  The dependencies of a sweep form a
// tree: up-sweep nodes read their two children, down-sweep nodes (and leaf down) their parent.
//
// The unit order comes from a list-scheduling simulation of the launch (one worker per CTA or
// CTA pair, time in K tiles): whenever a worker claims, the next node is the
// ready one (inputs finished in the simulation) that comes first in a depth-first order of the
// tree -- post-order for the up sweep, pre-order for the down sweep -- with all its units
// (column tile by column tile).  So a parent runs soon after its children while their tiles
// are still in L2, a node's column tiles run together (its A tiles are read from DRAM once),
// and the short top levels of one subtree overlap the wide lower levels of the next.  Every
// unit's inputs come earlier in the list, and units are claimed in list order, so the waits
// always end.
//
// Appends the run's units and returns 1; returns 0 (nothing appended) where the dependencies
// are not a tree or a node reads tiles that its own or a later level writes, and the run then
// keeps its level barriers.  Counters are allocated from `ndeps` on.
int Batch::dataflow_units(const Entry &e, size_t k, size_t end, const std::vector<int> &bn, std::vector<TcUnit> &units,
                          int &ndeps) const
{
    const bool pair = tile_pair(bn[k]);
    const int w = tile_width(bn[k]);
    std::vector<DfNode> nodes;
    std::map<std::tuple<int, int, int64_t>, int> by_out;  // (plan, tile buffer or -1 for Y, key)
    for (size_t q = k; q < end; ++q) {
        const MOp &m = ops[q];
        if (m.phase == PH_SPLITW) return 0;
        for (int t = m.first; t < m.first + m.count; ++t) {
            const TcTask &tk = tasks[t];
            if (tk.out_kind != OUT_TILES && tk.out_kind != OUT_Y) return 0;
            const auto id = std::make_tuple((int)tk.plan, tk.out_kind == OUT_TILES ? (int)tk.t_buf : -1,
                                            tk.out_kind == OUT_TILES ? tk.out_kt : tk.c_row);
            auto it = by_out.find(id);
            int n;
            if (it == by_out.end()) {
                n = (int)nodes.size();
                by_out[id] = n;
                DfNode nd;
                nd.plan = tk.plan;
                nd.level = (int)q;
                nd.key = std::get<2>(id);
                nd.ncol = (int)ceil_div(e.nrhs[tk.plan], w);
                nodes.push_back(nd);
            } else {
                n = it->second;
                if (nodes[n].level != (int)q) return 0;  // one output written at two levels
            }
            if (pair && tk.m0 % 256) continue;  // the pair's odd CTA takes rows m0 + 128
            nodes[n].tasks.push_back(t);
        }
    }
    for (int n = 0; n < (int)nodes.size(); ++n) {
        DfNode &nd = nodes[n];
        if (nd.tasks.empty()) return 0;
        const TcTask &t0 = tasks[nd.tasks[0]];
        for (int q = t0.item0; q < t0.item0 + t0.nitem; ++q) nd.kt += items[q].KT;
        for (int t : nd.tasks) {
            const TcTask &tk = tasks[t];
            for (int q = tk.item0; q < tk.item0 + tk.nitem; ++q) {
                auto it = by_out.find(std::make_tuple(nd.plan, (int)items[q].b_buf, items[q].b_base));
                if (it == by_out.end()) continue;  // written before this launch
                const int wn = it->second;
                if (nodes[wn].level >= nd.level) return 0;
                if (std::find(nd.dep.begin(), nd.dep.end(), wn) == nd.dep.end()) nd.dep.push_back(wn);
            }
        }
    }
    return dataflow_schedule(nodes, pair ? sm_count() / 2 : sm_count(), units, ndeps);
}

// Work units of every TC op for this entry's nrhs and column-tile choices.
// The list is uploaded on `stream`, ahead of the launches that read it.
int Batch::units_for(Entry &e, const std::vector<int> &bn, cudaStream_t stream)
{
    std::vector<TcUnit> units;
    e.unit_first.assign(ops.size(), 0);
    e.unit_count.assign(ops.size(), 0);
    if (one_launch) {
        // level k = op k: the W split (one unit per leaf and 128-column tile), then every
        // tensor-core op in sequence, each unit tagged with its operand parts
        if (ops.size() > (size_t)MAX_CHAIN) return batch_fail("too many levels for one launch");
        for (size_t k = 0; k < ops.size(); ++k) {
            const MOp &m = ops[k];
            e.unit_first[k] = (int)units.size();
            const int prev = k ? e.unit_count[k - 1] : 0;
            if (prev > 0xFFFFF) return batch_fail("a level of the one-launch evaluation has too many units");
            const int32_t chain = ((int32_t)k << 20) | prev;
            if (m.phase == PH_SPLITW) {
                // the 128-column tiles that the launch's units read (its tile is 64 or 128 wide)
                for (int t = split_task0; t < split_task0 + split_tasks; ++t) {
                    const int NT = (int)ceil_div(e.nrhs[tasks[t].plan], 128);
                    for (int nt = 0; nt < NT; ++nt) units.push_back(TcUnit{t, nt, 0, chain | (3 << 28)});
                }
            } else {
                const int w = tile_width(bn[k]);
                for (int t = m.first; t < m.first + m.count; ++t) {
                    int kt = 0;
                    for (int q = tasks[t].item0; q < tasks[t].item0 + tasks[t].nitem; ++q) kt += items[q].KT;
                    const int ncol = (int)ceil_div(e.nrhs[tasks[t].plan], w);
                    for (int c = 0; c < ncol; ++c) units.push_back(TcUnit{t, c, kt, chain | (m.P << 28)});
                }
            }
            e.unit_count[k] = (int)units.size() - e.unit_first[k];
        }
    }
    e.dataflow.assign(ops.size(), 0);
    int ndeps = 0;
    for (size_t k = 0; k < ops.size() && !one_launch; ++k) {
        const MOp &m = ops[k];
        e.unit_first[k] = (int)units.size();
        if (m.phase == PH_SPLITW) continue;
        if (!(bn[k] & TILE_CHAIN) && dataflow_enabled()) {
            // a chain head: its run waits on node counters where the sweep's dependencies allow
            size_t end = k + 1;
            while (end < ops.size() && ops[end].phase != PH_SPLITW && (bn[end] & TILE_CHAIN)) ++end;
            if (end - k >= 2) {
                const int r = dataflow_units(e, k, end, bn, units, ndeps);
                if (r < 0) return r;
                if (r == 1) {
                    e.dataflow[k] = 1;
                    e.unit_count[k] = (int)units.size() - e.unit_first[k];
                    for (size_t q = k + 1; q < end; ++q) e.unit_first[q] = (int)units.size();
                    k = end - 1;
                    continue;
                }
            }
        }
        const bool pair = tile_pair(bn[k]);
        // level of this op in its chained launch, and the units of the level before it
        int level = 0;
        for (size_t h = k; h > 0 && (bn[h] & TILE_CHAIN) && ops[h - 1].phase != PH_SPLITW; --h) ++level;
        if (level >= MAX_CHAIN || (level && e.unit_count[k - 1] > 0xFFFFF))
            return batch_fail("a chained launch exceeds its level or unit limits");
        const int32_t chain = level ? (level << 20) | e.unit_count[k - 1] : 0;
        auto task_kt = [&](int t) {
            int kt = 0;
            for (int q = tasks[t].item0; q < tasks[t].item0 + tasks[t].nitem; ++q) kt += items[q].KT;
            return kt;
        };
        auto ncol_of = [&](int t) { return (int)ceil_div(e.nrhs[tasks[t].plan], tile_width(bn[k])); };
        const int64_t group_bytes = unit_group_bytes();
        if (group_bytes > 0 && (m.phase == PH_FARNEAR || m.phase == PH_FAR || m.phase == PH_NEAR)) {
            // Coupling launches read each task's A tiles (CDS blocks) for every column tile and
            // share the B tiles (W / skeleton slabs) among the tasks of neighbouring nodes.
            // Tasks in tree order form groups whose A tiles fit in a slice of L2; a group
            // sweeps its column tiles one after the other (all its tasks at column tile 0,
            // then 1, ...), so its A tiles come from DRAM once and the in-flight units of one
            // column tile share their B tiles.  Groups run heaviest first.
            std::vector<int> ord;
            for (int t = m.first; t < m.first + m.count; ++t)
                if (!(pair && tasks[t].m0 % 256)) ord.push_back(t);
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
                const TcTask &x = tasks[a], &y = tasks[b];
                if (x.plan != y.plan) return x.plan < y.plan;
                if (x.out_kind != y.out_kind) return x.out_kind < y.out_kind;
                if (x.c_row != y.c_row) return x.c_row < y.c_row;
                return x.m0 < y.m0;
            });
            std::vector<std::pair<int64_t, std::vector<int>>> groups;  // (cost, tasks)
            int64_t bytes = 0;
            for (int t : ord) {
                const int kt = task_kt(t);
                const int64_t a = (int64_t)kt * m.P * TILE_BYTES * (pair ? 2 : 1);
                if (groups.empty() || bytes + a > group_bytes) {
                    groups.push_back({0, {}});
                    bytes = 0;
                }
                groups.back().second.push_back(t);
                groups.back().first += (int64_t)kt * ncol_of(t);
                bytes += a;
            }
            std::stable_sort(groups.begin(), groups.end(),
                             [](const auto &a, const auto &b) { return a.first > b.first; });
            for (const auto &g : groups) {
                int maxc = 0;
                for (int t : g.second) maxc = std::max(maxc, ncol_of(t));
                for (int c = 0; c < maxc; ++c)
                    for (int t : g.second)
                        if (c < ncol_of(t)) units.push_back(TcUnit{t, c, task_kt(t), chain});
            }
        } else {
            for (int t = m.first; t < m.first + m.count; ++t) {
                if (pair && tasks[t].m0 % 256) continue;  // the pair's odd CTA takes rows m0 + 128
                const int ncol = ncol_of(t);
                const int kt = task_kt(t);
                for (int c = 0; c < ncol; ++c) units.push_back(TcUnit{t, c, kt, chain});
            }
        }
        e.unit_count[k] = (int)units.size() - e.unit_first[k];
    }
    if (e.dUnits) cudaFree(e.dUnits);
    e.dUnits = nullptr;
    if (e.dDeps) cudaFree(e.dDeps);
    e.dDeps = nullptr;
    e.ndeps = ndeps;
    if (ndeps) {
        const cudaError_t derr = cudaMalloc(&e.dDeps, (size_t)ndeps * sizeof(int));
        if (derr != cudaSuccess) return batch_fail(std::string("node counters: ") + cudaGetErrorString(derr), MXB_ERR_NOMEM);
    }
    cudaError_t err = cudaMalloc(&e.dUnits, std::max<size_t>(units.size(), 1) * sizeof(TcUnit));
    if (err == cudaSuccess && !units.empty())
        err = cudaMemcpyAsync(e.dUnits, units.data(), units.size() * sizeof(TcUnit), cudaMemcpyHostToDevice, stream);
    if (err != cudaSuccess) return batch_fail(std::string("work units: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
    return MXB_OK;
}

namespace {
int kchain_for(int P);
}


int Batch::enqueue(Entry &e, cudaStream_t stream, int debug_flags, long long wait_cycles, const std::vector<int> &bn,
                   int only_op)
{
    bool first_tc = true;
    int maxnt = 0;
    for (Plan *p : plans) maxnt = std::max(maxnt, p->bf16->nt_cap);
    // work-unit and level counters of the tensor-core launches start at zero (both arrays in
    // one allocation: dLevel follows dNext)
    const size_t nops = std::max<size_t>(ops.size(), 1);
    cudaError_t zerr = cudaMemsetAsync(dNext, 0, 2 * nops * sizeof(int), stream);
    if (zerr == cudaSuccess && e.ndeps && (only_op < 0 || (only_op < (int)e.dataflow.size() && e.dataflow[only_op])))
        zerr = cudaMemsetAsync(e.dDeps, 0, (size_t)e.ndeps * sizeof(int), stream);
    if (zerr != cudaSuccess) return batch_fail(std::string("work-unit counters: ") + cudaGetErrorString(zerr), MXB_ERR_CUDA);
    if (one_launch) {
        // every op is a level of the launch of op 0 (profiling asks for op 0 to time it)
        if (only_op > 0) return MXB_OK;
        int w = 128;
        for (size_t k = 0; k < ops.size(); ++k)
            if (ops[k].phase != PH_SPLITW) {
                w = tile_width(bn[k]) >= 128 ? 128 : 64;
                break;
            }
        LaunchArgs a{};
        a.plans = e.dPlans;
        a.tasks = dTasks;
        a.items = dItems;
        a.units = e.dUnits;
        a.nunits = 0;
        for (int c : e.unit_count) a.nunits += c;
        a.next_unit = dNext;
        a.err = plans[0]->bf16->dErr;
        a.wait_cycles = wait_cycles > 0 ? wait_cycles : tc::WAIT_CYCLES;
        a.stall_test = (debug_flags & MXB_DEBUG_STALL_ONE_WAIT) != 0;
        a.kchain = kchain_for(3);
        a.nlevels = (int)ops.size();
        a.level_done = dLevel;
        a.stall_level = (debug_flags & MXB_DEBUG_STALL_LEVEL) != 0;
        a.level_ns = level_ns;
        const cudaError_t err = launch_tc(3, w, false, false, a, stream);
        if (err != cudaSuccess) return batch_fail(std::string("one-launch evaluation: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
        return MXB_OK;
    }
    for (size_t k = 0; k < ops.size(); ++k) {
        const MOp &m = ops[k];
        const bool run = only_op < 0 || (int)k == only_op;
        cudaError_t err = cudaSuccess;
        if (m.phase != PH_SPLITW && (bn[k] & TILE_CHAIN)) continue;  // runs in its chain head's launch
        if (m.phase == PH_SPLITW) {
            if (run) {
                if (e.order.empty())
                    split_w_kernel<false><<<dim3(m.count, m.max_kt, maxnt), 256, 0, stream>>>(dJobs + m.first, e.dPlans);
                else
                    split_w_kernel<true><<<dim3(m.count, m.max_kt, maxnt), 256, 0, stream>>>(dJobs + m.first, e.dPlans);
                err = cudaGetLastError();
            }
        } else {
            if (run) {
                LaunchArgs a{};
                a.plans = e.dPlans;
                a.tasks = dTasks;
                a.items = dItems;
                a.units = e.dUnits + e.unit_first[k];
                a.nunits = e.unit_count[k];
                a.next_unit = dNext + k;
                a.err = plans[0]->bf16->dErr;
                a.wait_cycles = wait_cycles > 0 ? wait_cycles : tc::WAIT_CYCLES;
                a.stall_test = (debug_flags & MXB_DEBUG_STALL_ONE_WAIT) && first_tc;
                a.kchain = kchain_for(m.P);
                // the ops chained to this one (same product count and tile) run as later levels
                bool writes_y = m.writes_y;
                size_t end = k + 1;
                while (end < ops.size() && ops[end].phase != PH_SPLITW && (bn[end] & TILE_CHAIN))
                    writes_y |= ops[end++].writes_y;
                if (end - k > (size_t)MAX_CHAIN) return batch_fail("a chained launch has too many levels");
                a.nlevels = (int)(end - k);
                a.level_done = dLevel + k;
                if (k < e.dataflow.size() && e.dataflow[k]) {
                    a.nlevels = 1;  // node counters instead of level barriers
                    a.deps = e.dDeps;
                }
                a.stall_level = (debug_flags & MXB_DEBUG_STALL_LEVEL) != 0;
                        int total = 0;
                for (size_t j = k; j < end; ++j) total += e.unit_count[j];
                a.nunits = total;
                err = launch_tc(m.P, tile_width(bn[k]), tile_pair(bn[k]), writes_y && !e.order.empty(), a, stream);
            }
            first_tc = false;
        }
        if (err != cudaSuccess) return batch_fail(std::string("split-BF16 launch: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
    }
    return MXB_OK;
}

namespace {

int split_buffers(Plan &p, SplitBF16 &S, int nrhs)
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
    ++S.buf_gen;
    return MXB_OK;
}

// Default column tile: the widest that the right-hand sides fill.
int default_bn(int P, int nrhs_max)
{
    if (P == 2) return nrhs_max > 128 ? 256 : (nrhs_max > 64 ? 128 : 64);
    return nrhs_max > 64 ? 128 : 64;
}

// MXB_TC_TILE=<code> runs every tensor-core launch with that tile (width, + MXB_TILE_PAIR for
// pairs), mapped to the nearest variant the launch's product count has; read when an
// evaluation graph is built.  For tests that must reach one kernel variant.
int forced_tile(int P)
{
    const char *e = getenv("MXB_TC_TILE");
    const int code = e && *e ? atoi(e) : 0;
    if (code <= 0) return 0;
    const int w = tile_width(code);
    if (tile_pair(code)) return (w >= 256 ? 256 : 128) | MXB_TILE_PAIR;
    if (P == 2) return w >= 256 ? 256 : (w >= 128 ? 128 : 64);
    return w >= 128 ? 128 : 64;
}

// K tiles per accumulator fill: 2 for bf16x3 products, 1 for bf16x6 (MXB_TC_KCHAIN overrides).
int kchain_for(int P)
{
    static const int forced = [] {
        const char *e = getenv("MXB_TC_KCHAIN");
        const int k = e && *e ? atoi(e) : 0;
        return k == 1 || k == 2 ? k : 0;
    }();
    return forced ? forced : (P == 2 ? 2 : 1);
}

// MXB_TC_PAIRS=0 keeps the autotuner to single-CTA launches.
bool pairs_enabled()
{
    static const bool on = [] {
        const char *e = getenv("MXB_TC_PAIRS");
        return !(e && *e == '0');
    }();
    return on;
}

// MXB_TC_CHAIN=0 keeps every tree level in a launch of its own; MXB_TC_CHAIN=2 chains every run
// of sweep levels that share a product count and a tile, without timing the alternatives (read
// when an evaluation graph is built).
bool chains_enabled()
{
    const char *e = getenv("MXB_TC_CHAIN");
    return !(e && *e == '0');
}
bool chains_forced()
{
    const char *e = getenv("MXB_TC_CHAIN");
    return e && *e == '2';
}

// MXB_AUTOTUNE=0 keeps the default tiles (read when an evaluation graph is built).
bool autotune_enabled()
{
    const char *e = getenv("MXB_AUTOTUNE");
    return !(e && *e == '0');
}

}  // namespace

// Autotuner: runs the op sequence once; every tensor-core op is timed with each candidate
// column-tile width (second of two runs, CUDA events) with the Y outputs redirected to
// scratch, and the fastest width is kept.  Each op's outputs are left in place for the next.
// One-launch mode: the whole evaluation is one launch, so its one column-tile width (64 or 128)
// is picked by timing the launch with each (Y redirected to scratch).
int Batch::tune_one_launch(Entry &e, std::vector<PlanArgs> pa, std::vector<int> &bn, cudaStream_t stream,
                           long long wait_cycles)
{
    const int np = (int)plans.size();
    std::vector<double *> scratch(np, nullptr);
    PlanArgs *dTune = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Entry te;
    te.nrhs = e.nrhs;
    int rc = MXB_OK;
    for (int i = 0; i < np && !rc; ++i) {
        Plan &p = *plans[i];
        size_t ext = 0;
        for (int l = 0; l < p.nleaf; ++l)
            ext = std::max<size_t>(ext, (size_t)p.ofs_host[1][l] + (size_t)p.Ddim[l] * e.nrhs[i]);
        if (cudaMalloc(&scratch[i], std::max<size_t>(ext, 1) * sizeof(double)) != cudaSuccess)
            rc = batch_fail("autotune scratch allocation failed", MXB_ERR_NOMEM);
        else
            pa[i].Y = scratch[i];
        pa[i].y_perm = nullptr;
    }
    if (!rc && cudaMalloc(&dTune, np * sizeof(PlanArgs)) != cudaSuccess)
        rc = batch_fail("autotune table allocation failed", MXB_ERR_NOMEM);
    if (!rc && cudaMemcpyAsync(dTune, pa.data(), np * sizeof(PlanArgs), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        rc = batch_fail("autotune table upload failed", MXB_ERR_CUDA);
    te.dPlans = dTune;
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = batch_fail("autotune events", MXB_ERR_CUDA);
    float best = 1e30f;
    int best_w = 128;
    for (int w : {128, 64}) {
        if (rc) break;
        std::vector<int> trial = bn;
        for (size_t k = 0; k < ops.size(); ++k)
            if (ops[k].phase != PH_SPLITW) trial[k] = w;
        rc = units_for(te, trial, stream);
        float ms = 0.f;
        for (int rep = 0; rep < 2 && !rc; ++rep) {
            cudaEventRecord(e0, stream);
            rc = enqueue(te, stream, 0, wait_cycles, trial, -1);
            cudaEventRecord(e1, stream);
            if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = batch_fail("autotune sync", MXB_ERR_CUDA);
            if (!rc) cudaEventElapsedTime(&ms, e0, e1);
        }
        if (!rc && ms < best) {
            best = ms;
            best_w = w;
        }
    }
    for (size_t k = 0; k < ops.size(); ++k)
        if (ops[k].phase != PH_SPLITW) bn[k] = best_w;
    if (!rc && cudaStreamSynchronize(stream) != cudaSuccess) rc = batch_fail("autotune sync", MXB_ERR_CUDA);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (te.dUnits) cudaFree(te.dUnits);
    if (dTune) cudaFree(dTune);
    for (double *x : scratch)
        if (x) cudaFree(x);
    return rc;
}

int Batch::tune(Entry &e, std::vector<PlanArgs> pa, std::vector<int> &bn, cudaStream_t stream, long long wait_cycles)
{
    if (one_launch) return tune_one_launch(e, pa, bn, stream, wait_cycles);
    const int np = (int)plans.size();
    const int maxn = *std::max_element(e.nrhs.begin(), e.nrhs.end());
    std::vector<double *> scratch(np, nullptr);
    PlanArgs *dTune = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Entry te;
    te.nrhs = e.nrhs;
    te.order = e.order;  // the same kernel instantiations as the evaluation (Y goes to scratch)
    int rc = MXB_OK;
    for (int i = 0; i < np && !rc; ++i) {
        Plan &p = *plans[i];
        size_t ext = 0;
        for (int l = 0; l < p.nleaf; ++l)
            ext = std::max<size_t>(ext, (size_t)p.ofs_host[1][l] + (size_t)p.Ddim[l] * e.nrhs[i]);
        if (cudaMalloc(&scratch[i], std::max<size_t>(ext, 1) * sizeof(double)) != cudaSuccess)
            rc = batch_fail("autotune scratch allocation failed", MXB_ERR_NOMEM);
        else
            pa[i].Y = scratch[i];
        pa[i].y_perm = nullptr;  // the scratch is leaf-blocked (packed offsets)
    }
    if (!rc && cudaMalloc(&dTune, np * sizeof(PlanArgs)) != cudaSuccess)
        rc = batch_fail("autotune table allocation failed", MXB_ERR_NOMEM);
    if (!rc && cudaMemcpyAsync(dTune, pa.data(), np * sizeof(PlanArgs), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        rc = batch_fail("autotune table upload failed", MXB_ERR_CUDA);
    te.dPlans = dTune;
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = batch_fail("autotune events", MXB_ERR_CUDA);
    std::vector<float> op_ms(ops.size(), 0.f);
    for (size_t k = 0; k < ops.size() && !rc; ++k) {
        if (ops[k].phase == PH_SPLITW) {
            rc = units_for(te, bn, stream);
            if (!rc) rc = enqueue(te, stream, 0, wait_cycles, bn, (int)k);
            continue;
        }
        std::vector<int> cands = ops[k].P == 2 ? std::vector<int>{256, 128, 64} : std::vector<int>{128, 64};
        if (ops[k].max_m > 128 && pairs_enabled()) {
            cands.push_back(256 | MXB_TILE_PAIR);
            cands.push_back(128 | MXB_TILE_PAIR);
        }
        float best = 1e30f;
        int best_bn = bn[k];
        for (int c : cands) {
            if (tile_width(c) > 2 * std::max(64, maxn)) continue;
            std::vector<int> trial = bn;
            trial[k] = c;
            rc = units_for(te, trial, stream);
            float ms = 0.f;
            bool refused = false;
            for (int rep = 0; rep < 2 && !rc && !refused; ++rep) {
                cudaEventRecord(e0, stream);
                const int lrc = enqueue(te, stream, 0, wait_cycles, trial, (int)k);
                cudaEventRecord(e1, stream);
                if (lrc) {
                    // a launch the device refuses (e.g. no room for a cluster) is not a candidate;
                    // launch-configuration errors are not sticky
                    refused = true;
                    (void)cudaGetLastError();
                    continue;
                }
                if (cudaEventSynchronize(e1) != cudaSuccess) rc = batch_fail("autotune sync", MXB_ERR_CUDA);
                if (!rc) cudaEventElapsedTime(&ms, e0, e1);
            }
            if (rc) break;
            if (refused) continue;
            if (ms < best) {
                best = ms;
                best_bn = c;
            }
        }
        bn[k] = best_bn;
        op_ms[k] = best;
        if (!rc) rc = units_for(te, bn, stream);
        if (!rc) rc = enqueue(te, stream, 0, wait_cycles, bn, (int)k);
    }
    // Chains: a run of consecutive up-sweep launches (or down-sweep launches, leaf down
    // included) of one product count may run as one launch whose levels wait for each other on
    // the device.  Each run is timed chained, with every candidate tile shared by its levels,
    // against the sum of its separately tuned launches; the faster is kept.  Every op's inputs
    // are in place from the pass above, and re-running an op rewrites the same outputs.
    for (size_t k = 0; k < ops.size() && !rc && chains_enabled();) {
        const int fam = chain_family(ops[k].phase);
        size_t j = k + 1;
        while (fam && j < ops.size() && chain_family(ops[j].phase) == fam && ops[j].P == ops[k].P &&
               j - k < (size_t)MAX_CHAIN)
            ++j;
        if (!fam || j - k < 2) {
            k = j;
            continue;
        }
        float separate = 0.f;
        int max_m = 0;
        for (size_t q = k; q < j; ++q) {
            separate += op_ms[q];
            max_m = std::max(max_m, ops[q].max_m);
        }
        std::vector<int> cands = ops[k].P == 2 ? std::vector<int>{256, 128, 64} : std::vector<int>{128, 64};
        if (max_m > 128 && pairs_enabled()) cands.push_back(128 | MXB_TILE_PAIR);
        float best = separate;
        std::vector<int> best_bn;
        for (int c : cands) {
            if (tile_width(c) > 2 * std::max(64, maxn)) continue;
            std::vector<int> trial = bn;
            trial[k] = c;
            for (size_t q = k + 1; q < j; ++q) trial[q] = c | TILE_CHAIN;
            rc = units_for(te, trial, stream);
            float ms = 0.f;
            bool refused = false;
            for (int rep = 0; rep < 2 && !rc && !refused; ++rep) {
                cudaEventRecord(e0, stream);
                const int lrc = enqueue(te, stream, 0, wait_cycles, trial, (int)k);
                cudaEventRecord(e1, stream);
                if (lrc) {
                    refused = true;
                    (void)cudaGetLastError();
                    continue;
                }
                if (cudaEventSynchronize(e1) != cudaSuccess) rc = batch_fail("autotune sync", MXB_ERR_CUDA);
                if (!rc) cudaEventElapsedTime(&ms, e0, e1);
            }
            if (rc) break;
            if (refused) continue;
            if (ms < best) {
                best = ms;
                best_bn = trial;
            }
        }
        if (!best_bn.empty()) bn = best_bn;
        k = j;
    }
    if (!rc) rc = units_for(te, bn, stream);
    if (!rc && cudaStreamSynchronize(stream) != cudaSuccess) rc = batch_fail("autotune sync", MXB_ERR_CUDA);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (te.dUnits) cudaFree(te.dUnits);
    if (dTune) cudaFree(dTune);
    for (double *s : scratch)
        if (s) cudaFree(s);
    return rc;
}

int Batch::evaluate(const double *const *W, double *const *Y, const int *nrhs, int accumulate, cudaStream_t stream,
                    int debug_flags, long long wait_cycles, const CallerOrder *order)
{
    const int np = (int)plans.size();
    int cur = -1;
    MXB_CUDA_OR(cudaGetDevice(&cur));
    if (cur != device) return batch_fail("batch used on a different device than it was created on");
    std::vector<int> nr(nrhs, nrhs + np);
    if (one_launch && order) return batch_fail("the one-launch mode takes leaf-blocked W and Y", MXB_ERR_UNSUPPORTED);
    bool realloc = false;
    if (buf_gens.size() != (size_t)np) buf_gens.assign(np, -1);
    for (int i = 0; i < np; ++i) {
        if (nr[i] < 1 || !W[i] || !Y[i]) return batch_fail("bad operand or nrhs in batch");
        int rc = split_buffers(*plans[i], *plans[i]->bf16, nr[i]);
        if (rc) return rc;
        realloc |= plans[i]->bf16->buf_gen != buf_gens[i];
        buf_gens[i] = plans[i]->bf16->buf_gen;
    }
    if (realloc) clear();
    MXB_CUDA_OR(configure_all_tc());
    Entry *hit = find(W, Y, nr, accumulate, debug_flags, order);
    if (!hit) {
        if (entries.size() >= 8) {
            release(entries.front());
            entries.erase(entries.begin());
        }
        Entry e;
        e.W.assign(W, W + np);
        e.Y.assign(Y, Y + np);
        e.nrhs = nr;
        e.accumulate = accumulate;
        e.debug_flags = debug_flags;
        if (order) e.order.assign(order, order + np);
        std::vector<PlanArgs> pa(np);
        for (int i = 0; i < np; ++i) {
            Plan &p = *plans[i];
            SplitBF16 &S = *p.bf16;
            for (int k = 0; k < NPOOL; ++k) pa[i].pool[k] = S.pool[k];
            pa[i].buf[BUF_W] = S.Wt;
            pa[i].buf[BUF_WSKEL] = S.wT;
            pa[i].buf[BUF_USKEL] = S.uT;
            pa[i].W = W[i];
            pa[i].Y = Y[i];
            pa[i].wofs = p.dOfs;
            pa[i].yofs = p.dOfs + p.nleaf;
            pa[i].skel = S.u32;
            pa[i].NT = S.nt_cap;
            pa[i].nrhs = nr[i];
            pa[i].beta_arg = accumulate ? 1 : 0;
            if (order) {
                pa[i].w_perm = pa[i].y_perm = order[i].perm;
                pa[i].tofs = order[i].tofs;
                pa[i].w_rs = order[i].w_rs;
                pa[i].w_cs = order[i].w_cs;
                pa[i].y_rs = order[i].y_rs;
                pa[i].y_cs = order[i].y_cs;
            }
        }
        cudaError_t err = cudaMalloc(&e.dPlans, np * sizeof(PlanArgs));
        // on the evaluation stream, ahead of the graph launch that reads it
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(e.dPlans, pa.data(), np * sizeof(PlanArgs), cudaMemcpyHostToDevice, stream);
        if (err != cudaSuccess) {
            release(e);
            return batch_fail(std::string("batch plan table: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
        }
        // column tiles: measured per op on the first evaluation of an nrhs signature
        const int maxn = *std::max_element(nr.begin(), nr.end());
        std::vector<int> bn(ops.size(), 0);
        for (size_t k = 0; k < ops.size(); ++k)
            if (ops[k].phase != PH_SPLITW) bn[k] = default_bn(ops[k].P, maxn);
        auto t = tuned.find(nr);
        if (forced_tile(2)) {
            for (size_t k = 0; k < ops.size(); ++k)
                if (ops[k].phase != PH_SPLITW) bn[k] = forced_tile(ops[k].P);
        } else if (t != tuned.end()) {
            bn = t->second;
        } else if (autotune_enabled() && !debug_flags) {
            int rc = tune(e, pa, bn, stream, wait_cycles);
            if (rc) {
                release(e);
                return rc;
            }
            tuned[nr] = bn;
        }
        if ((debug_flags & (MXB_DEBUG_CHAIN_LEVELS | MXB_DEBUG_STALL_LEVEL)) || chains_forced()) chain_all(bn);
        if (one_launch) {
            // one tile for the whole launch: the first tensor-core op's width, 64 or 128
            int w = 0;
            for (size_t k = 0; k < ops.size() && !w; ++k)
                if (ops[k].phase != PH_SPLITW) w = tile_width(bn[k]) >= 128 ? 128 : 64;
            for (size_t k = 0; k < ops.size(); ++k)
                if (ops[k].phase != PH_SPLITW) bn[k] = w;
        }
        e.bn = bn;
        int rc = units_for(e, bn, stream);
        if (rc) {
            release(e);
            return rc;
        }
        if (!capture_stream && cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
            release(e);
            return batch_fail("creating the capture stream failed", MXB_ERR_CUDA);
        }
        if (cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            release(e);
            return batch_fail("beginning the graph capture failed", MXB_ERR_CUDA);
        }
        rc = enqueue(e, capture_stream, debug_flags, wait_cycles, bn);
        cudaGraph_t graph = nullptr;
        err = cudaStreamEndCapture(capture_stream, &graph);
        if (rc || err != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            release(e);
            return rc ? rc : batch_fail(std::string("capturing the evaluation: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
        }
        err = cudaGraphInstantiate(&e.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (err != cudaSuccess) {
            release(e);
            return batch_fail(std::string("instantiating the evaluation graph: ") + cudaGetErrorString(err), MXB_ERR_CUDA);
        }
        entries.push_back(std::move(e));
        hit = &entries.back();
    }
    MXB_CUDA_OR(cudaGraphLaunch(hit->exec, stream));
    return MXB_OK;
}

Batch::Entry *Batch::find(const double *const *W, double *const *Y, const std::vector<int> &nr, int accumulate,
                          int debug_flags, const CallerOrder *order)
{
    Entry *hit = nullptr;
    for (Entry &e : entries) {
        bool same = e.accumulate == accumulate && e.nrhs == nr && e.debug_flags == debug_flags &&
                    e.order.empty() == !order;
        for (size_t i = 0; same && order && i < plans.size(); ++i) {
            const CallerOrder &a = e.order[i], &b = order[i];
            same = a.perm == b.perm && a.tofs == b.tofs && a.w_rs == b.w_rs && a.w_cs == b.w_cs && a.y_rs == b.y_rs &&
                   a.y_cs == b.y_cs;
        }
        for (size_t i = 0; same && i < plans.size(); ++i) same = e.W[i] == W[i] && e.Y[i] == Y[i];
        if (same) hit = &e;
    }
    return hit;
}

// Launch-by-launch timing of one evaluation (mxb_batch_profile / mxb_plan_profile); the
// evaluation graph of these operands has been built (and run) by the caller.
int Batch::profile(const double *const *W, double *const *Y, const int *nrhs, cudaStream_t stream, mxb_op_profile *out,
                   int cap, int *nops)
{
    const std::vector<int> nr(nrhs, nrhs + plans.size());
    Entry *e = find(W, Y, nr, 0, 0);
    if (!e) return batch_fail("profile: no evaluation graph for these operands");
    std::vector<cudaEvent_t> ev(ops.size() + 1, nullptr);
    int rc = MXB_OK;
    for (cudaEvent_t &x : ev)
        if (!rc && cudaEventCreate(&x) != cudaSuccess) rc = batch_fail("profile: creating CUDA events failed", MXB_ERR_CUDA);
    // one launch: each level's span on the device, from the kernel's own timestamps
    std::vector<unsigned long long> lns(ops.size() + 1, 0);
    if (!rc && one_launch) {
        if (cudaMalloc(&level_ns, lns.size() * sizeof(unsigned long long)) != cudaSuccess) {
            level_ns = nullptr;
            rc = batch_fail("profile: level timer allocation failed", MXB_ERR_NOMEM);
        }
    }
    for (int rep = 0; rep < 2 && !rc; ++rep) {
        if (level_ns) {
            cudaMemsetAsync(level_ns, 0, lns.size() * sizeof(unsigned long long), stream);
            cudaMemsetAsync(level_ns, 0xff, sizeof(unsigned long long), stream);  // start: minimum of
        }
        cudaEventRecord(ev[0], stream);
        for (size_t k = 0; k < ops.size() && !rc; ++k) {
            rc = enqueue(*e, stream, 0, 0, e->bn, (int)k);
            cudaEventRecord(ev[k + 1], stream);
        }
        if (!rc && cudaStreamSynchronize(stream) != cudaSuccess)
            rc = batch_fail("profile: stream synchronisation failed", MXB_ERR_CUDA);
    }
    if (level_ns) {
        if (!rc && cudaMemcpy(lns.data(), level_ns, lns.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) !=
                       cudaSuccess)
            rc = batch_fail("profile: reading the level timers failed", MXB_ERR_CUDA);
        cudaFree(level_ns);
        level_ns = nullptr;
    }
    if (nops) *nops = (int)ops.size();
    std::vector<TcUnit> units;
    if (!rc) {
        size_t n = 0;
        for (int c : e->unit_count) n += (size_t)c;
        units.resize(n);
        if (n && cudaMemcpy(units.data(), e->dUnits, n * sizeof(TcUnit), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = batch_fail("profile: reading the work units failed", MXB_ERR_CUDA);
    }
    // the op of each unit, from its task (the units of a dataflow launch interleave its ops)
    std::vector<int> task_op(tasks.size(), -1);
    for (size_t k = 0; k < ops.size(); ++k) {
        if (ops[k].phase == PH_SPLITW) {
            for (int t = split_task0; t < split_task0 + split_tasks; ++t) task_op[t] = (int)k;
            continue;
        }
        for (int t = ops[k].first; t < ops[k].first + ops[k].count; ++t) task_op[t] = (int)k;
    }
    for (size_t k = 0; k < ops.size() && !rc && (int)k < cap && out; ++k) {
        const MOp &m = ops[k];
        mxb_op_profile &o = out[k];
        o = mxb_op_profile{};
        o.phase = m.phase;
        o.level = m.level;
        o.width = tile_width(e->bn[k]);
        o.pair = tile_pair(e->bn[k]) ? 1 : 0;
        o.chained = one_launch ? (k > 0) : ((m.phase != PH_SPLITW && (e->bn[k] & TILE_CHAIN)) ? 1 : 0);
        cudaEventElapsedTime(&o.ms, ev[k], ev[k + 1]);
        if (o.chained) o.ms = 0.f;
        if (one_launch && lns[k + 1] >= lns[k] && lns[0] != ~0ull)
            o.level_ms = (float)((double)(lns[k + 1] - (k ? lns[k] : lns[0])) * 1e-6);
    }
    for (size_t u = 0; u < units.size() && !rc && out; ++u) {
        const TcTask &t = tasks[units[u].task];
        const int k = task_op[units[u].task];
        if (k < 0 || k >= cap) continue;
        mxb_op_profile &o = out[k];
        ++o.units;
        const double products = ops[k].P == 2 ? 3.0 : 6.0;
        const int tile_rows = o.pair ? 256 : 128;
        const double rows = std::min(tile_rows, t.M - t.m0);
        const double cols = std::min(o.width, nr[t.plan] - units[u].col * o.width);
        for (int q = t.item0; q < t.item0 + t.nitem; ++q) {
            o.flops += 2.0 * rows * items[q].K * cols;
            o.issued_flops += products * 2.0 * tile_rows * (64.0 * items[q].KT) * o.width;
        }
    }
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    return rc;
}

// ---------------------------------------------------------------------------------------
// plan set-up
// ---------------------------------------------------------------------------------------

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
    // the adjoint's operands: D_xy^T (m_y x m_x) and B_xy^T (s_y x s_x)
    std::vector<uint64_t> neart_a, fart_a;
    if (want_adjoint) {
        neart_a.resize(near_x.size());
        fart_a.resize(far_x.size());
        for (size_t k = 0; k < near_x.size(); ++k)
            neart_a[k] = add_pool(POOL_NEART, 0, near_off[k], Ddim[near_x[k]], Ddim[near_y[k]], Ddim[near_x[k]], 1,
                                  near_parts);
        for (size_t k = 0; k < far_x.size(); ++k)
            fart_a[k] = add_pool(POOL_FART, 1, far_off[k], slen[far_x[k]], slen[far_y[k]], slen[far_x[k]], 1, far_parts);
    }
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
    std::vector<Op> *op_list = &S->ops;  // the forward's, then the adjoint's
    auto begin_op = [&](int phase, int level, int P) {
        Op o{};
        o.key = op_key(phase, level, P);
        o.phase = phase;
        o.level = level;
        o.P = P;
        o.first = phase == PH_SPLITW ? (int)S->jobs.size() : (int)S->tasks.size();
        op_list->push_back(o);
    };
    auto end_op = [&]() {
        Op &o = op_list->back();
        o.count = (o.phase == PH_SPLITW ? (int)S->jobs.size() : (int)S->tasks.size()) - o.first;
        if (o.count == 0) op_list->pop_back();
    };
    auto add_tasks = [&](int16_t out_kind, int64_t c_row, int64_t out_kt, int ldc, int M, int item0,
                         int16_t beta, int t_buf) {
        for (int m0 = 0; m0 < M; m0 += 128) {
            TcTask t{};
            t.c_row = c_row;
            t.out_kt = out_kt;
            t.ldc = ldc;
            t.M = M;
            t.m0 = m0;
            t.item0 = item0;
            t.nitem = (int)S->items.size() - item0;
            t.plan = 0;
            t.out_kind = out_kind;
            t.beta = beta;
            t.t_buf = t_buf;
            S->tasks.push_back(t);
        }
    };
    auto item = [&](int a_pool, uint64_t a_off, int b_buf, int64_t b_base, int K) {
        TcItem it{};
        it.a_pool = (int16_t)a_pool;
        it.a_off = a_off;
        it.b_buf = (int16_t)b_buf;
        it.b_base = b_base;
        it.KT = KT(K);
        it.K = K;
        if (it.KT > 0) S->items.push_back(it);
    };

    // W -> tiles
    begin_op(PH_SPLITW, 0, 0);
    for (int i = 0; i < nleaf; ++i) {
        SplitJob j{};
        j.src_row = i;
        j.dst_kt = S->leaf_kt[i];
        j.ld = Ddim[i];
        j.K = Ddim[i];
        j.KT = KT(Ddim[i]);
        j.plan = 0;
        if (j.KT > 0) S->jobs.push_back(j);
    }
    end_op();
    // up-sweep by height: the epilogue writes wskel directly as operand tiles
    for (int h = 0; h <= maxh; ++h) {
        begin_op(PH_UP, h, 3);
        for (int v : bfs) {
            if (height[v] != h || !projects(v)) continue;
            const int item0 = (int)S->items.size();
            if (lch[v] == -1) {
                item(POOL_VU3, up_a[v], BUF_W, S->leaf_kt[lm[v]], Ddim[lm[v]]);
            } else {
                if (slen[lch[v]] > 0) item(POOL_VU3, up_a[v], BUF_WSKEL, S->node_kt[lch[v]], slen[lch[v]]);
                if (slen[rch[v]] > 0) item(POOL_VU3, up_b[v], BUF_WSKEL, S->node_kt[rch[v]], slen[rch[v]]);
            }
            add_tasks(OUT_TILES, skel_row[v], S->node_kt[v], slen[v], slen[v], item0, 0, BUF_WSKEL);
        }
        end_op();
    }
    // far couplings of every depth in one launch (they read only wskel): a node whose parent
    // projects keeps its far result in FP32 for its down launch, which adds its own product and
    // writes uskel tiles; other nodes' far results become tiles directly.  The near field
    // (Y (+)= D W, reads only W) joins that launch when it uses the same product count.
    auto has_down = [&](int c) { return parent[c] >= 0 && projects(parent[c]); };
    std::vector<std::vector<int>> far_out(numnodes);
    for (size_t k = 0; k < far_x.size(); ++k) far_out[far_x[k]].push_back((int)k);
    std::vector<std::vector<int>> near_out(nleaf);
    for (size_t k = 0; k < near_x.size(); ++k) near_out[near_x[k]].push_back((int)k);
    auto near_tasks = [&]() {
        for (int v : bfs) {
            if (lch[v] != -1) continue;
            const int x = lm[v];
            const int item0 = (int)S->items.size();
            for (int k : near_out[x]) item(POOL_NEAR, near_a[k], BUF_W, S->leaf_kt[near_y[k]], Ddim[near_y[k]]);
            add_tasks(OUT_Y, x, 0, Ddim[x], Ddim[x], item0, 2, BUF_W);
        }
    };
    const bool near_with_far = near_parts == far_parts;
    begin_op(near_with_far ? PH_FARNEAR : PH_FAR, 0, far_parts);
    for (int c : bfs) {
        if (!projects(c)) continue;
        const int item0 = (int)S->items.size();
        for (int k : far_out[c])
            if (slen[far_y[k]] > 0) item(POOL_FAR, far_a[k], BUF_WSKEL, S->node_kt[far_y[k]], slen[far_y[k]]);
        add_tasks(has_down(c) ? OUT_F32 : OUT_TILES, skel_row[c], S->node_kt[c], slen[c], slen[c], item0, 0,
                  BUF_USKEL);
    }
    if (near_with_far) near_tasks();
    end_op();
    for (int dd = 1; dd <= maxd; ++dd) {
        begin_op(PH_DOWN, dd, 3);
        for (int c : bfs) {
            if (depth[c] != dd || !projects(c) || !has_down(c)) continue;
            const int item0 = (int)S->items.size();
            item(POOL_VD3, down_child[c], BUF_USKEL, S->node_kt[parent[c]], slen[parent[c]]);
            add_tasks(OUT_TILES, skel_row[c], S->node_kt[c], slen[c], slen[c], item0, 1, BUF_USKEL);
        }
        end_op();
    }
    // near (if not with the far couplings), then leaf down (Y += P^T uskel)
    if (!near_with_far) {
        begin_op(PH_NEAR, 0, near_parts);
        near_tasks();
        end_op();
    }
    begin_op(PH_LEAFDOWN, 0, 3);
    for (int v : bfs) {
        if (lch[v] != -1 || !projects(v)) continue;
        const int item0 = (int)S->items.size();
        item(POOL_VD3, down_a[v], BUF_USKEL, S->node_kt[v], slen[v]);
        add_tasks(OUT_Y, lm[v], 0, Ddim[lm[v]], Ddim[lm[v]], item0, 1, BUF_W);
    }
    end_op();

    // ---- the transposed traversal (dGW = K~^T dG) ----
    // The same W split, up sweep, down sweep and leaf down; the far couplings and the near field
    // transposed: far pair (x, y) adds B_xy^T wskel[x] to node y, near pair (x, y) adds
    // D_xy^T G[x] to leaf y (the FP64 adjoint's traversal, with the transposed tiled pools).
    if (want_adjoint) {
        op_list = &S->ops_adj;
        for (const Op &o : S->ops)
            if (o.phase == PH_SPLITW || o.phase == PH_UP || o.phase == PH_DOWN || o.phase == PH_LEAFDOWN)
                S->ops_adj.push_back(o);
        std::vector<std::vector<int>> far_in(numnodes), near_in(nleaf);
        for (size_t k = 0; k < far_x.size(); ++k) far_in[far_y[k]].push_back((int)k);
        for (size_t k = 0; k < near_x.size(); ++k) near_in[near_y[k]].push_back((int)k);
        auto near_tasks_t = [&]() {
            for (int v : bfs) {
                if (lch[v] != -1) continue;
                const int x = lm[v];
                const int item0 = (int)S->items.size();
                for (int k : near_in[x]) item(POOL_NEART, neart_a[k], BUF_W, S->leaf_kt[near_x[k]], Ddim[near_x[k]]);
                add_tasks(OUT_Y, x, 0, Ddim[x], Ddim[x], item0, 2, BUF_W);
            }
        };
        begin_op(near_with_far ? PH_FARNEAR : PH_FAR, 0, far_parts);
        for (int c : bfs) {
            if (!projects(c)) continue;
            const int item0 = (int)S->items.size();
            for (int k : far_in[c])
                if (slen[far_x[k]] > 0) item(POOL_FART, fart_a[k], BUF_WSKEL, S->node_kt[far_x[k]], slen[far_x[k]]);
            add_tasks(has_down(c) ? OUT_F32 : OUT_TILES, skel_row[c], S->node_kt[c], slen[c], slen[c], item0, 0,
                      BUF_USKEL);
        }
        if (near_with_far) near_tasks_t();
        end_op();
        if (!near_with_far) {
            begin_op(PH_NEAR, 0, near_parts);
            near_tasks_t();
            end_op();
        }
        op_list = &S->ops;
    }

    // the split path reads only the tiled pools: release the FP64 copies of the CDS
    const uint64_t fp64_len[3] = {D_len, B_len, VT_len};
    double **fp64_buf[3] = {&dD, &dB, &dVT};
    for (int q = 0; q < 3; ++q) {
        if (!*fp64_buf[q]) continue;
        cudaFree(*fp64_buf[q]);
        allocations.erase(std::remove(allocations.begin(), allocations.end(), (void *)*fp64_buf[q]),
                          allocations.end());
        *fp64_buf[q] = nullptr;
        device_bytes -= std::max<uint64_t>(fp64_len[q], 1) * sizeof(double);
    }
    int rc = alloc((void **)&S->dErr, sizeof(int));
    if (rc) return rc;
    if (cudaMemset(S->dErr, 0, sizeof(int)) != cudaSuccess) {
        set_error("clearing the error word failed");
        return MXB_ERR_CUDA;
    }
    // the batch of this plan alone, used by mxb_plan_evaluate
    S->self = new Batch();
    rc = S->self->build({this});
    if (!rc && want_adjoint) {
        S->self_adj = new Batch();
        rc = S->self_adj->build({this}, true);
    }
    return rc;
}

int Plan::run_split_bf16(const std::vector<Launch> &L, const double *dW, double *dY, int nrhs, int accumulate,
                         cudaStream_t stream, const CallerOrder *order)
{
    Batch *b = bf16->self;
    if (&L == &launches_adj) {
        if (!bf16->self_adj) {
            set_error("this split-BF16 plan has no adjoint: create it with precision | MXB_PLAN_ADJOINT (or use an "
                      "FP64 plan)");
            return MXB_ERR_UNSUPPORTED;
        }
        b = bf16->self_adj;
    }
    const int rc = batch_set_one_launch(b, (debug_flags & MXB_DEBUG_ONE_LAUNCH) != 0);
    if (rc) return rc;
    return b->evaluate(&dW, &dY, &nrhs, accumulate, stream, debug_flags, debug_wait_cycles, order);
}

void Plan::clear_split_graphs()
{
    if (bf16 && bf16->self) bf16->self->clear();
    if (bf16 && bf16->self_adj) bf16->self_adj->clear();
}

int split_bf16_prepare() { return configure_all_tc() == cudaSuccess ? MXB_OK : MXB_ERR_CUDA; }

// Launches of an evaluation: one per op, less the ops chained into the launch before them in
// the most recent evaluation graph.
int launch_count(const Batch *b)
{
    if (!b) return 0;
    if (b->one_launch) return 1;
    int n = (int)b->ops.size();
    if (!b->entries.empty()) {
        const std::vector<int> &bn = b->entries.back().bn;
        for (size_t k = 0; k < bn.size() && k < b->ops.size(); ++k)
            if (b->ops[k].phase != PH_SPLITW && (bn[k] & TILE_CHAIN)) --n;
    }
    return n;
}

int split_bf16_launches(const Plan &p) { return p.bf16 ? launch_count(p.bf16->self) : 0; }

Batch *split_bf16_batch(Plan &p) { return p.bf16 ? p.bf16->self : nullptr; }

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
    if (bf16) {
        delete bf16->self;
        delete bf16->self_adj;
    }
    delete bf16;
    bf16 = nullptr;
}

// ---- batch entry points used by the C-ABI ----
int batch_create(Plan *const *plans, int count, Batch **out)
{
    if (!plans || count < 1 || !out) return batch_fail("bad batch arguments");
    std::unique_ptr<Batch> b(new Batch());
    int rc = b->build(std::vector<Plan *>(plans, plans + count));
    if (rc) return rc;
    *out = b.release();
    return MXB_OK;
}

int batch_evaluate(Batch *b, const double *const *W, double *const *Y, const int *nrhs, int accumulate,
                   cudaStream_t stream)
{
    if (!b || !W || !Y || !nrhs) return batch_fail("bad batch arguments");
    for (size_t i = 0; i < b->plans.size(); ++i) {
        if (nrhs[i] < 1) return batch_fail("nrhs must be >= 1");
        int rc = b->plans[i]->stage_offsets(0, nullptr, nrhs[i], stream);
        if (!rc) rc = b->plans[i]->stage_offsets(1, nullptr, nrhs[i], stream);
        if (rc) return rc;
    }
    return b->evaluate(W, Y, nrhs, accumulate, stream, 0, 0);
}

int batch_profile(Batch *b, const double *const *W, double *const *Y, const int *nrhs, cudaStream_t stream,
                  mxb_op_profile *out, int cap, int *nops)
{
    if (!b || !W || !Y || !nrhs) return batch_fail("bad batch arguments");
    int rc = batch_evaluate(b, W, Y, nrhs, 0, stream);  // builds the entry (and tunes) if needed
    if (rc) return rc;
    return b->profile(W, Y, nrhs, stream, out, cap, nops);
}

int batch_status(Batch *b)
{
    if (!b) return batch_fail("null batch");
    MXB_CUDA_OR(cudaDeviceSynchronize());
    int rc = MXB_OK;
    for (Plan *p : b->plans) {
        const int r = split_bf16_status(*p);
        if (r && !rc) rc = r;
    }
    return rc;
}

void batch_destroy(Batch *b) { delete b; }

int batch_launches(const Batch *b) { return launch_count(b); }

int batch_set_one_launch(Batch *b, int on)
{
    if (!b) return batch_fail("null batch");
    if (b->one_launch != (on != 0)) {
        b->one_launch = on != 0;
        b->clear();
        b->tuned.clear();
    }
    return MXB_OK;
}

int batch_tuned_widths(const Batch *b, int *widths, int cap)
{
    if (!b || b->entries.empty()) return 0;
    const std::vector<int> &bn = b->entries.back().bn;
    int n = 0;
    for (size_t k = 0; k < bn.size() && n < cap; ++k)
        if (bn[k]) widths[n++] = bn[k];
    return n;
}

}  // namespace mxb

// Test hook (no counterpart in the reference): the unit order of a chained sweep, as the dataflow
// launches use it, for a synthetic dependency forest; host code only.
extern "C" int32_t mxb_debug_dataflow_order(int32_t nnodes, const int32_t *dep_first, const int32_t *deps,
                                            const int32_t *ntask, const int32_t *kt, int32_t ncol, int32_t workers,
                                            int32_t *node, int32_t *col, int32_t *dep0, int32_t *dep1,
                                            int32_t *need, int32_t *sig, int64_t cap, int64_t *count)
{
    if (nnodes < 1 || !dep_first || !ntask || !kt || ncol < 1 || workers < 1 || !node || !col || !dep0 || !dep1 ||
        !need || !sig || !count || cap < 0) {
        mxb::set_error("bad dataflow-order arguments");
        return MXB_ERR_ARG;
    }
    std::vector<mxb::DfNode> nodes(nnodes);
    int task = 0;
    for (int n = 0; n < nnodes; ++n) {
        mxb::DfNode &nd = nodes[n];
        if (ntask[n] < 1 || kt[n] < 0 || dep_first[n + 1] < dep_first[n] || (dep_first[n + 1] > dep_first[n] && !deps)) {
            mxb::set_error("bad dataflow-order node");
            return MXB_ERR_ARG;
        }
        nd.key = n;
        nd.ncol = ncol;
        nd.kt = kt[n];
        for (int t = 0; t < ntask[n]; ++t) nd.tasks.push_back(task++);
        for (int q = dep_first[n]; q < dep_first[n + 1]; ++q) nd.dep.push_back(deps[q]);
    }
    // levels as the sweeps number them: every node after the nodes it reads
    for (int pass = 0; pass < nnodes; ++pass) {
        bool moved = false;
        for (mxb::DfNode &nd : nodes)
            for (int d : nd.dep)
                if (d >= 0 && d < nnodes && nodes[d].level + 1 > nd.level) {
                    nd.level = nodes[d].level + 1;
                    moved = true;
                }
        if (!moved) break;
    }
    std::vector<mxb::TcUnit> units;
    std::vector<int> unit_node;
    int ndeps = 0;
    const int rc = mxb::dataflow_schedule(nodes, workers, units, ndeps, &unit_node);
    if (rc < 0) return rc;
    if (rc == 0) {
        mxb::set_error("the dependencies are not a tree");
        return MXB_ERR_UNSUPPORTED;
    }
    *count = (int64_t)units.size();
    if ((int64_t)units.size() > cap) {
        mxb::set_error("output arrays too short");
        return MXB_ERR_ARG;
    }
    for (size_t u = 0; u < units.size(); ++u) {
        node[u] = unit_node[u];
        col[u] = units[u].col;
        dep0[u] = units[u].dep0;
        dep1[u] = units[u].dep1;
        need[u] = units[u].need;
        sig[u] = units[u].sig;
    }
    return MXB_OK;
}
