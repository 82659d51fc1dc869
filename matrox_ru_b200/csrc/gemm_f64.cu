// FP64 grouped variable-size GEMM on the B200's FP64 tensor path.
//
// tcgen05.mma has no f64 kind, so FP64 products use the DMMA instruction
// mma.sync.m8n8k4.f64 (sm_80+).  One CTA computes a 64 x 64 tile of one task's output
// block C: the sum over the task's items of op(A)[m0:m0+64, :] * B[:, n0:n0+64].  The
// K loop runs over all items back to back through a 2-stage cp.async pipeline, so a
// near-field row (several D_xy * W_y) or a transfer (two child projections) is one
// pipeline with one epilogue and no atomics: every output tile has exactly one writer.
//
// Shared-memory layout per stage: A tile as [k][m] (m contiguous, row pitch 72 doubles), or,
// for a transposed A (whose K is contiguous in memory), as [m][k] (pitch 20); B tile as [n][k]
// (k contiguous, pitch 20 doubles).  The pitches make the DMMA fragment reads (A: 8 rows x 4 k
// per warp, B: 4 k x 8 cols) hit every bank pair exactly twice, the 2-wavefront minimum of a
// 256-byte warp load.  Global -> shared copies move pairs of doubles along the contiguous
// dimension as one 16-byte cp.async where the block is 16-byte aligned with an even leading
// dimension, single doubles otherwise.
//
// Occupancy: 4 CTAs (16 warps) per SM at <= 128 registers and 40 KB of shared memory each.
// Measured at N = 65536 / 1024 rhs this is 2.4 % faster than 3 CTAs with 3 stages (160
// registers); 5 or 6 CTAs per SM gain nothing more (the DMMA pipe is the limit).
#include <cstdio>

#include "mxb_internal.h"

namespace mxb {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, STAGES = 2, THREADS = 128;
constexpr int A_LD = BM + 8;
constexpr int B_LD = BK + 4;
constexpr int T_LD = BK + 4;  // transposed A operand: [m][k], k contiguous, like B
constexpr int A_TILE = (BK * A_LD > BM * T_LD) ? BK * A_LD : BM * T_LD;
constexpr int B_TILE = BN * B_LD;
constexpr int STAGE = A_TILE + B_TILE;
constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE * sizeof(double);

__device__ __forceinline__ void cp_async8(double *dst, const double *src, bool valid)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int n = valid ? 8 : 0;  // 0 source bytes: the 8 destination bytes are zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(n));
}
// 16 bytes (two doubles); `bytes` < 16 copies that many and zero-fills the rest
__device__ __forceinline__ void cp_async16(double *dst, const double *src, int bytes)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

struct Loader {
    const double *A;
    const double *B;
    int lda, ldb, K, trans;
    int k0;
    int q;
    bool a16, b16;  // pairs of doubles along the contiguous dimension are 16-byte aligned
    bool t16;       // the same for a transposed A (pairs along K)
};

__device__ __forceinline__ const double *operand_ptr(const Operands &ops, int kind, int64_t row)
{
    switch (kind) {
    case KIND_W: return ops.W + ops.wofs[row];
    case KIND_WSKEL: return ops.wskel + row * ops.nrhs;
    default: return ops.uskel + row * ops.nrhs;
    }
}

__device__ __forceinline__ void load_item(Loader &L, const Item *items, const Operands &ops)
{
    const Item it = items[L.q];
    // a switch, not ops.pool[it.a_pool]: a dynamic index into a kernel parameter array
    // would spill the parameter struct to local memory
    const double *pool = it.a_pool == 0 ? ops.pool[0] : (it.a_pool == 1 ? ops.pool[1] : ops.pool[2]);
    L.A = pool + it.a_off;
    L.B = operand_ptr(ops, it.b_kind, it.b_row);
    L.lda = it.lda;
    L.ldb = it.ldb;
    L.K = it.K;
    L.trans = it.trans;
    L.k0 = 0;
    // tile rows m0 and K offsets k0 are even, so every pair starts 16-byte aligned when the
    // block does and its leading dimension is even
    L.a16 = !it.trans && ((reinterpret_cast<uintptr_t>(L.A) & 15) == 0) && !(it.lda & 1);
    L.t16 = it.trans && ((reinterpret_cast<uintptr_t>(L.A) & 15) == 0) && !(it.lda & 1);
    L.b16 = ((reinterpret_cast<uintptr_t>(L.B) & 15) == 0) && !(it.ldb & 1);
}

__global__ void __launch_bounds__(THREADS, 4)
gemm_f64_kernel(const Task *__restrict__ tasks, const Item *__restrict__ items, Operands ops)
{
    extern __shared__ __align__(16) double smem[];
    // column tiles of one task run in neighbouring CTAs, so its A tiles come from DRAM once
    const int ncol = (ops.nrhs + BN - 1) / BN;
    const Task t = tasks[blockIdx.x / ncol];
    const int n0 = (blockIdx.x % ncol) * BN;
    const int nrhs = ops.nrhs;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const Item *titems = items + t.item0;

    int ktiles = 0;
    for (int q = 0; q < t.nitem; ++q) ktiles += (titems[q].K + BK - 1) / BK;

    Loader L;
    L.q = 0;
    if (t.nitem > 0) load_item(L, titems, ops);

    // bit s: stage s holds a transposed A tile, in the [m][k] layout
    int trmask = 0;
    auto issue = [&](int stage) {
        while (L.k0 >= L.K) {  // next item with work (items with K == 0 are skipped)
            ++L.q;
            load_item(L, titems, ops);
        }
        trmask = L.trans ? (trmask | (1 << stage)) : (trmask & ~(1 << stage));
        double *As = smem + stage * STAGE;
        double *Bs = As + A_TILE;
        const int k0 = L.k0;
        if (L.a16) {
            // two consecutive rows per copy: 16 bytes, the second zero-filled past M
#pragma unroll
            for (int i = 0; i < (BM * BK) / (2 * THREADS); ++i) {
                const int idx = tid + i * THREADS;
                const int m = (idx & (BM / 2 - 1)) * 2, k = idx / (BM / 2);
                const int nv = (k0 + k < L.K) ? max(0, min(2, t.M - (t.m0 + m))) : 0;
                const double *src = nv ? L.A + (size_t)(t.m0 + m) + (size_t)(k0 + k) * L.lda : L.A;
                cp_async16(As + k * A_LD + m, src, nv * 8);
            }
        } else if (!L.trans) {
#pragma unroll
            for (int i = 0; i < (BM * BK) / THREADS; ++i) {
                const int idx = tid + i * THREADS;
                const int m = idx & (BM - 1), k = idx / BM;
                const bool v = (t.m0 + m < t.M) && (k0 + k < L.K);
                const double *src = v ? L.A + (size_t)(t.m0 + m) + (size_t)(k0 + k) * L.lda : L.A;
                cp_async8(As + k * A_LD + m, src, v);
            }
        } else if (L.t16) {
            // transposed A: K is contiguous in memory; kept [m][k] so K pairs move as 16 bytes
#pragma unroll
            for (int i = 0; i < (BM * BK) / (2 * THREADS); ++i) {
                const int idx = tid + i * THREADS;
                const int k = (idx & (BK / 2 - 1)) * 2, m = idx / (BK / 2);
                const int nv = (t.m0 + m < t.M) ? max(0, min(2, L.K - (k0 + k))) : 0;
                const double *src = nv ? L.A + (size_t)(k0 + k) + (size_t)(t.m0 + m) * L.lda : L.A;
                cp_async16(As + m * T_LD + k, src, nv * 8);
            }
        } else {
#pragma unroll
            for (int i = 0; i < (BM * BK) / THREADS; ++i) {
                const int idx = tid + i * THREADS;
                const int k = idx & (BK - 1), m = idx / BK;
                const bool v = (t.m0 + m < t.M) && (k0 + k < L.K);
                const double *src = v ? L.A + (size_t)(k0 + k) + (size_t)(t.m0 + m) * L.lda : L.A;
                cp_async8(As + m * T_LD + k, src, v);
            }
        }
        if (L.b16) {
            // two consecutive K per copy
#pragma unroll
            for (int i = 0; i < (BN * BK) / (2 * THREADS); ++i) {
                const int idx = tid + i * THREADS;
                const int k = (idx & (BK / 2 - 1)) * 2, n = idx / (BK / 2);
                const int nv = (n0 + n < nrhs) ? max(0, min(2, L.K - (k0 + k))) : 0;
                const double *src = nv ? L.B + (size_t)(k0 + k) + (size_t)(n0 + n) * L.ldb : L.B;
                cp_async16(Bs + n * B_LD + k, src, nv * 8);
            }
        } else {
#pragma unroll
            for (int i = 0; i < (BN * BK) / THREADS; ++i) {
                const int idx = tid + i * THREADS;
                const int k = idx & (BK - 1), n = idx / BK;
                const bool v = (k0 + k < L.K) && (n0 + n < nrhs);
                const double *src = v ? L.B + (size_t)(k0 + k) + (size_t)(n0 + n) * L.ldb : L.B;
                cp_async8(Bs + n * B_LD + k, src, v);
            }
        }
        L.k0 += BK;
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) issue(s);
        cp_async_commit();
    }

    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        if (kt + STAGES - 1 < ktiles) issue((kt + STAGES - 1) % STAGES);
        cp_async_commit();

        const double *As = smem + (kt % STAGES) * STAGE;
        const double *Bs = As + A_TILE;
        const bool tr = (trmask >> (kt % STAGES)) & 1;
#pragma unroll
        for (int kk = 0; kk < BK / 4; ++kk) {
            double a[4], b[4];
            const int kr = kk * 4 + (lane & 3);
            if (tr) {
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[(wm * 32 + i * 8 + (lane >> 2)) * T_LD + kr];
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[kr * A_LD + wm * 32 + i * 8 + (lane >> 2)];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(wn * 32 + j * 8 + (lane >> 2)) * B_LD + kr];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_async_wait<0>();

    double *C;
    switch (t.c_kind) {
    case KIND_Y: C = ops.Y + ops.yofs[t.c_row]; break;
    case KIND_WSKEL: C = ops.wskel + t.c_row * nrhs; break;
    default: C = ops.uskel + t.c_row * nrhs; break;
    }
    const int beta = (t.beta == 2) ? ops.beta_arg : t.beta;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = t.m0 + wm * 32 + i * 8 + (lane >> 2);
        if (r >= t.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + e;
                if (c < nrhs) {
                    double *p = C + (size_t)r + (size_t)c * t.ldc;
                    *p = beta ? *p + acc[i][j][e] : acc[i][j][e];
                }
            }
        }
    }
}

}  // namespace

cudaError_t launch_gemm_f64(const Task *tasks, const Item *items, int ntasks, const Operands &ops,
                            cudaStream_t stream)
{
    static bool configured[128];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        e = cudaFuncSetAttribute(gemm_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (ntasks <= 0) return cudaSuccess;
    const int64_t blocks = (int64_t)ntasks * ((ops.nrhs + BN - 1) / BN);
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    gemm_f64_kernel<<<(unsigned)blocks, THREADS, SMEM_BYTES, stream>>>(tasks, items, ops);
    return cudaGetLastError();
}

int f64_row_tile() { return BM; }

cudaError_t prepare_gemm_f64()
{
    Operands ops{};
    ops.nrhs = 1;
    return launch_gemm_f64(nullptr, nullptr, 0, ops, 0) == cudaSuccess ? cudaSuccess : cudaErrorUnknown;
}

}  // namespace mxb
