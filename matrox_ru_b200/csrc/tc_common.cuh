// Blackwell (sm_100a) primitives used by the split-BF16 path: mbarriers with bounded waits,
// 1-D bulk copies into shared memory, TMEM allocation, tcgen05.mma / commit / ld, and the
// shared-memory matrix descriptor of a 128-byte-swizzled K-major operand tile.
#pragma once
#include <cstdint>

#include <cuda_bf16.h>

namespace mxb {
namespace tc {

// One operand tile: 128 rows x 64 K-elements of bf16, K-major, 128-byte swizzle.  Row r
// occupies bytes [128 r, 128 r + 128); its 16-byte chunk c (K elements 8c..8c+7) is stored
// at chunk position c ^ (r % 8).  Tiles are 1024-byte aligned everywhere.
constexpr int TILE_ROWS = 128;
constexpr int TILE_K = 64;
constexpr int TILE_BYTES = TILE_ROWS * TILE_K * 2;  // 16 KiB

__host__ __device__ constexpr uint32_t swizzled_offset(int r, int k)
{
    return (uint32_t)(r * 128 + ((((k >> 3) ^ (r & 7)) & 7) << 4) + ((k & 7) << 1));
}

// Spin limit of every wait, in SM clock cycles (~2 s at 1.9 GHz).  A wait that runs out
// marks the CTA aborted and reports MXB_ERR_TIMEOUT through the plan's error word.
constexpr long long WAIT_CYCLES = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on `parity`; gives up when the CTA's abort word is set or `limit` cycles pass.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_word,
                                          long long limit = WAIT_CYCLES)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_word) return false;
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

// Bounded wait until a global counter that other CTAs raise reaches `target` (acquire at GPU
// scope), then a proxy fence so that the bulk copies this thread issues next (async proxy) see
// the memory those CTAs wrote before raising it.  False when the wait gives up or an abort is
// raised.
__device__ __forceinline__ bool wait_counter(const int *ctr, int target, volatile int *abort_word,
                                             long long limit = WAIT_CYCLES)
{
    const long long t0 = clock64();
    for (;;) {
        int v;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(ctr) : "memory");
        if (v >= target) break;
        if (*abort_word) return false;
        if (clock64() - t0 > limit) return false;
        __nanosleep(32);
    }
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    return true;
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Acquire (GPU scope) of a counter another thread of this warp has seen complete: orders this
// thread's later loads after the writes that the counter's releases published.
__device__ __forceinline__ void acquire_counter(const int *ctr)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(ctr) : "memory");
    (void)v;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile (8-row groups 1024
// bytes apart).  Bits: start address >> 4 [0,14), leading byte offset >> 4 [16,30) (unused
// with this swizzle, 1 by convention), stride byte offset >> 4 [32,46), fixed version 1 at
// [46,48), base offset 0, layout type 2 (128-byte swizzle) at [61,64).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4)             // D format F32
           | (1u << 7)           // A format BF16
           | (1u << 10)          // B format BF16
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- CTA pairs (cluster of 2): one 256-row MMA over both SMs' shared memory ----
// A pair's tcgen05.mma.cta_group::2 takes rows 0-127 of A from the even CTA and rows
// 128-255 from the odd one, columns [0, N/2) of B from the even CTA and [N/2, N) from the
// odd one (same shared-memory offsets in both), and leaves each CTA its own 128 rows x N
// accumulator in its own TMEM.  Only the even CTA issues MMAs and commits.

__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}

// Address of the same shared-memory variable in CTA `rank` of this cluster.
__device__ __forceinline__ uint32_t peer_smem(const void *p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void st_remote_u32(uint32_t cluster_addr, uint32_t v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.u32 [%0], %1;\n" ::"r"(cluster_addr), "r"(v) : "memory");
}

// try_wait with cluster-scope acquire: for phases completed by the peer CTA's arrivals.
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity, volatile int *abort_word,
                                                  long long limit = WAIT_CYCLES)
{
    const long long t0 = clock64();
    while (!mbar_try_wait_cluster(bar, parity)) {
        if (*abort_word) return false;
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

// Every thread of both CTAs; orders all earlier shared-memory and barrier traffic.
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// One warp in EACH CTA of the pair issues these (same warp index in both).
__device__ __forceinline__ void tmem_alloc_pair(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::);
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mma_bf16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on the barrier at this offset in both CTAs once the pair's earlier MMAs complete.
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar)
{
    asm volatile(
        "{\n\t.reg .b16 m;\n\t"
        "mov.b16 m, 3;\n\t"
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], m;\n\t}\n" ::"r"(
            smem_u32(bar))
        : "memory");
}

// 64 consecutive FP32 columns of this thread's TMEM lane, one load and one wait.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float *v)
{
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// hi / mid / lo bf16 parts of x: hi = RN(x), mid = RN(x - hi), lo = RN(x - hi - mid).
// The differences are exact in the source precision, so hi + mid + lo carries 24 bits.
__device__ __forceinline__ void split3(double x, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l)
{
    h = __double2bfloat16(x);
    const double r1 = x - (double)__bfloat162float(h);
    m = __double2bfloat16(r1);
    const double r2 = r1 - (double)__bfloat162float(m);
    l = __double2bfloat16(r2);
}
__device__ __forceinline__ void split3(float x, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l)
{
    h = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(h);
    m = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(m);
    l = __float2bfloat16_rn(r2);
}

// Eight FP32 values -> their three bf16 parts, 16 bytes each (value e in bytes 2e, 2e + 1):
// the same round-to-nearest splits as split3, two values per conversion.
__device__ __forceinline__ void split3x8(const float (&x)[8], uint4 &h, uint4 &m, uint4 &l)
{
    uint32_t ph[4], pm[4], pl[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float a = x[2 * i], b = x[2 * i + 1];
        uint32_t p;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(p) : "f"(b), "f"(a));  // upper half: b
        const float ra = a - __uint_as_float(p << 16), rb = b - __uint_as_float(p & 0xFFFF0000u);
        ph[i] = p;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(p) : "f"(rb), "f"(ra));
        const float sa = ra - __uint_as_float(p << 16), sb = rb - __uint_as_float(p & 0xFFFF0000u);
        pm[i] = p;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(p) : "f"(sb), "f"(sa));
        pl[i] = p;
    }
    h = make_uint4(ph[0], ph[1], ph[2], ph[3]);
    m = make_uint4(pm[0], pm[1], pm[2], pm[3]);
    l = make_uint4(pl[0], pl[1], pl[2], pl[3]);
}

}  // namespace tc
}  // namespace mxb
