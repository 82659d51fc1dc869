// Batched column interpolative decomposition (ID) on the GPU: the compression step of the
// CDS, matroxTest-V1/compression.h:446-523 `decomposition`, which the reference runs on the
// host per tree node with LAPACKE_dgeqp3 followed by cblas_dtrsm.
//
// One CTA per node matrix A (nrows x ncols, column-major, nrows samples of the kernel against
// ncols candidate points), in place in global memory:
//   1. Householder QR with column pivoting.  The pivot of step i is the first column of
//      largest remaining norm; the norms are downdated after every step and recomputed where
//      the downdate has cancelled (LAPACK's dlaqp2 / dlaqps recurrence, tolerance
//      sqrt(machine epsilon)).
//   2. The reference's rank rule: s is the first s >= 1 with |R[s,s] / R[0,0]| < tol, at most
//      max_rank and at most min(nrows, ncols).  The QR stops there: only R[0:s, :] is needed.
//   3. P (s x ncols) with R11 P[:, piv] = R[0:s, :] by back substitution (upper triangular
//      R11), columns in parallel.  If R[0,0] == 0 (a zero matrix), P = 0: the reference then
//      returns R's upper rows, which are zero, without the solve.
// The factorisation is a sequence of rank-1 steps over the trailing matrix, each bound by
// the memory traffic of that matrix (L2 for a few nodes in flight, HBM beyond).
#include <cfloat>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"

namespace mxb {
namespace {

constexpr int MAX_COLS = 8192;  // shared memory holds 20 bytes per column

struct IdJob {
    uint64_t a_off;    // A: nrows x ncols, column-major (leading dimension nrows)
    uint64_t p_off;    // P and its scratch: pmax x ncols each, pmax = min(max_rank, ncols)
    uint64_t piv_off;  // ncols pivots
    int32_t nrows, ncols;
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block; every thread gets the result.  `red` holds WARPS + 1 doubles.
template <int THREADS>
__device__ double block_sum(double v, double *red)
{
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < WARPS ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[WARPS] = t;
    }
    __syncthreads();
    const double r = red[WARPS];
    __syncthreads();  // red is reused by the next call
    return r;
}

// First index of the largest value in x[lo, hi); every thread gets it.
template <int THREADS>
__device__ int block_argmax(const double *x, int lo, int hi, double *redv, int *redi)
{
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double bv = -1.0;
    int bi = hi;
    for (int j = lo + threadIdx.x; j < hi; j += THREADS)
        if (x[j] > bv) {  // ascending j per thread: the first of equal values stays
            bv = x[j];
            bi = j;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    if (lane == 0) {
        redv[warp] = bv;
        redi[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < WARPS; ++w)
            if (redv[w] > redv[0] || (redv[w] == redv[0] && redi[w] < redi[0])) {
                redv[0] = redv[w];
                redi[0] = redi[w];
            }
        redi[WARPS] = redi[0] < hi ? redi[0] : lo;
    }
    __syncthreads();
    const int r = redi[WARPS];
    __syncthreads();
    return r;
}

// THREADS: 256 when the launch has enough nodes to fill the GPU, 1024 (more warps on the
// trailing columns of one node) when it has fewer nodes than SMs.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) id_qrcp_kernel(const IdJob *__restrict__ jobs, double *__restrict__ A,
                                                          double *__restrict__ P, double *__restrict__ Z,
                                                          int32_t *__restrict__ piv, int32_t *__restrict__ rank,
                                                          double tol, int max_rank)
{
    constexpr int WARPS = THREADS / 32;
    extern __shared__ double sm[];
    __shared__ double red[WARPS + 1];
    __shared__ int redi[WARPS + 1];
    __shared__ double s_beta, s_tau, s_scale;
    const IdJob jb = jobs[blockIdx.x];
    const int ns = jb.nrows, nc = jb.ncols;
    const int pmax = min(max_rank, nc);
    double *a = A + jb.a_off;
    double *vn1 = sm, *vn2 = sm + nc;
    int *jp = reinterpret_cast<int *>(sm + 2 * nc);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double tol3z = sqrt(DBL_EPSILON / 2);  // sqrt of LAPACK's relative machine epsilon

    // ---- column norms ----
    for (int j = warp; j < nc; j += WARPS) {
        const double *col = a + (size_t)j * ns;
        double t = 0.0;
        for (int r = lane; r < ns; r += 32) t += col[r] * col[r];
        t = warp_sum(t);
        if (lane == 0) vn1[j] = vn2[j] = sqrt(t);
    }
    for (int j = threadIdx.x; j < nc; j += THREADS) jp[j] = j;
    __syncthreads();

    // ---- pivoted Householder QR up to the rank ----
    const int kmax = min(ns, nc);
    int s = min(kmax, max_rank);
    double r00 = 0.0;
    for (int i = 0; i < kmax; ++i) {
        if (i >= max_rank) break;  // s = max_rank
        const int p = block_argmax<THREADS>(vn1, i, nc, red, redi);
        if (p != i) {
            double *ci = a + (size_t)i * ns, *cp = a + (size_t)p * ns;
            for (int r = threadIdx.x; r < ns; r += THREADS) {
                const double t = ci[r];
                ci[r] = cp[r];
                cp[r] = t;
            }
            if (threadIdx.x == 0) {
                const int tj = jp[i];
                jp[i] = jp[p];
                jp[p] = tj;
                vn1[p] = vn1[i];
                vn2[p] = vn2[i];
            }
        }
        __syncthreads();
        // reflector for a[i:, i] (dlarfg): beta = -sign(alpha) |x|, v = x[1:] / (alpha - beta)
        double *ci = a + (size_t)i * ns;
        double x2 = 0.0;
        for (int r = i + 1 + threadIdx.x; r < ns; r += THREADS) x2 += ci[r] * ci[r];
        x2 = block_sum<THREADS>(x2, red);
        if (threadIdx.x == 0) {
            const double alpha = ci[i];
            const double xnorm = sqrt(x2);
            if (xnorm == 0.0) {
                s_beta = alpha;
                s_tau = 0.0;
                s_scale = 0.0;
            } else {
                const double beta = -copysign(hypot(alpha, xnorm), alpha);
                s_beta = beta;
                s_tau = (beta - alpha) / beta;
                s_scale = 1.0 / (alpha - beta);
            }
        }
        __syncthreads();
        const double beta = s_beta, tau = s_tau, scale = s_scale;
        // the rank rule looks at R[i, i] = beta
        if (i == 0) {
            r00 = beta;
        } else if (r00 != 0.0 && fabs(beta / r00) < tol) {
            s = i;
            break;
        }
        if (tau != 0.0)
            for (int r = i + 1 + threadIdx.x; r < ns; r += THREADS) ci[r] *= scale;
        __syncthreads();
        if (threadIdx.x == 0) ci[i] = beta;
        // apply I - tau v v^T (v = [1; a[i+1:, i]]) to the columns right of i, one warp per
        // column, then downdate that column's norm
        for (int j = i + 1 + warp; j < nc; j += WARPS) {
            double *cj = a + (size_t)j * ns;
            double w = 0.0;
            if (tau != 0.0) {
                for (int r = i + 1 + lane; r < ns; r += 32) w += ci[r] * cj[r];
                w = warp_sum(w) + cj[i];
                w *= tau;
                for (int r = i + 1 + lane; r < ns; r += 32) cj[r] -= w * ci[r];
            }
            __syncwarp();
            double rij = cj[i];
            if (lane == 0 && tau != 0.0) {
                rij -= w;
                cj[i] = rij;
            }
            rij = __shfl_sync(0xffffffffu, rij, 0);
            const double v1 = vn1[j];
            bool recompute = false;
            if (v1 != 0.0) {
                double t = fabs(rij) / v1;
                t = fmax(0.0, (1.0 + t) * (1.0 - t));
                const double q = v1 / vn2[j];
                if (t * q * q <= tol3z) recompute = true;
                else if (lane == 0) vn1[j] = v1 * sqrt(t);
            }
            if (recompute) {  // uniform across the warp
                double t = 0.0;
                for (int r = i + 1 + lane; r < ns; r += 32) t += cj[r] * cj[r];
                t = warp_sum(t);
                if (lane == 0) vn1[j] = vn2[j] = i + 1 < ns ? sqrt(t) : 0.0;
            }
        }
        __syncthreads();
    }
    s = max(1, min(s, pmax));

    // ---- outputs: rank, pivots, P = R11^{-1} R[0:s, :] with columns in pivot order ----
    int32_t *pv = piv + jb.piv_off;
    for (int j = threadIdx.x; j < nc; j += THREADS) pv[j] = jp[j];
    if (threadIdx.x == 0) rank[blockIdx.x] = s;
    double *pout = P + jb.p_off;  // s x nc, leading dimension s
    if (r00 == 0.0) {
        for (int e = threadIdx.x; e < s * nc; e += THREADS) pout[e] = 0.0;
        return;
    }
    // z[k][j] (row-major, j fastest: coalesced across the threads) = R[k, j]
    double *z = Z + jb.p_off;
    for (int k = 0; k < s; ++k)
        for (int j = threadIdx.x; j < nc; j += THREADS)
            z[(size_t)k * nc + j] = (j >= k || j >= s) ? a[k + (size_t)j * ns] : 0.0;
    __syncthreads();
    // back substitution, all columns at once: x_k = z_k / R[k,k], then z_t -= x_k R[t,k], t < k
    for (int k = s - 1; k >= 0; --k) {
        const double *rk = a + (size_t)k * ns;  // column k of R11
        double *zk = z + (size_t)k * nc;
        for (int j = threadIdx.x; j < nc; j += THREADS) {
            const double x = zk[j] / rk[k];
            zk[j] = x;
            for (int t = 0; t < k; ++t) z[(size_t)t * nc + j] -= x * rk[t];
        }
    }
    __syncthreads();
    for (int k = 0; k < s; ++k)
        for (int j = threadIdx.x; j < nc; j += THREADS) pout[k + (size_t)jp[j] * s] = z[(size_t)k * nc + j];
}

int fail_id(const std::string &m, int code = MXB_ERR_ARG)
{
    set_error("mxb_batched_id: " + m);
    return code;
}

}  // namespace
}  // namespace mxb

using namespace mxb;

extern "C" int32_t mxb_batched_id(double *dA, const int32_t *nrows, const int32_t *ncols, int32_t count, double tol,
                                  int32_t max_rank, int32_t *dRank, int32_t *dPiv, double *dP, void *stream)
{
    if (count < 0) return fail_id("negative count");
    if (count == 0) return MXB_OK;
    if (!dA || !nrows || !ncols || !dRank || !dPiv || !dP) return fail_id("null argument");
    if (max_rank < 1) return fail_id("max_rank must be >= 1");
    if (!(tol >= 0.0)) return fail_id("tolerance must be >= 0");
    std::vector<IdJob> jobs((size_t)count);
    uint64_t a = 0, p = 0, q = 0;
    int maxc = 1;
    for (int b = 0; b < count; ++b) {
        const int ns = nrows[b], nc = ncols[b];
        if (ns < 1 || nc < 1) return fail_id("empty matrix");
        if (nc > MAX_COLS) return fail_id("more than " + std::to_string(MAX_COLS) + " columns", MXB_ERR_UNSUPPORTED);
        jobs[b] = IdJob{a, p, q, ns, nc};
        a += (uint64_t)ns * nc;
        p += (uint64_t)std::min(max_rank, nc) * nc;
        q += (uint64_t)nc;
        maxc = std::max(maxc, nc);
    }
    cudaStream_t s = (cudaStream_t)stream;
    IdJob *dJobs = nullptr;
    double *dZ = nullptr;
    cudaError_t e = cudaMallocAsync(&dJobs, jobs.size() * sizeof(IdJob), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dZ, std::max<uint64_t>(p, 1) * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dJobs, jobs.data(), jobs.size() * sizeof(IdJob), cudaMemcpyHostToDevice, s);
    const size_t smem = (size_t)maxc * (2 * sizeof(double) + sizeof(int));
    int dev = 0, sms = 148;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const bool wide = count < sms;
    if (e == cudaSuccess)
        e = wide ? cudaFuncSetAttribute(id_qrcp_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                 : cudaFuncSetAttribute(id_qrcp_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        if (wide)
            id_qrcp_kernel<1024><<<(unsigned)count, 1024, smem, s>>>(dJobs, dA, dP, dZ, dPiv, dRank, tol, max_rank);
        else
            id_qrcp_kernel<256><<<(unsigned)count, 256, smem, s>>>(dJobs, dA, dP, dZ, dPiv, dRank, tol, max_rank);
        e = cudaGetLastError();
    }
    if (dJobs) cudaFreeAsync(dJobs, s);
    if (dZ) cudaFreeAsync(dZ, s);
    if (e != cudaSuccess) return fail_id(cudaGetErrorString(e), MXB_ERR_CUDA);
    return MXB_OK;
}
