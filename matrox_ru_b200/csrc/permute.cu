// Row permutation between the caller's point order and the evaluator's leaf-blocked
// tree order (matroxTest-V1/hcds.h:766-788 `transform`; its inverse is new: the
// reference leaves Y in tree order, matroxTest-V1/Util.h:320).
//
// A 32 x 32 tile (32 tree positions x 32 right-hand sides) is staged in shared memory so
// both sides stay coalesced whatever the caller's strides: a row-major (N, r) matrix is
// walked along r, a leaf-blocked column-major block along the tree positions.  Pure data
// movement: bound by HBM bandwidth.
#include "mxb_internal.h"

namespace mxb {
namespace {

constexpr int T = 32;

__device__ __forceinline__ int leaf_of(const int32_t *leafofs, int nleaf, int64_t t)
{
    int lo = 0, hi = nleaf;  // leafofs[lo] <= t < leafofs[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (leafofs[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// dir 0: TW[block(t), j] = W[perm[t], j];  dir 1: Y[perm[t], j] (+)= TY[block(t), j]
__global__ void permute_kernel(const int32_t *__restrict__ perm, const int32_t *__restrict__ leafofs,
                               const int32_t *__restrict__ blockofs, int nleaf, int64_t n,
                               const double *__restrict__ src, double *__restrict__ dst, int64_t rs,
                               int64_t cs, int nrhs, int dir, int accumulate)
{
    __shared__ double tile[T][T + 1];  // [position][column]
    __shared__ int64_t qbase[T];       // leaf-blocked offset of each position's column 0
    __shared__ int32_t qld[T];         // its leaf's row count (the block's leading dimension)
    const int64_t t0 = (int64_t)blockIdx.x * T;
    const int j0 = blockIdx.y * T;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const bool caller_j_fast = cs < rs;
    if (ty == 0 && t0 + tx < n) {  // one leaf lookup per position, not per element
        const int64_t t = t0 + tx;
        const int leaf = leaf_of(leafofs, nleaf, t);
        qbase[tx] = (int64_t)blockofs[leaf] + (t - leafofs[leaf]);
        qld[tx] = leafofs[leaf + 1] - leafofs[leaf];
    }
    __syncthreads();
    for (int phase = 0; phase < 2; ++phase) {
        const bool caller_side = (phase == 0) == (dir == 0);
        const bool j_fast = caller_side && caller_j_fast;
        for (int r = ty; r < T; r += 8) {
            const int a = j_fast ? r : tx;
            const int b = j_fast ? tx : r;
            const int64_t t = t0 + a;
            const int j = j0 + b;
            if (t >= n || j >= nrhs) continue;
            if (caller_side) {
                const int64_t p = (int64_t)perm[t] * rs + (int64_t)j * cs;
                if (phase == 0) tile[a][b] = src[p];
                else dst[p] = accumulate ? dst[p] + tile[a][b] : tile[a][b];
            } else {
                const int64_t q = qbase[a] + (int64_t)j * qld[a];
                if (phase == 0) tile[a][b] = src[q];
                else dst[q] = tile[a][b];
            }
        }
        if (phase == 0) __syncthreads();
    }
}

}  // namespace

cudaError_t launch_permute(const int32_t *perm, const int32_t *leafofs, const int32_t *blockofs, int nleaf,
                           int64_t n, const double *src, double *dst, int64_t rs, int64_t cs, int nrhs,
                           int dir, int accumulate, cudaStream_t stream)
{
    if (n <= 0 || nrhs <= 0) return cudaSuccess;
    dim3 grid((unsigned)((n + T - 1) / T), (nrhs + T - 1) / T);
    dim3 block(T, 8);
    permute_kernel<<<grid, block, 0, stream>>>(perm, leafofs, blockofs, nleaf, n, src, dst, rs, cs, nrhs, dir,
                                               accumulate);
    return cudaGetLastError();
}

}  // namespace mxb
