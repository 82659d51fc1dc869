// Kernel-matrix blocks of the CDS computed on the GPU from the points.
//
// The reference builds every near block D_xy and far coupling B_xy on the host with
// Fsubmatrix (matroxTest-V1/compression.h:256-360): the block K(X[rows], X[cols]) of the
// points of two index sets (leaf points for near blocks, skeleton points for far couplings),
// stored column-major (element (i, j) at i + j * rows), and packed at the offsets Dptr / Bptr
// by CacheNear / CacheFar (matroxTest-V1/hcds.h:339-460).  Here one kernel fills any list of
// such blocks: a CTA computes a 64 x 64 tile of one block from the tile's row and column
// points staged in shared memory, squared distances summed coordinate by coordinate in FP64,
// then the kernel function.  The output writes are coalesced along the block's rows.  At
// d = 28 the work is bound by the FP64 arithmetic (d FMAs and one exp per element), not by the
// writes (8 bytes per element).
#include <algorithm>
#include <string>
#include <vector>

#include "matrox_b200.h"
#include "mxb_internal.h"

namespace mxb {
namespace {

constexpr int TILE = 64, THREADS = 256, MAX_DIM = 128;

struct BlockTile {
    uint64_t out;      // element offset of the block in the output
    int64_t rows0;     // start of the row set in the index list
    int64_t cols0;     // start of the column set
    int32_t nrows;     // rows of the block (its leading dimension)
    int32_t ncols;
    int32_t r0, c0;    // this tile's first row and column
};

__device__ __forceinline__ double kernel_value(double d2, int kind, double s)
{
    // s: -1 / (2 h^2) for the Gaussian, 1 / h^2 for the inverse multiquadric
    if (kind == MXB_KERNEL_GAUSSIAN) return exp(s * d2);
    if (kind == MXB_KERNEL_IMQ) return rsqrt(1.0 + s * d2);
    return d2 == 0.0 ? 1.0 : rsqrt(d2);  // 1 / |x - y|, 1 on coincident points
}

__global__ void __launch_bounds__(THREADS) kernel_block_kernel(const BlockTile *__restrict__ tiles,
                                                               const int32_t *__restrict__ idx,
                                                               const double *__restrict__ X, int d, int kind,
                                                               double s, double *__restrict__ out)
{
    extern __shared__ double pts[];  // [2][TILE][d + 1]: row points, then column points
    const int ld = d + 1;            // odd pitch: the per-coordinate reads below hit distinct banks
    double *P = pts, *Q = pts + TILE * ld;
    const BlockTile t = tiles[blockIdx.x];
    const int nr = min(TILE, t.nrows - t.r0), nc = min(TILE, t.ncols - t.c0);
    for (int e = threadIdx.x; e < TILE * d; e += THREADS) {
        const int p = e / d, k = e - p * d;
        P[p * ld + k] = p < nr ? X[(int64_t)idx[t.rows0 + t.r0 + p] * d + k] : 0.0;
        Q[p * ld + k] = p < nc ? X[(int64_t)idx[t.cols0 + t.c0 + p] * d + k] : 0.0;
    }
    __syncthreads();
    // thread (tr, tc): rows tr + 16 a and columns tc + 16 b (a, b < 4), a 4 x 4 register
    // block: 8 shared-memory loads per coordinate for 16 FMAs; the writes of 16 consecutive
    // threads cover 16 consecutive rows of a column
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    double d2[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) d2[a][b] = 0.0;
    for (int k = 0; k < d; ++k) {
        double pa[4], qb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) pa[a] = P[(tr + 16 * a) * ld + k];
#pragma unroll
        for (int b = 0; b < 4; ++b) qb[b] = Q[(tc + 16 * b) * ld + k];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const double diff = pa[a] - qb[b];
                d2[a][b] = fma(diff, diff, d2[a][b]);
            }
    }
    double *o = out + t.out + (uint64_t)t.r0 + (uint64_t)t.c0 * (uint64_t)t.nrows;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = tc + 16 * b;
        if (j >= nc) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tr + 16 * a;
            if (i < nr) o[(uint64_t)i + (uint64_t)j * t.nrows] = kernel_value(d2[a][b], kind, s);
        }
    }
}

int fail_arg(const std::string &m, int code = MXB_ERR_ARG)
{
    set_error("mxb_kernel_blocks: " + m);
    return code;
}

}  // namespace
}  // namespace mxb

using namespace mxb;

extern "C" int32_t mxb_kernel_blocks(const double *dX, int64_t n, int32_t d, int32_t kind, double h,
                                     const int64_t *set_ofs, const int32_t *set_idx, int32_t nsets,
                                     const int32_t *blk_row, const int32_t *blk_col, const uint64_t *blk_ofs,
                                     int32_t nblk, double *dOut, uint64_t out_len, void *stream)
{
    if (!dX || !set_ofs || !set_idx || (nblk > 0 && (!blk_row || !blk_col || !blk_ofs || !dOut)))
        return fail_arg("null argument");
    if (n < 1 || d < 1 || nsets < 0 || nblk < 0) return fail_arg("bad sizes");
    if (d > MAX_DIM) return fail_arg("point dimension above " + std::to_string(MAX_DIM), MXB_ERR_UNSUPPORTED);
    if (kind != MXB_KERNEL_GAUSSIAN && kind != MXB_KERNEL_IMQ && kind != MXB_KERNEL_NEWTON)
        return fail_arg("unknown kernel kind");
    if (kind != MXB_KERNEL_NEWTON && !(h > 0)) return fail_arg("kernel bandwidth must be positive");
    if (set_ofs[0] != 0) return fail_arg("set offsets must start at 0");
    for (int s = 0; s < nsets; ++s)
        if (set_ofs[s + 1] < set_ofs[s]) return fail_arg("set offsets not monotone", MXB_ERR_STRUCTURE);
    const int64_t nidx = set_ofs[nsets];
    for (int64_t e = 0; e < nidx; ++e)
        if (set_idx[e] < 0 || set_idx[e] >= n) return fail_arg("point index out of range", MXB_ERR_STRUCTURE);
    std::vector<BlockTile> tiles;
    for (int b = 0; b < nblk; ++b) {
        const int r = blk_row[b], c = blk_col[b];
        if (r < 0 || r >= nsets || c < 0 || c >= nsets) return fail_arg("block set out of range", MXB_ERR_STRUCTURE);
        const int64_t nr = set_ofs[r + 1] - set_ofs[r], nc = set_ofs[c + 1] - set_ofs[c];
        if (nr > INT32_MAX || nc > INT32_MAX) return fail_arg("set too large", MXB_ERR_UNSUPPORTED);
        if (blk_ofs[b] + (uint64_t)nr * (uint64_t)nc > out_len)
            return fail_arg("block past the end of the output", MXB_ERR_STRUCTURE);
        for (int r0 = 0; r0 < nr; r0 += TILE)
            for (int c0 = 0; c0 < nc; c0 += TILE)
                tiles.push_back(BlockTile{blk_ofs[b], set_ofs[r], set_ofs[c], (int32_t)nr, (int32_t)nc, r0, c0});
    }
    if (tiles.empty()) return MXB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    BlockTile *dTiles = nullptr;
    int32_t *dIdx = nullptr;
    cudaError_t e = cudaMallocAsync(&dTiles, tiles.size() * sizeof(BlockTile), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dIdx, std::max<int64_t>(nidx, 1) * sizeof(int32_t), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dTiles, tiles.data(), tiles.size() * sizeof(BlockTile), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && nidx)
        e = cudaMemcpyAsync(dIdx, set_idx, nidx * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    const size_t smem = 2 * (size_t)TILE * (d + 1) * sizeof(double);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const double sc = kind == MXB_KERNEL_GAUSSIAN ? -0.5 / (h * h) : (kind == MXB_KERNEL_IMQ ? 1.0 / (h * h) : 0.0);
    if (e == cudaSuccess) {
        kernel_block_kernel<<<(unsigned)tiles.size(), THREADS, smem, s>>>(dTiles, dIdx, dX, d, kind, sc, dOut);
        e = cudaGetLastError();
    }
    if (dTiles) cudaFreeAsync(dTiles, s);
    if (dIdx) cudaFreeAsync(dIdx, s);
    if (e != cudaSuccess) return fail_arg(cudaGetErrorString(e), MXB_ERR_CUDA);
    return MXB_OK;
}
