// Plans over a device layout the caller owns (hbdia_plan_create): the HBDIA
// arrays exactly as the reference's prepareForGPU leaves them on the device
// (src/Format/HBDIA.cpp:720-816; getters include/Format/HBDIA.hpp:155-165) --
// values [block][offsetIdx][lane] at blockStart * blockWidth, the flattened
// ascending offsets, blockStartIndices (numBlocks + 1, offset units), and the
// row-sorted COO remainder with its CSR row pointer -- run through this
// library's fused kernels without a copy.  The plan borrows those arrays and
// owns only a small allocation: the COO range of every 32-row tile (derived
// from the row pointer on the device) and the status word of the bounded
// waits.
//
// The arrays are checked on the device before the plan is returned (block
// starts from 0 to totalOffsets and non-decreasing, the row pointer from 0 to
// numCoo and non-decreasing, every COO row consistent with it and every COO
// column inside the matrix), so a malformed layout is refused instead of
// being read out of bounds.  Offsets need no check: the kernels bound every
// column.
#include <cuda_runtime.h>

#include <algorithm>

#include "hbdia_internal.hpp"

namespace hbdia {
namespace {

// flags: 1 block starts, 2 row pointer, 4 COO row vs row pointer, 8 COO column
__global__ void check_layout(const int32_t *__restrict__ blk, int32_t nb, int64_t total,
                             const int32_t *__restrict__ rp, const int32_t *__restrict__ cr,
                             const int32_t *__restrict__ cc, int32_t n, int32_t nCols, int64_t nCoo,
                             int32_t *__restrict__ flags) {
    int32_t f = 0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t b = i0; b <= nb; b += stride) {
        const int32_t v = blk[b];
        if (b == 0 && v != 0) f |= 1;
        if (b == nb && v != total) f |= 1;
        if (b > 0 && blk[b - 1] > v) f |= 1;
    }
    if (nCoo > 0) {
        for (int64_t r = i0; r <= n; r += stride) {
            const int32_t v = rp[r];
            if (r == 0 && v != 0) f |= 2;
            if (r == n && v != nCoo) f |= 2;
            if (r > 0 && rp[r - 1] > v) f |= 2;
            if (v < 0 || v > nCoo) f |= 2;
        }
        for (int64_t e = i0; e < nCoo; e += stride) {
            const int32_t r = cr[e], c = cc[e];
            if (r < 0 || r >= n) {
                f |= 4;
            } else {
                const int32_t a = rp[r], z = rp[r + 1];
                if (a < 0 || z > nCoo || e < a || e >= z) f |= 4;
            }
            if (c < 0 || c >= nCols) f |= 8;
        }
    }
    if (f) atomicOr(flags, f);
}

// cooTile[t] = rowPtr[min(32 t, n)]: the COO range of each 32-row tile.
__global__ void tile_ranges(const int32_t *__restrict__ rp, int32_t n, int32_t numTiles, bool hasCoo,
                            int32_t *__restrict__ tile) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > numTiles) return;
    tile[t] = hasCoo ? rp[std::min<int64_t>(t * 32, n)] : 0;
}

inline size_t up256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

}  // namespace

void borrow_plan(const hbdia_layout_desc &d, DevicePlan &P) {
    if (d.dtype != HBDIA_F64 && d.dtype != HBDIA_F32) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (d.storage < HBDIA_STORE_NATIVE || d.storage > HBDIA_STORE_BF16_SCALED)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown value storage");
    if (d.dtype == HBDIA_F32 && d.storage != HBDIA_STORE_NATIVE)
        throw Error(HBDIA_ERR_UNSUPPORTED, "reduced value storage needs a double layout");
    if (d.numRows <= 0 || d.numCols <= 0 || d.blockWidth <= 0 || d.numBlocks < 0 || d.totalOffsets < 0 ||
        d.numCoo < 0)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad layout sizes");
    const int64_t maxBlocks = (static_cast<int64_t>(std::min(d.numRows, d.numCols)) + d.blockWidth - 1) / d.blockWidth;
    if (d.numBlocks > maxBlocks)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "numBlocks exceeds ceil(min(numRows, numCols) / blockWidth)");
    if (d.totalOffsets > 0 && (!d.values || !d.offsets))
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null values or offsets");
    if (!d.blockStart) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null blockStart");
    if (d.storage == HBDIA_STORE_BF16_SCALED && d.numBlocks > 0 && !d.scales)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bf16 storage needs the per-block scales");
    if (d.numCoo > 0 && (!d.cooRow || !d.cooCol || !d.cooVal || !d.cooRowPtr))
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null COO array");
    if (d.numCoo > INT32_MAX || d.totalOffsets > INT32_MAX)
        throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^31-1 offsets or COO entries");

    DevicePlan Q;
    Q.dtype = d.dtype;
    Q.storage = d.storage;
    Q.n = d.numRows;
    Q.numCols = d.numCols;
    Q.xn = d.numRows;  // the reference's bound: columns in [0, numRows)
    Q.bw = d.blockWidth;
    Q.numBlocks = d.numBlocks;
    Q.numTiles = static_cast<int32_t>((static_cast<int64_t>(d.numRows) + 31) / 32);
    Q.totalOffsets = d.totalOffsets;
    Q.slots = d.totalOffsets * d.blockWidth;
    Q.nCoo = d.numCoo;
    Q.vals = const_cast<void *>(d.values);
    Q.scale = d.storage == HBDIA_STORE_BF16_SCALED ? const_cast<float *>(d.scales) : nullptr;
    Q.offs = const_cast<int32_t *>(d.offsets);
    Q.blkOff = const_cast<int32_t *>(d.blockStart);
    Q.cooRow = const_cast<int32_t *>(d.cooRow);
    Q.cooCol = const_cast<int32_t *>(d.cooCol);
    Q.cooVal = const_cast<void *>(d.cooVal);
    Q.cooRowPtr = const_cast<int32_t *>(d.cooRowPtr);
    // owned: tile ranges, status word, check flags
    const size_t oTile = 0;
    const size_t oStatus = up256((static_cast<size_t>(Q.numTiles) + 1) * sizeof(int32_t));
    const size_t oFlags = oStatus + 256;
    Q.bytes = oFlags + 256;
    check_cuda(dev_alloc(&Q.base, Q.bytes), "cudaMalloc(plan)");
    try {
        char *base = static_cast<char *>(Q.base);
        Q.cooTile = reinterpret_cast<int32_t *>(base + oTile);
        Q.status = reinterpret_cast<int32_t *>(base + oStatus);
        int32_t *flags = reinterpret_cast<int32_t *>(base + oFlags);
        check_cuda(cudaMemset(Q.status, 0, sizeof(int32_t)), "cudaMemset(status)");
        check_cuda(cudaMemset(flags, 0, sizeof(int32_t)), "cudaMemset(flags)");
        const int64_t work = std::max<int64_t>({static_cast<int64_t>(d.numBlocks) + 1, d.numCoo,
                                                static_cast<int64_t>(d.numRows) + 1});
        const unsigned grid = static_cast<unsigned>(std::min<int64_t>((work + 255) / 256, 148 * 8));
        check_layout<<<grid, 256>>>(Q.blkOff, Q.numBlocks, Q.totalOffsets, Q.cooRowPtr, Q.cooRow, Q.cooCol, Q.n,
                                    Q.numCols, Q.nCoo, flags);
        check_cuda(cudaGetLastError(), "check_layout");
        int32_t f = 0;
        check_cuda(cudaMemcpy(&f, flags, sizeof(int32_t), cudaMemcpyDeviceToHost), "cudaMemcpy(flags)");
        if (f & 1) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "blockStart is not 0 .. totalOffsets non-decreasing");
        if (f & 2) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "cooRowPtr is not 0 .. numCoo non-decreasing");
        if (f & 4) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "COO rows disagree with cooRowPtr (not row-sorted)");
        if (f & 8) throw Error(HBDIA_ERR_OUT_OF_RANGE, "a COO column lies outside the matrix");
        tile_ranges<<<static_cast<unsigned>((Q.numTiles + 1 + 255) / 256), 256>>>(Q.cooRowPtr, Q.n, Q.numTiles,
                                                                                  Q.nCoo > 0, Q.cooTile);
        check_cuda(cudaGetLastError(), "tile_ranges");
        cudaStream_t s;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        Q.stream = s;
        check_cuda(cudaGetDevice(&Q.device), "cudaGetDevice");
        check_cuda(cudaDeviceSynchronize(), "plan set-up");
    } catch (...) {
        free_plan(Q);
        throw;
    }
    const int64_t vsz = d.storage == HBDIA_STORE_NATIVE ? (d.dtype == HBDIA_F32 ? 4 : 8)
                        : d.storage == HBDIA_STORE_F32 ? 4 : 2;
    const int64_t xs = d.dtype == HBDIA_F32 ? 4 : 8;
    int64_t bytes = Q.slots * vsz + 4 * Q.totalOffsets + 4 * (static_cast<int64_t>(Q.numBlocks) + 1) +
                    2 * xs * Q.n + (8 + xs) * Q.nCoo + xs * Q.nCoo;
    if (Q.scale) bytes += 4 * static_cast<int64_t>(Q.numBlocks);
    if (Q.nCoo > 0) bytes += Q.bw == 32 ? 4 * (static_cast<int64_t>(Q.numTiles) + 1) : 4 * (static_cast<int64_t>(Q.n) + 1);
    Q.bytesPerSpmv = bytes;
    P = Q;
}

}  // namespace hbdia
