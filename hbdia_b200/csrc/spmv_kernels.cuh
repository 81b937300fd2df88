// Device-side kernels of the fused HBDIA SpMV (sm_100a).
//
// y = A x for A in HBDIA form: a blocked-DIA part (per row block of width bw,
// an ascending list of diagonal offsets, bw values per offset) plus a
// row-sorted COO remainder.  One launch computes both parts and writes every
// row of y once; the reference needs a DIA kernel, a separate COO SpMV and a
// vector_add kernel (src/Operations/HBDIASpMV.cu:7-88,
// src/Operations/HBDIASpMV.cpp:186-251).
//
// Arithmetic matches the reference's hbdiaSpMV bit for bit:
//  * DIA part: per row, offsets in ascending order, stored zeros and columns
//    outside [0, numRows) skipped, sum = fma(v, x[col], sum) -- what nvcc
//    makes of `sum += matrixValue * vectorValue` (src/Operations/HBDIASpMV.cu:42-71);
//  * COO part: per row, entries in list order, c = c + v * x[col] with a
//    separately rounded multiply and add -- the reference's host COO SpMV
//    (src/Operations/HBDIASpMV.cpp:76-92) built without FMA contraction;
//  * merge: y = dia + coo when the matrix has a COO remainder, else y = dia
//    (src/Operations/HBDIASpMV.cu:77-88, src/Operations/HBDIASpMV.cpp:235-250).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hbdia {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;

// Kernel arguments (device pointers into one plan allocation).
template <typename VT, typename XT>
struct SpmvArgs {
    const VT *vals;          // DIA values [slots], [block][offsetIdx][lane]
    const float *scale;      // per-block scale (bf16 storage) or nullptr
    const int32_t *offs;     // kept offsets, ascending per block
    const int32_t *blkOff;   // numBlocks + 1, offset units
    const int32_t *cooRow;   // row-sorted COO remainder
    const int32_t *cooCol;
    const XT *cooVal;
    const int32_t *cooRowPtr;  // numRows + 1 (row-per-thread kernel)
    const int32_t *cooTile;    // numTiles + 1 (warp kernels): COO range of each 32-row tile
    int32_t n;               // numRows
    int32_t xn;              // DIA column bound: numRows (the reference's col < numRows),
                             // or the x-window length of a partial matrix
    int32_t bw;              // blockWidth
    int32_t numBlocks;       // DIA blocks
    int32_t numTiles;        // ceil(n / 32)
    int32_t hasCoo;          // COO remainder non-empty
    int32_t quadLayout;      // 4- / 2-byte values of uniform quads interleaved (spmv_quad.cuh)
};

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Streaming loads of the value arrays (read once: evict-first, no L1 fill).
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16 *p) {
    unsigned short r = __ldcs(reinterpret_cast<const unsigned short *>(p));
    return __ushort_as_bfloat16(r);
}

// Stored value -> accumulation type.
template <typename XT>
__device__ __forceinline__ XT widen(double v, float) { return static_cast<XT>(v); }
template <typename XT>
__device__ __forceinline__ XT widen(float v, float) { return static_cast<XT>(v); }
template <typename XT>
__device__ __forceinline__ XT widen(__nv_bfloat16 v, float s) {
    return static_cast<XT>(__bfloat162float(v)) * static_cast<XT>(s);
}

// ---------------------------------------------------------------------------
// Row-per-thread kernel for any block width (the reference's thread mapping),
// with the row's COO entries summed through the CSR row pointer.
template <typename VT, typename XT>
__global__ void __launch_bounds__(256)
spmv_rowwise(const SpmvArgs<VT, XT> a, const XT *__restrict__ x, XT *__restrict__ y) {
    const int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (row >= a.n) return;
    XT sum = XT(0);
    const int32_t b = static_cast<int32_t>(row / a.bw);
    const int32_t lane = static_cast<int32_t>(row - static_cast<int64_t>(b) * a.bw);
    if (b < a.numBlocks) {
        const int32_t k0 = __ldg(a.blkOff + b), k1 = __ldg(a.blkOff + b + 1);
        const float s = a.scale ? __ldg(a.scale + b) : 1.0f;
        for (int32_t k = k0; k < k1; ++k) {
            const XT v = widen<XT>(ld_stream(a.vals + static_cast<int64_t>(k) * a.bw + lane), s);
            if (v == XT(0)) continue;
            const int64_t col = row + __ldg(a.offs + k);
            if (col < 0 || col >= a.xn) continue;
            sum = fma_rn(v, __ldg(x + col), sum);
        }
    }
    if (a.hasCoo) {
        XT c = XT(0);
        const int32_t e1 = __ldg(a.cooRowPtr + row + 1);
        for (int32_t e = __ldg(a.cooRowPtr + row); e < e1; ++e)
            c = add_rn(c, mul_rn(__ldg(a.cooVal + e), __ldg(x + __ldg(a.cooCol + e))));
        sum = add_rn(sum, c);
    }
    y[row] = sum;
}

// ---------------------------------------------------------------------------
// COO remainder of one 32-row tile, summed by the warp: entries are loaded
// coalesced (32 per step), each lane forms one product, and the products are
// handed to their row's lane by warp shuffles in list order, so every row's
// sum keeps the sequential order of the reference.
template <typename XT>
__device__ __forceinline__ XT tile_coo(const int32_t *__restrict__ cooRow,
                                       const int32_t *__restrict__ cooCol,
                                       const XT *__restrict__ cooVal, int32_t e0, int32_t e1,
                                       int64_t tileRow0, int lane, const XT *__restrict__ x,
                                       XT c = XT(0)) {
    // c: this lane's row sum of the entries before e0 (continued in order)
    for (int32_t base = e0; base < e1; base += 32) {
        const int32_t e = base + lane;
        int lr = -1;
        XT p = XT(0);
        if (e < e1) {
            lr = static_cast<int>(__ldg(cooRow + e) - tileRow0);
            p = mul_rn(__ldg(cooVal + e), __ldg(x + __ldg(cooCol + e)));
        }
        const int m = min(32, e1 - base);
        for (int t = 0; t < m; ++t) {
            const int rt = __shfl_sync(kFull, lr, t);
            const XT pt = __shfl_sync(kFull, p, t);
            if (rt == lane) c = add_rn(c, pt);
        }
    }
    return c;
}

// ---------------------------------------------------------------------------
// blockWidth == 32: one warp per row block, lane = row within the block.
// The block's offsets are fetched once (one coalesced load of up to 32) and
// broadcast by shuffles; each offset's 32 values are one coalesced 256-byte
// (fp64) load; U offsets are in flight per lane at a time; x is read through
// L1, where the block's neighbouring diagonals (col, col+1, ...) and the
// neighbouring blocks of the same CTA hit the same lines.
template <typename VT, typename XT, int U>
__device__ __forceinline__ void bw32_tile(const SpmvArgs<VT, XT> &a, const XT *__restrict__ x, XT *__restrict__ y,
                                          int32_t tile, int lane) {
    const int64_t row0 = static_cast<int64_t>(tile) * 32;
    const int64_t row = row0 + lane;
    XT sum = XT(0);
    if (tile < a.numBlocks) {
        const int32_t k0 = __ldg(a.blkOff + tile), k1 = __ldg(a.blkOff + tile + 1);
        const float s = a.scale ? __ldg(a.scale + tile) : 1.0f;
        for (int32_t kb = k0; kb < k1; kb += 32) {
            const int cnt = min(32, k1 - kb);
            const int32_t myoff = lane < cnt ? __ldg(a.offs + kb + lane) : 0;
            const VT *vp = a.vals + static_cast<int64_t>(kb) * 32 + lane;
            int j = 0;
            for (; j + U <= cnt; j += U) {  // full groups: U values and x loads in flight
                VT v[U];
                XT xv[U];
                bool ok[U];
                int64_t col[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    col[u] = row + __shfl_sync(kFull, myoff, j + u);
                    ok[u] = static_cast<uint64_t>(col[u]) < static_cast<uint64_t>(a.xn);
                    v[u] = ld_stream(vp + static_cast<int64_t>(j + u) * 32);
                    xv[u] = XT(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (ok[u]) xv[u] = __ldg(x + col[u]);
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const XT vv = widen<XT>(v[u], s);
                    if (ok[u] && vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
                }
            }
            for (; j < cnt; ++j) {  // warp-uniform tail
                const int64_t col = row + __shfl_sync(kFull, myoff, j);
                const XT vv = widen<XT>(ld_stream(vp + static_cast<int64_t>(j) * 32), s);
                if (static_cast<uint64_t>(col) < static_cast<uint64_t>(a.xn) && vv != XT(0))
                    sum = fma_rn(vv, __ldg(x + col), sum);
            }
        }
    }
    if (a.hasCoo) {
        const int32_t e0 = __ldg(a.cooTile + tile), e1 = __ldg(a.cooTile + tile + 1);
        sum = add_rn(sum, tile_coo<XT>(a.cooRow, a.cooCol, a.cooVal, e0, e1, row0, lane, x));
    }
    if (row < a.n) __stcs(y + row, sum);
}

template <typename VT, typename XT, int U>
__global__ void __launch_bounds__(256)
spmv_bw32(const SpmvArgs<VT, XT> a, const XT *__restrict__ x, XT *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int32_t tile = static_cast<int32_t>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (tile >= a.numTiles) return;  // warp-uniform
    bw32_tile<VT, XT, U>(a, x, y, tile, lane);
}

// ---------------------------------------------------------------------------
// blockWidth == 32, persistent and software-pipelined across tiles.  Warp g of
// W walks tiles g, g + W, ... (neighbouring warps stay on neighbouring tiles,
// so x lines are shared through L1/L2).  While it computes tile t it already
// has tile t+W's block / COO pointers and first 32 offsets in registers (loaded
// during t-W) and the first 32 COO entries of tile t plus their x values in
// flight, so nearly every stall is a stall on value loads.  Same arithmetic
// and order as spmv_bw32.
struct TileMeta {
    int32_t k0, k1, c0, c1;
};

template <typename VT, typename XT>
__device__ __forceinline__ TileMeta load_meta(const SpmvArgs<VT, XT> &a, int32_t t) {
    TileMeta m{0, 0, 0, 0};
    if (t < a.numBlocks) {
        m.k0 = __ldg(a.blkOff + t);
        m.k1 = __ldg(a.blkOff + t + 1);
    }
    if (a.hasCoo && t < a.numTiles) {
        m.c0 = __ldg(a.cooTile + t);
        m.c1 = __ldg(a.cooTile + t + 1);
    }
    return m;
}

// Bulk prefetch of [p, p + bytes) into L2 (bytes a multiple of 16, p 16-byte
// aligned): a hint, no registers, no completion to wait for.
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// PF: one lane also asks L2 for tile t+W's value rows (up to 32 KB) while tile
// t is computed, so its value loads find them in L2.
// MT: the offsets after the last full group of U run as masked groups of 4
// (their loads in flight together) instead of one at a time.
template <typename VT, typename XT, int U, bool PF = false, bool MT = false>
__global__ void __launch_bounds__(256)
spmv_bw32_pipe(const SpmvArgs<VT, XT> a, const XT *__restrict__ x, XT *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int32_t W = static_cast<int32_t>((static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5);
    int32_t t = static_cast<int32_t>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (t >= a.numTiles) return;  // warp-uniform
    const uint32_t n = static_cast<uint32_t>(a.xn);  // column bound
    TileMeta m = load_meta(a, t);
    int32_t offNext = (lane < m.k1 - m.k0) ? __ldg(a.offs + m.k0 + lane) : 0;
    while (t < a.numTiles) {
        const int32_t tn = t + W;
        const TileMeta mn = tn < a.numTiles ? load_meta(a, tn) : TileMeta{0, 0, 0, 0};
        if (PF && lane == 0 && mn.k1 > mn.k0) {  // values of [k0, k1) are contiguous, 64-byte aligned
            const int64_t bytes = static_cast<int64_t>(mn.k1 - mn.k0) * 32 * static_cast<int64_t>(sizeof(VT));
            prefetch_l2_bulk(a.vals + static_cast<int64_t>(mn.k0) * 32,
                             static_cast<uint32_t>(bytes < 32768 ? bytes : 32768));
        }
        const int32_t row0 = t * 32;
        const int32_t row = row0 + lane;
        // first 32 COO entries of this tile and their x values, consumed at the end
        int lr = -1;
        XT cv = XT(0), cx = XT(0);
        int32_t ccol = 0;
        const int32_t ce = m.c0 + lane;
        const bool hasC = ce < min(m.c1, m.c0 + 32);
        if (hasC) {
            lr = __ldg(a.cooRow + ce) - row0;
            ccol = __ldg(a.cooCol + ce);
            cv = __ldg(a.cooVal + ce);
        }
        XT sum = XT(0);
        const float s = a.scale && t < a.numBlocks ? __ldg(a.scale + t) : 1.0f;
        int32_t myoff = offNext;
        bool gathered = false;
        // interior tile (at most 32 offsets, every column of every offset in
        // [0, n)): full groups skip the column checks, x read at x + row +
        // offset.  For 4- and 2-byte values only, where the instruction stream
        // co-limits the kernel; the 8-byte instance is bandwidth-bound and the
        // extra path would cost it registers (80 instead of 64: fewer warps).
        const int32_t K = m.k1 - m.k0;
        const bool interior = sizeof(VT) < 8 && K > 0 && K <= 32 && row0 + __shfl_sync(kFull, myoff, 0) >= 0 &&
                              static_cast<int64_t>(row0) + 31 + __shfl_sync(kFull, myoff, K > 0 && K <= 32 ? K - 1 : 0) <
                                  static_cast<int64_t>(a.xn);
        const XT *xr = x + row;
        (void)xr;
        for (int32_t kb = m.k0; kb < m.k1; kb += 32) {
            const int cnt = min(32, m.k1 - kb);
            if (kb != m.k0) myoff = lane < cnt ? __ldg(a.offs + kb + lane) : 0;
            const VT *vp = a.vals + static_cast<int64_t>(kb) * 32 + lane;
            int j = 0;
            if constexpr (sizeof(VT) < 8) {
                if (interior) {
                    for (; j + U <= cnt; j += U) {
                        VT v[U];
                        XT xv[U];
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            v[u] = ld_stream(vp + (j + u) * 32);
                            xv[u] = __ldg(xr + __shfl_sync(kFull, myoff, j + u));
                        }
                        if (!gathered) {  // COO columns have arrived by now
                            if (hasC) cx = __ldg(x + ccol);
                            gathered = true;
                        }
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const XT vv = widen<XT>(v[u], s);
                            if (vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
                        }
                    }
                }
            }
            for (; j + U <= cnt; j += U) {
                VT v[U];
                XT xv[U];
                bool ok[U];
                int32_t col[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    col[u] = row + __shfl_sync(kFull, myoff, j + u);
                    ok[u] = static_cast<uint32_t>(col[u]) < n;
                    v[u] = ld_stream(vp + (j + u) * 32);
                    xv[u] = XT(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (ok[u]) xv[u] = __ldg(x + col[u]);
                if (!gathered) {  // COO columns have arrived by now
                    if (hasC) cx = __ldg(x + ccol);
                    gathered = true;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const XT vv = widen<XT>(v[u], s);
                    if (ok[u] && vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
                }
            }
            if (MT) {
                // the last cnt - j < U offsets in masked groups of 4 (loads in flight together)
                for (; j < cnt; j += 4) {
                    const int rem = cnt - j;
                    VT v[4];
                    XT xv[4];
                    bool ok[4];
                    int32_t col[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const bool in = u < rem;  // warp-uniform
                        col[u] = row + __shfl_sync(kFull, myoff, in ? j + u : j);
                        ok[u] = in && static_cast<uint32_t>(col[u]) < n;
                        v[u] = in ? ld_stream(vp + (j + u) * 32) : VT(0);
                        xv[u] = XT(0);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (ok[u]) xv[u] = __ldg(x + col[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const XT vv = widen<XT>(v[u], s);
                        if (ok[u] && vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
                    }
                }
            } else {
                for (; j < cnt; ++j) {
                    const int32_t col = row + __shfl_sync(kFull, myoff, j);
                    const XT vv = widen<XT>(ld_stream(vp + j * 32), s);
                    if (static_cast<uint32_t>(col) < n && vv != XT(0)) sum = fma_rn(vv, __ldg(x + col), sum);
                }
            }
        }
        // next tile's first offsets (its pointers arrived during this tile)
        offNext = (lane < mn.k1 - mn.k0) ? __ldg(a.offs + mn.k0 + lane) : 0;
        if (a.hasCoo) {
            if (!gathered && hasC) cx = __ldg(x + ccol);
            XT c = XT(0);
            {
                const XT p = mul_rn(cv, cx);
                const int mcnt = min(32, m.c1 - m.c0);
                for (int q = 0; q < mcnt; ++q) {
                    const int rt = __shfl_sync(kFull, lr, q);
                    const XT pt = __shfl_sync(kFull, p, q);
                    if (rt == lane) c = add_rn(c, pt);
                }
            }
            if (m.c1 - m.c0 > 32)  // rare: more than 32 entries in the tile, continue in order
                c = tile_coo<XT>(a.cooRow, a.cooCol, a.cooVal, m.c0 + 32, m.c1, row0, lane, x, c);
            sum = add_rn(sum, c);
        }
        if (row < a.n) __stcs(y + row, sum);
        t = tn;
        m = mn;
    }
}

}  // namespace dev
}  // namespace hbdia
