// Multi-RHS product Y = A X on the HBDIA layout (sm_100a).
//
// X (n x k) and Y are row-major with leading dimensions ldx, ldy.  Column j of
// Y is computed with exactly the SpMV's arithmetic (ascending-offset FMA chain
// over the blocked-DIA values, sequential multiply-then-add over the row's COO
// entries, one final add), so it equals hbdia_spmv(A, X[:, j]) bit for bit.
//
// Each stored value is fetched from HBM once and used for every right-hand
// side: the RHS are processed in tiles of KT columns inside the warp that owns
// the row block, and the block's values (a few KB) stay in L1 between tiles.
#pragma once

#include "spmv_kernels.cuh"

namespace hbdia {
namespace dev {

// X[col][r0 .. r0+KT) of this lane's column: paired 16-byte loads when the row
// segment is aligned, else scalar loads.
template <typename XT, int KT>
__device__ __forceinline__ void load_x_row(const XT *__restrict__ p, int kc, bool vec2, XT (&xv)[KT]) {
    if (sizeof(XT) == 8 && vec2) {
#pragma unroll
        for (int q = 0; q < KT; q += 2) {
            if (q < kc) {
                const double2 d = __ldg(reinterpret_cast<const double2 *>(p) + q / 2);
                xv[q] = static_cast<XT>(d.x);
                if (q + 1 < KT) xv[q + 1] = static_cast<XT>(d.y);
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < KT; ++q)
            if (q < kc) xv[q] = __ldg(p + q);
    }
}

// blockWidth 32: one warp per 32-row block, lane = row.
template <typename VT, typename XT, int KT>
__device__ __forceinline__ void bw32_spmm_tile(const SpmvArgs<VT, XT> &a, const XT *__restrict__ X, int64_t ldx,
                                               XT *__restrict__ Y, int64_t ldy, int32_t k, int32_t tile,
                                               int lane) {
    const int64_t row0 = static_cast<int64_t>(tile) * 32;
    const int64_t row = row0 + lane;
    int32_t k0 = 0, k1 = 0;
    if (tile < a.numBlocks) {
        k0 = __ldg(a.blkOff + tile);
        k1 = __ldg(a.blkOff + tile + 1);
    }
    const int32_t c0 = a.hasCoo ? __ldg(a.cooTile + tile) : 0;
    const int32_t c1 = a.hasCoo ? __ldg(a.cooTile + tile + 1) : 0;
    const float s = (a.scale && tile < a.numBlocks) ? __ldg(a.scale + tile) : 1.0f;
    const bool xAligned = (reinterpret_cast<uintptr_t>(X) & 15) == 0 && (ldx & 1) == 0;
    for (int32_t r0 = 0; r0 < k; r0 += KT) {
        const int kc = min(KT, k - r0);
        const bool vec2 = xAligned && (r0 & 1) == 0;
        XT acc[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) acc[q] = XT(0);
        for (int32_t kb = k0; kb < k1; kb += 32) {
            const int cnt = min(32, k1 - kb);
            const int32_t myoff = lane < cnt ? __ldg(a.offs + kb + lane) : 0;
            const VT *vp = a.vals + static_cast<int64_t>(kb) * 32 + lane;
            for (int j = 0; j < cnt; ++j) {
                const int64_t col = row + __shfl_sync(kFull, myoff, j);
                const XT vv = widen<XT>(__ldg(vp + j * 32), s);
                if (static_cast<uint64_t>(col) < static_cast<uint64_t>(a.n) && vv != XT(0)) {
                    XT xv[KT];
                    load_x_row<XT, KT>(X + col * ldx + r0, kc, vec2, xv);
#pragma unroll
                    for (int q = 0; q < KT; ++q)
                        if (q < kc) acc[q] = fma_rn(vv, xv[q], acc[q]);
                }
            }
        }
        if (a.hasCoo) {
            // per column: the row's COO entries in list order, then one add
#pragma unroll
            for (int q = 0; q < KT; ++q) {
                if (q >= kc) break;
                XT c = XT(0);
                for (int32_t base = c0; base < c1; base += 32) {
                    const int32_t e = base + lane;
                    int lr = -1;
                    XT p = XT(0);
                    if (e < c1) {
                        lr = static_cast<int>(__ldg(a.cooRow + e) - row0);
                        p = mul_rn(__ldg(a.cooVal + e), __ldg(X + static_cast<int64_t>(__ldg(a.cooCol + e)) * ldx + r0 + q));
                    }
                    const int m = min(32, c1 - base);
                    for (int t = 0; t < m; ++t) {
                        const int rt = __shfl_sync(kFull, lr, t);
                        const XT pt = __shfl_sync(kFull, p, t);
                        if (rt == lane) c = add_rn(c, pt);
                    }
                }
                acc[q] = add_rn(acc[q], c);
            }
        }
        if (row < a.n) {
            XT *yp = Y + row * ldy + r0;
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) yp[q] = acc[q];
        }
    }
}

template <typename VT, typename XT, int KT>
__global__ void __launch_bounds__(256)
spmm_bw32(const SpmvArgs<VT, XT> a, const XT *__restrict__ X, int64_t ldx, XT *__restrict__ Y, int64_t ldy,
          int32_t k) {
    const int lane = threadIdx.x & 31;
    const int32_t tile = static_cast<int32_t>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (tile >= a.numTiles) return;  // warp-uniform
    bw32_spmm_tile<VT, XT, KT>(a, X, ldx, Y, ldy, k, tile, lane);
}

// Any block width: one thread per row (the reference's mapping).
template <typename VT, typename XT, int KT>
__global__ void __launch_bounds__(256)
spmm_rowwise(const SpmvArgs<VT, XT> a, const XT *__restrict__ X, int64_t ldx, XT *__restrict__ Y, int64_t ldy,
             int32_t k) {
    const int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (row >= a.n) return;
    const int32_t b = static_cast<int32_t>(row / a.bw);
    const int32_t lane = static_cast<int32_t>(row - static_cast<int64_t>(b) * a.bw);
    int32_t k0 = 0, k1 = 0;
    if (b < a.numBlocks) {
        k0 = __ldg(a.blkOff + b);
        k1 = __ldg(a.blkOff + b + 1);
    }
    const float s = (a.scale && b < a.numBlocks) ? __ldg(a.scale + b) : 1.0f;
    for (int32_t r0 = 0; r0 < k; r0 += KT) {
        const int kc = min(KT, k - r0);
        XT acc[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) acc[q] = XT(0);
        for (int32_t kk = k0; kk < k1; ++kk) {
            const XT vv = widen<XT>(__ldg(a.vals + static_cast<int64_t>(kk) * a.bw + lane), s);
            const int64_t col = row + __ldg(a.offs + kk);
            if (vv == XT(0) || col < 0 || col >= a.n) continue;
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) acc[q] = fma_rn(vv, __ldg(X + col * ldx + r0 + q), acc[q]);
        }
        if (a.hasCoo) {
            const int32_t e0 = __ldg(a.cooRowPtr + row), e1 = __ldg(a.cooRowPtr + row + 1);
#pragma unroll
            for (int q = 0; q < KT; ++q) {
                if (q >= kc) break;
                XT c = XT(0);
                for (int32_t e = e0; e < e1; ++e)
                    c = add_rn(c, mul_rn(__ldg(a.cooVal + e),
                                         __ldg(X + static_cast<int64_t>(__ldg(a.cooCol + e)) * ldx + r0 + q)));
                acc[q] = add_rn(acc[q], c);
            }
        }
#pragma unroll
        for (int q = 0; q < KT; ++q)
            if (q < kc) Y[row * ldy + r0 + q] = acc[q];
    }
}

}  // namespace dev
}  // namespace hbdia
