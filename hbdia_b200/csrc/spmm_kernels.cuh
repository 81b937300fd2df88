// Multi-RHS product Y = A X on the HBDIA layout (sm_100a).
//
// X (n x k) and Y are row-major with leading dimensions ldx, ldy (CM = false:
// element (i, j) at X[i * ldx + j]) or column-major (CM = true: X[j * ldx + i],
// each right-hand side a contiguous vector).  Column j of Y is computed with
// exactly the SpMV's arithmetic (ascending-offset FMA chain over the
// blocked-DIA values, sequential multiply-then-add over the row's COO
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
            if (q + 1 < kc) {  // both elements of the pair are in the block
                const double2 d = __ldg(reinterpret_cast<const double2 *>(p) + q / 2);
                xv[q] = static_cast<XT>(d.x);
                xv[q + 1] = static_cast<XT>(d.y);
            } else if (q < kc) {  // odd last column: never read past it
                xv[q] = __ldg(p + q);
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < KT; ++q)
            if (q < kc) xv[q] = __ldg(p + q);
    }
}

// Offset of element (row i, column j) of an X or Y block.
template <bool CM>
__device__ __forceinline__ int64_t blk(int64_t i, int64_t j, int64_t ld) {
    return CM ? j * ld + i : i * ld + j;
}

// How one pass reads its KT right-hand sides at column c: from a block (X
// row- or column-major with leading dimension ld; Xp is the pass's first
// column, column-major, or X + r0, row-major; IT is the element-index type,
// 32-bit whenever the pass's block fits, which keeps the address arithmetic
// to one instruction per gather) ...
template <typename XT, int KT, bool CM, typename IT, bool FULL>
struct XBlock {
    const XT *Xp;
    IT ld;
    bool vec2;
    __device__ __forceinline__ void load(IT c, int kc, XT (&xv)[KT]) const {
        if (CM) {
#pragma unroll
            for (int q = 0; q < KT; ++q)
                xv[q] = (FULL || q < kc) ? __ldg(Xp + (static_cast<IT>(q) * ld + c)) : XT(0);
        } else {
            load_x_row<XT, KT>(Xp + c * ld, FULL ? KT : kc, vec2, xv);
        }
    }
};

// ... or from KT separate vectors (column q at p[q]).
template <typename XT, int KT, bool FULL>
struct XList {
    const XT *p[KT];
    __device__ __forceinline__ void load(int32_t c, int kc, XT (&xv)[KT]) const {
#pragma unroll
        for (int q = 0; q < KT; ++q) xv[q] = (FULL || q < kc) ? __ldg(p[q] + c) : XT(0);
    }
};

// U offsets of one row block for the KT right-hand sides of one pass: the U
// values and all U x KT x gathers are issued before any product is formed, so
// a group costs one memory round trip.  Column q's products are added in
// ascending offset order.
// CHECK: some column of the group may fall outside [0, xn) (else every one
// is inside: no range test, no index select).
template <typename VT, typename XT, int KT, int U, typename IT, bool FULL, bool CHECK, typename XS>
__device__ __forceinline__ void spmm_group(const SpmvArgs<VT, XT> &a, const XS &xs, const VT *vp, int32_t myoff, int j,
                                           int64_t row, int kc, float s, XT (&acc)[KT]) {
    VT v[U];
    bool ok[U];
    XT xv[U][KT];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t col = row + __shfl_sync(kFull, myoff, j + u);
        ok[u] = !CHECK || static_cast<uint64_t>(col) < static_cast<uint64_t>(a.xn);
        v[u] = __ldg(vp + (j + u) * 32);
        xs.load(ok[u] ? static_cast<IT>(col) : IT(0), kc, xv[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const XT vv = widen<XT>(v[u], s);
        if (ok[u] && vv != XT(0)) {
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (FULL || q < kc) acc[q] = fma_rn(vv, xv[u][q], acc[q]);
        }
    }
}

// The offsets of one row block for one pass, in groups of U = 16 / KT (at
// least 1), so about 16 x gathers per lane are in flight (32 measured slower
// on B200 at every tile width); the offsets after the last full group go in
// groups of 4 and then one group of the remaining 1-3, so each group is one
// load round trip.
template <typename VT, typename XT, int KT, typename IT, bool FULL, bool CHECK, typename XS>
__device__ __forceinline__ void spmm_chunk(const SpmvArgs<VT, XT> &a, const XS &xs, const VT *vp, int32_t myoff,
                                           int cnt, int64_t row, int kc, float s, XT (&acc)[KT]) {
    constexpr int U = KT >= 16 ? 1 : 16 / KT;
    int j = 0;
    for (; j + U <= cnt; j += U)
        spmm_group<VT, XT, KT, U, IT, FULL, CHECK>(a, xs, vp, myoff, j, row, kc, s, acc);
    if constexpr (U > 4)
        for (; j + 4 <= cnt; j += 4) spmm_group<VT, XT, KT, 4, IT, FULL, CHECK>(a, xs, vp, myoff, j, row, kc, s, acc);
    const int rest = cnt - j;  // < min(U, 4), warp-uniform
    if constexpr (U > 3)
        if (rest == 3) spmm_group<VT, XT, KT, 3, IT, FULL, CHECK>(a, xs, vp, myoff, j, row, kc, s, acc);
    if constexpr (U > 2)
        if (rest == 2) spmm_group<VT, XT, KT, 2, IT, FULL, CHECK>(a, xs, vp, myoff, j, row, kc, s, acc);
    if constexpr (U > 1)
        if (rest == 1) spmm_group<VT, XT, KT, 1, IT, FULL, CHECK>(a, xs, vp, myoff, j, row, kc, s, acc);
}

// Chunks of up to 32 offsets (ascending) whose columns all lie in [0, xn) for
// every row of the tile run without range tests.
template <typename VT, typename XT, int KT, typename IT, bool FULL, typename XS>
__device__ __forceinline__ void spmm_pass(const SpmvArgs<VT, XT> &a, const XS &xs, int32_t k0, int32_t k1,
                                          int64_t row, int lane, int kc, float s, XT (&acc)[KT]) {
    const int64_t row0 = row - lane;
    for (int32_t kb = k0; kb < k1; kb += 32) {
        const int cnt = min(32, k1 - kb);
        const int32_t myoff = lane < cnt ? __ldg(a.offs + kb + lane) : 0;
        const VT *vp = a.vals + static_cast<int64_t>(kb) * 32 + lane;
        const int32_t offFirst = __shfl_sync(kFull, myoff, 0), offLast = __shfl_sync(kFull, myoff, cnt - 1);
        if (row0 + offFirst >= 0 && row0 + 31 + offLast < a.xn)
            spmm_chunk<VT, XT, KT, IT, FULL, false>(a, xs, vp, myoff, cnt, row, kc, s, acc);
        else
            spmm_chunk<VT, XT, KT, IT, FULL, true>(a, xs, vp, myoff, cnt, row, kc, s, acc);
    }
}

// The COO remainder of one 32-row tile for one pass of the vector-list form,
// added to acc: per column, the row's COO entries in list order, then one
// add; each batch of 32 entries is loaded once for all columns.  xat(cc, q)
// reads x_q[cc].  (bw32_spmm_tile_t keeps the same steps inline.)
template <typename XT, int KT, typename XAt>
__device__ __forceinline__ void spmm_coo(const int32_t *cooRow, const int32_t *cooCol, const XT *cooVal, int32_t c0,
                                         int32_t c1, int64_t row0, int lane, int kc, XAt xat, XT (&acc)[KT]) {
    XT c[KT];
#pragma unroll
    for (int q = 0; q < KT; ++q) c[q] = XT(0);
    for (int32_t base = c0; base < c1; base += 32) {
        const int32_t e = base + lane;
        int lr = -1;
        XT p[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) p[q] = XT(0);
        if (e < c1) {
            lr = static_cast<int>(__ldg(cooRow + e) - row0);
            const int64_t cc = __ldg(cooCol + e);
            const XT cv = __ldg(cooVal + e);
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) p[q] = mul_rn(cv, xat(cc, q));
        }
        const int m = min(32, c1 - base);
        for (int t = 0; t < m; ++t) {
            const int rt = __shfl_sync(kFull, lr, t);
#pragma unroll
            for (int q = 0; q < KT; ++q) {
                const XT pt = __shfl_sync(kFull, p[q], t);
                if (rt == lane) c[q] = add_rn(c[q], pt);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < KT; ++q) acc[q] = add_rn(acc[q], c[q]);
}

// blockWidth 32: one warp per 32-row block, lane = row, k right-hand sides in
// passes of KT.  IT: element-index type of the gathers (int32_t only when
// every pass's block has fewer than 2^31 elements); FULL: k is a multiple of
// KT (no partial pass).
template <typename VT, typename XT, int KT, bool CM, typename IT, bool FULL>
__device__ __forceinline__ void bw32_spmm_tile_t(const SpmvArgs<VT, XT> &a, const XT *__restrict__ X, int64_t ldx,
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
    const bool xAligned = !CM && (reinterpret_cast<uintptr_t>(X) & 15) == 0 && (ldx & 1) == 0;
    for (int32_t r0 = 0; r0 < k; r0 += KT) {
        const int kc = min(KT, k - r0);
        const XBlock<XT, KT, CM, IT, FULL> xs{CM ? X + static_cast<int64_t>(r0) * ldx : X + r0,
                                              static_cast<IT>(ldx), xAligned && (r0 & 1) == 0};
        XT acc[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) acc[q] = XT(0);
        spmm_pass<VT, XT, KT, IT, FULL>(a, xs, k0, k1, row, lane, kc, s, acc);
        if (a.hasCoo) {
            // per column: the row's COO entries in list order, then one add;
            // each batch of 32 entries is loaded once for all columns
            XT c[KT];
#pragma unroll
            for (int q = 0; q < KT; ++q) c[q] = XT(0);
            for (int32_t base = c0; base < c1; base += 32) {
                const int32_t e = base + lane;
                int lr = -1;
                XT p[KT];
#pragma unroll
                for (int q = 0; q < KT; ++q) p[q] = XT(0);
                if (e < c1) {
                    lr = static_cast<int>(__ldg(a.cooRow + e) - row0);
                    const int64_t cc = __ldg(a.cooCol + e);
                    const XT cv = __ldg(a.cooVal + e);
#pragma unroll
                    for (int q = 0; q < KT; ++q)
                        if (q < kc) p[q] = mul_rn(cv, __ldg(X + blk<CM>(cc, r0 + q, ldx)));
                }
                const int m = min(32, c1 - base);
                for (int t = 0; t < m; ++t) {
                    const int rt = __shfl_sync(kFull, lr, t);
#pragma unroll
                    for (int q = 0; q < KT; ++q) {
                        const XT pt = __shfl_sync(kFull, p[q], t);
                        if (rt == lane) c[q] = add_rn(c[q], pt);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < KT; ++q) acc[q] = add_rn(acc[q], c[q]);
        }
        if (row < a.n) {
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) Y[blk<CM>(row, r0 + q, ldy)] = acc[q];
        }
    }
}

// k <= kVecListMax separate vectors: x_j and y_j anywhere in device memory,
// passed by value in the kernel's parameter block (no table in memory, so a
// launch allocates nothing and can be captured in a graph).
constexpr int kVecListMax = 32;
template <typename XT>
struct VecList {
    const XT *x[kVecListMax];
    XT *y[kVecListMax];
};

// The vector-list form of bw32_spmm_tile_t (x_j read at x[j] + col, 32-bit
// offsets: each vector has fewer than 2^31 elements).
template <typename VT, typename XT, int KT, bool FULL>
__device__ __forceinline__ void bw32_spmm_list_tile(const SpmvArgs<VT, XT> &a, const VecList<XT> &L, int32_t k,
                                                    int32_t tile, int lane) {
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
    for (int32_t r0 = 0; r0 < k; r0 += KT) {
        const int kc = min(KT, k - r0);
        XList<XT, KT, FULL> xs;
#pragma unroll
        for (int q = 0; q < KT; ++q) xs.p[q] = (FULL || q < kc) ? L.x[r0 + q] : L.x[r0];
        XT acc[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) acc[q] = XT(0);
        spmm_pass<VT, XT, KT, int32_t, FULL>(a, xs, k0, k1, row, lane, kc, s, acc);
        if (a.hasCoo)
            spmm_coo<XT, KT>(a.cooRow, a.cooCol, a.cooVal, c0, c1, row0, lane, kc,
                             [&](int64_t cc, int q) { return __ldg(xs.p[q] + cc); }, acc);
        if (row < a.n) {
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) L.y[r0 + q][row] = acc[q];
        }
    }
}

// Any k, any size (the batch kernel's form).
template <typename VT, typename XT, int KT, bool CM = false>
__device__ __forceinline__ void bw32_spmm_tile(const SpmvArgs<VT, XT> &a, const XT *__restrict__ X, int64_t ldx,
                                               XT *__restrict__ Y, int64_t ldy, int32_t k, int32_t tile,
                                               int lane) {
    bw32_spmm_tile_t<VT, XT, KT, CM, int64_t, false>(a, X, ldx, Y, ldy, k, tile, lane);
}

template <typename VT, typename XT, int KT, bool CM, typename IT, bool FULL>
__global__ void __launch_bounds__(256)
spmm_bw32(const SpmvArgs<VT, XT> a, const XT *__restrict__ X, int64_t ldx, XT *__restrict__ Y, int64_t ldy,
          int32_t k) {
    const int lane = threadIdx.x & 31;
    const int32_t tile = static_cast<int32_t>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (tile >= a.numTiles) return;  // warp-uniform
    bw32_spmm_tile_t<VT, XT, KT, CM, IT, FULL>(a, X, ldx, Y, ldy, k, tile, lane);
}

template <typename VT, typename XT, int KT, bool FULL>
__global__ void __launch_bounds__(256)
spmm_bw32_list(const SpmvArgs<VT, XT> a, const __grid_constant__ VecList<XT> L, int32_t k) {
    const int lane = threadIdx.x & 31;
    const int32_t tile = static_cast<int32_t>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (tile >= a.numTiles) return;  // warp-uniform
    bw32_spmm_list_tile<VT, XT, KT, FULL>(a, L, k, tile, lane);
}

// Any block width: one thread per row (the reference's mapping).
template <typename VT, typename XT, int KT, bool CM>
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
            if (vv == XT(0) || col < 0 || col >= a.xn) continue;
#pragma unroll
            for (int q = 0; q < KT; ++q)
                if (q < kc) acc[q] = fma_rn(vv, __ldg(X + blk<CM>(col, r0 + q, ldx)), acc[q]);
        }
        if (a.hasCoo) {
            const int32_t e0 = __ldg(a.cooRowPtr + row), e1 = __ldg(a.cooRowPtr + row + 1);
#pragma unroll
            for (int q = 0; q < KT; ++q) {
                if (q >= kc) break;
                XT c = XT(0);
                for (int32_t e = e0; e < e1; ++e)
                    c = add_rn(c, mul_rn(__ldg(a.cooVal + e), __ldg(X + blk<CM>(__ldg(a.cooCol + e), r0 + q, ldx))));
                acc[q] = add_rn(acc[q], c);
            }
        }
#pragma unroll
        for (int q = 0; q < KT; ++q)
            if (q < kc) Y[blk<CM>(row, r0 + q, ldy)] = acc[q];
    }
}

}  // namespace dev
}  // namespace hbdia
