// Quad-tile HBDIA SpMV for blockWidth 32 on sm_100a.
//
// The single-block kernels (spmv_kernels.cuh) spend about 25 instructions per
// stored offset of a 32-row block: the offset's broadcast, the column, its
// bound check, the x address, the value and x loads, the widening, the zero
// check and the FMA.  With 4- and 2-byte value storage that instruction
// stream, not HBM, bounds the SpMV (B200: ~60 % issue utilisation at 45 % of
// the HBM bandwidth).  Most HBDIA matrices store the same offset list in
// neighbouring blocks (every interior block of a stencil, every block of a
// banded matrix), so here one warp takes four consecutive blocks (a 128-row
// quad) and, when their offset lists are equal, shares the per-offset work:
// lane l owns rows row0 + l + 32 q (q = 0..3); per offset one broadcast and
// one x address serve the four blocks, whose value loads (one coalesced row of
// 32 values each) and x loads (32 consecutive elements each, 256 bytes apart:
// immediate offsets of one address) follow.  Four independent FMA chains per
// lane give the loads and FMAs room to overlap.  Quads whose blocks differ run
// block by block with the single-block code.
//
// The offsets of a uniform quad go in full groups of U (all of a group's value
// and x loads issued before its FMAs, no per-offset range test), then the 1-3
// left over as one more group, so a 27-offset quad takes 7 load round trips;
// quads whose columns all lie in [0, xn) skip the column checks.  Predicating
// every load and FMA on the group's range instead doubled the instruction
// count on B200.
//
// The COO remainder of the quad (row-sorted entries; its first 64 loaded one
// quad ahead) goes 32 entries at a time; each entry's product is formed by its
// lane, and the first entry of every row segment (its "head") sums the segment
// in list order with shuffles
// -- segments are short (1 % extra entries: mostly one entry per row).  A
// segment cut by the 32-entry chunk boundary carries its partial sum into the
// next chunk.  The quad's 128 DIA sums wait in a per-warp shared buffer, each
// head adds its row's COO sum there once, and the owning lanes write y.
//
// Quad-interleaved value storage (HBDIA_STORE_F32_QUAD / _BF16_QUAD): the
// values of a uniform quad -- four blocks with one offset list of at most 32
// offsets -- are stored [offset][lane][block] instead of [block][offset][lane]
// (same region, same size), so a lane's four values of one offset are ONE
// 16-byte (FP32) or 8-byte (BF16) load, a warp's request 512 / 256 bytes --
// what an FP64 value row gives the other kernels.  Non-uniform quads keep the
// per-block order.  The layout is built by build_plan with the same
// uniformity test this kernel makes at run time.
//
// Arithmetic is the reference's, in the reference's order: per row, offsets
// ascending, stored zeros and columns outside [0, xn) skipped, fma; COO
// products summed from zero in list order with separately rounded multiply
// and add; y = dia + coo for rows with remainder entries, y = dia otherwise
// (src/Operations/HBDIASpMV.cu:42-88, src/Operations/HBDIASpMV.cpp:76-92).
// (dia + 0 would equal dia: the FMA chain from +0 never yields -0.)
#pragma once

#include "spmv_kernels.cuh"

namespace hbdia {
namespace dev {

constexpr int kQuadWarps = 8;  // warps per CTA

// DIA sum of one 32-row block straight from its offset range [k0, k1): full
// groups of 8 offsets with all loads in flight, then one group of 4 and one of
// the remaining 1-3; ascending order.
template <typename VT, typename XT, int U>
__device__ __forceinline__ XT block_group(const XT *__restrict__ x, const VT *__restrict__ vp, int32_t myoff, int j,
                                          int32_t row, uint32_t n, float s, XT sum) {
    VT v[U];
    XT xv[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t col = row + __shfl_sync(kFull, myoff, (j + u) & 31);
        ok[u] = static_cast<uint32_t>(col) < n;
        v[u] = ld_stream(vp + (j + u) * 32);
        xv[u] = XT(0);
        if (ok[u]) xv[u] = __ldg(x + col);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const XT vv = widen<XT>(v[u], s);
        if (ok[u] && vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
    }
    return sum;
}

template <typename VT, typename XT>
__device__ __forceinline__ XT block_dia(const SpmvArgs<VT, XT> &a, const XT *__restrict__ x, int32_t k0, int32_t k1,
                                        int32_t row, int lane, float s) {
    const uint32_t n = static_cast<uint32_t>(a.xn);
    XT sum = XT(0);
    for (int32_t kb = k0; kb < k1; kb += 32) {
        const int cnt = min(32, k1 - kb);
        const int32_t myoff = lane < cnt ? __ldg(a.offs + kb + lane) : 0;
        const VT *vp = a.vals + static_cast<int64_t>(kb) * 32 + lane;
        int j = 0;
        for (; j + 8 <= cnt; j += 8) sum = block_group<VT, XT, 8>(x, vp, myoff, j, row, n, s, sum);
        if (j + 4 <= cnt) {
            sum = block_group<VT, XT, 4>(x, vp, myoff, j, row, n, s, sum);
            j += 4;
        }
        const int rest = cnt - j;  // 0-3, warp-uniform: one group
        if (rest == 3) sum = block_group<VT, XT, 3>(x, vp, myoff, j, row, n, s, sum);
        else if (rest == 2) sum = block_group<VT, XT, 2>(x, vp, myoff, j, row, n, s, sum);
        else if (rest == 1) sum = block_group<VT, XT, 1>(x, vp, myoff, j, row, n, s, sum);
    }
    return sum;
}

// U offsets g .. g+U-1 (all < K) of the four blocks of a uniform quad: the
// 4U values and 4U x gathers issued before any product is formed.  Values at
// val(k, q) (element k * 32 of block q for this lane); offsets: lane k holds
// offset k.  CHECK: some column may fall outside [0, xn).
template <typename VT, typename XT, int U, bool CHECK, typename Val>
__device__ __forceinline__ void quad_group(const XT *__restrict__ x, Val val, int32_t g, int32_t myoff, int32_t row,
                                           uint32_t xn, const float (&sc)[4], XT (&sum)[4]) {
    VT v[U][4];
    XT xv[U][4];
    bool ok[U][4];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t off = __shfl_sync(kFull, myoff, (g + u) & 31);
        val(g + u, v[u]);
        const int32_t col = row + off;
        const XT *xp = x + col;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ok[u][q] = !CHECK || static_cast<uint32_t>(col + 32 * q) < xn;
            xv[u][q] = XT(0);
            if (ok[u][q]) xv[u][q] = __ldg(xp + 32 * q);
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const XT vv = widen<XT>(v[u][q], sc[q]);
            if (ok[u][q] && vv != XT(0)) sum[q] = fma_rn(vv, xv[u][q], sum[q]);
        }
    }
}

// The K offsets of a uniform quad in ascending order: full groups of U, then
// groups of 4 (when U > 4), then the remaining 1-3 offsets as one group -- no
// per-offset range test inside a group, and every group one load round trip.
template <typename VT, typename XT, int U, bool CHECK, typename Val>
__device__ __forceinline__ void quad_offsets(const XT *__restrict__ x, Val val, int32_t K, int32_t myoff,
                                             int32_t row, uint32_t xn, const float (&sc)[4], XT (&sum)[4]) {
    int32_t g = 0;
    for (; g + U <= K; g += U) quad_group<VT, XT, U, CHECK>(x, val, g, myoff, row, xn, sc, sum);
    if constexpr (U > 4)
        for (; g + 4 <= K; g += 4) quad_group<VT, XT, 4, CHECK>(x, val, g, myoff, row, xn, sc, sum);
    const int32_t rest = K - g;  // < min(U, 4), warp-uniform
    if constexpr (U > 3)
        if (rest == 3) quad_group<VT, XT, 3, CHECK>(x, val, g, myoff, row, xn, sc, sum);
    if constexpr (U > 2)
        if (rest == 2) quad_group<VT, XT, 2, CHECK>(x, val, g, myoff, row, xn, sc, sum);
    if constexpr (U > 1)
        if (rest == 1) quad_group<VT, XT, 1, CHECK>(x, val, g, myoff, row, xn, sc, sum);
}

// Values of the four blocks in their own regions (vb[q] + k * 32 + lane).
template <typename VT>
struct QuadVals {
    const VT *v0, *v1, *v2, *v3;
    __device__ __forceinline__ void operator()(int32_t k, VT (&v)[4]) const {
        v[0] = ld_stream(v0 + k * 32);
        v[1] = ld_stream(v1 + k * 32);
        v[2] = ld_stream(v2 + k * 32);
        v[3] = ld_stream(v3 + k * 32);
    }
};

// The lane's values of the four blocks for offset k of a quad-interleaved
// region (vq: the quad's first value): one vector load.
template <typename VT>
struct QuadValsInterleaved;
template <>
struct QuadValsInterleaved<float> {
    const float *vq;
    int lane;
    __device__ __forceinline__ void operator()(int32_t k, float (&v)[4]) const {
        const float4 f = __ldcs(reinterpret_cast<const float4 *>(vq) + (k * 32 + lane));
        v[0] = f.x;
        v[1] = f.y;
        v[2] = f.z;
        v[3] = f.w;
    }
};
template <>
struct QuadValsInterleaved<__nv_bfloat16> {
    const __nv_bfloat16 *vq;
    int lane;
    __device__ __forceinline__ void operator()(int32_t k, __nv_bfloat16 (&v)[4]) const {
        const uint2 r = __ldcs(reinterpret_cast<const uint2 *>(vq) + (k * 32 + lane));
        v[0] = __ushort_as_bfloat16(static_cast<unsigned short>(r.x & 0xffffu));
        v[1] = __ushort_as_bfloat16(static_cast<unsigned short>(r.x >> 16));
        v[2] = __ushort_as_bfloat16(static_cast<unsigned short>(r.y & 0xffffu));
        v[3] = __ushort_as_bfloat16(static_cast<unsigned short>(r.y >> 16));
    }
};

// What the warp needs of a quad before its DIA part: the block pointers and
// COO tile starts of its four tiles (lanes 0..4), whether the four blocks
// share one offset list (and lane k's offset k), and its first 32 COO entries.
template <typename XT>
struct QuadFront {
    int32_t kb, cb;  // lane i < 5: blkOff / cooTile of tile 4 Q + i (clamped)
    int32_t myoff;   // lane k < K: offset k of the first block
    bool uni;        // the four blocks have the same offsets (warp-uniform)
    int32_t cr, cc;  // COO entry c0 + lane: local row (or INT_MAX), column
    XT cv;
    int32_t cr2, cc2;  // COO entry c0 + 32 + lane
    XT cv2;
};

// Persistent: warp g of W walks quads g, g + W, ...  Software-pipelined: while
// it computes quad i it has quad i+1's offsets and first COO entries and quad
// i+2's block pointers in flight.  U offsets of the four blocks in flight per
// lane; PF: ask L2 for the next quad's value rows.
template <typename VT, typename XT, int U, bool PF>
__global__ void __launch_bounds__(kQuadWarps * 32)
spmv_bw32_quad(const SpmvArgs<VT, XT> a, const XT *__restrict__ x, XT *__restrict__ y) {
    __shared__ XT dbuf[kQuadWarps][128];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    XT *db = dbuf[w];
    const int32_t W = static_cast<int32_t>(gridDim.x) * kQuadWarps;
    const int32_t numQuads = (a.numTiles + 3) >> 2;
    const uint32_t xn = static_cast<uint32_t>(a.xn);
    int32_t Q = static_cast<int32_t>(blockIdx.x) * kQuadWarps + w;
    if (Q >= numQuads) return;  // warp-uniform
    auto loadMeta = [&](int32_t q0, QuadFront<XT> &f) {
        f.kb = 0;
        f.cb = 0;
        if (q0 < numQuads && lane < 5) {
            const int32_t t = q0 * 4 + lane;
            f.kb = __ldg(a.blkOff + min(t, a.numBlocks));
            if (a.hasCoo) f.cb = __ldg(a.cooTile + min(t, a.numTiles));
        }
    };
    // offsets and first COO entries of quad q0 (its meta in f); the
    // comparison of the four offset lists waits for the loads
    int32_t o1 = 0, o2 = 0, o3 = 0;
    auto loadBody = [&](int32_t q0, QuadFront<XT> &f) {
        const int32_t k0 = __shfl_sync(kFull, f.kb, 0), k1 = __shfl_sync(kFull, f.kb, 1);
        const int32_t k2 = __shfl_sync(kFull, f.kb, 2), k3 = __shfl_sync(kFull, f.kb, 3);
        const int32_t k4 = __shfl_sync(kFull, f.kb, 4);
        const int32_t c0 = __shfl_sync(kFull, f.cb, 0), c4 = __shfl_sync(kFull, f.cb, 4);
        const int32_t K = k1 - k0;
        f.uni = q0 < numQuads && K <= 32 && k2 - k1 == K && k3 - k2 == K && k4 - k3 == K;
        f.myoff = 0;
        o1 = o2 = o3 = 0;
        if (f.uni && lane < K) {
            f.myoff = __ldg(a.offs + k0 + lane);
            o1 = __ldg(a.offs + k1 + lane);
            o2 = __ldg(a.offs + k2 + lane);
            o3 = __ldg(a.offs + k3 + lane);
        }
        f.cr = f.cr2 = 0x7fffffff;
        f.cc = f.cc2 = 0;
        f.cv = f.cv2 = XT(0);
        const int32_t e = c0 + lane;
        if (q0 < numQuads && e < c4) {
            f.cr = __ldg(a.cooRow + e) - q0 * 128;
            f.cc = __ldg(a.cooCol + e);
            f.cv = __ldg(a.cooVal + e);
        }
        if (q0 < numQuads && e + 32 < c4) {
            f.cr2 = __ldg(a.cooRow + e + 32) - q0 * 128;
            f.cc2 = __ldg(a.cooCol + e + 32);
            f.cv2 = __ldg(a.cooVal + e + 32);
        }
    };
    auto finishBody = [&](QuadFront<XT> &f) {
        const int diff = (o1 != f.myoff) | (o2 != f.myoff) | (o3 != f.myoff);
        f.uni = f.uni && !__any_sync(kFull, diff);
    };

    QuadFront<XT> cur, nxt, nn;
    loadMeta(Q, cur);
    loadMeta(Q + W, nxt);
    loadBody(Q, cur);
    finishBody(cur);
    for (; Q < numQuads; Q += W) {
        const int32_t t0 = Q * 4;
        const int32_t row0 = t0 * 32;
        const int32_t row = row0 + lane;
        int32_t kq[5], cq[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            kq[i] = __shfl_sync(kFull, cur.kb, i);
            cq[i] = __shfl_sync(kFull, cur.cb, i);
        }
        // x of this quad's first COO entries (columns loaded one quad ago)
        const XT cx = cur.cr != 0x7fffffff ? __ldg(x + cur.cc) : XT(0);
        const XT cx2 = cur.cr2 != 0x7fffffff ? __ldg(x + cur.cc2) : XT(0);
        // quad i+2's pointers, quad i+1's offsets and COO entries
        loadMeta(Q + 2 * W, nn);
        loadBody(Q + W, nxt);
        if (PF) {  // quad i+1's value rows (contiguous, 64-byte aligned) into L2
            const int32_t nk0 = __shfl_sync(kFull, nxt.kb, 0), nk4 = __shfl_sync(kFull, nxt.kb, 4);
            if (lane == 0 && Q + W < numQuads && nk4 > nk0) {
                const int64_t bytes = static_cast<int64_t>(nk4 - nk0) * 32 * static_cast<int64_t>(sizeof(VT));
                prefetch_l2_bulk(a.vals + static_cast<int64_t>(nk0) * 32,
                                 static_cast<uint32_t>(bytes < 32768 ? bytes : 32768));
            }
        }
        float sc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) sc[q] = (a.scale && t0 + q < a.numBlocks) ? __ldg(a.scale + t0 + q) : 1.0f;
        XT sum[4] = {XT(0), XT(0), XT(0), XT(0)};
        const int32_t K = kq[1] - kq[0];
        if (cur.uni) {
            if (K > 0) {
                const int32_t offFirst = __shfl_sync(kFull, cur.myoff, 0);
                const int32_t offLast = __shfl_sync(kFull, cur.myoff, K - 1);
                const bool interior = int64_t(row0) + offFirst >= 0 && int64_t(row0) + 127 + offLast < int64_t(a.xn);
                bool done = false;
                if constexpr (sizeof(VT) < 8) {
                    if (a.quadLayout) {  // interleaved region of the quad
                        const QuadValsInterleaved<VT> vals{a.vals + static_cast<int64_t>(kq[0]) * 32, lane};
                        if (interior) quad_offsets<VT, XT, U, false>(x, vals, K, cur.myoff, row, xn, sc, sum);
                        else quad_offsets<VT, XT, U, true>(x, vals, K, cur.myoff, row, xn, sc, sum);
                        done = true;
                    }
                }
                if (!done) {
                    const QuadVals<VT> vals{a.vals + static_cast<int64_t>(kq[0]) * 32 + lane,
                                            a.vals + static_cast<int64_t>(kq[1]) * 32 + lane,
                                            a.vals + static_cast<int64_t>(kq[2]) * 32 + lane,
                                            a.vals + static_cast<int64_t>(kq[3]) * 32 + lane};
                    if (interior) quad_offsets<VT, XT, U, false>(x, vals, K, cur.myoff, row, xn, sc, sum);
                    else quad_offsets<VT, XT, U, true>(x, vals, K, cur.myoff, row, xn, sc, sum);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (kq[q + 1] > kq[q]) sum[q] = block_dia<VT, XT>(a, x, kq[q], kq[q + 1], row + 32 * q, lane, sc[q]);
        }
        // COO remainder: the heads of row segments add their sums into db
#pragma unroll
        for (int q = 0; q < 4; ++q) db[lane + 32 * q] = sum[q];
        __syncwarp();
        const int32_t c0 = cq[0], c4 = cq[4];
        if (c4 > c0) {
            int32_t cr = cur.cr;
            XT cp = cur.cr != 0x7fffffff ? mul_rn(cur.cv, cx) : XT(0);
            XT carry = XT(0);
            int32_t carryRow = -1;
            for (int32_t base = c0; base < c4; base += 32) {
                if (base == c0 + 32) {  // entries 32..63, prefetched with the first ones
                    cr = cur.cr2;
                    cp = cur.cr2 != 0x7fffffff ? mul_rn(cur.cv2, cx2) : XT(0);
                } else if (base != c0) {  // rare: more than 64 entries in the quad
                    const int32_t e = base + lane;
                    cr = 0x7fffffff;
                    cp = XT(0);
                    if (e < c4) {
                        cr = __ldg(a.cooRow + e) - row0;
                        cp = mul_rn(__ldg(a.cooVal + e), __ldg(x + __ldg(a.cooCol + e)));
                    }
                }
                const bool valid = base + lane < c4;
                const int32_t prevR = __shfl_up_sync(kFull, cr, 1);
                const bool cont = lane == 0 && cr == carryRow;  // continues the carried segment
                const bool head = valid && (lane == 0 || cr != prevR);
                if (lane == 0 && carryRow >= 0 && cr != carryRow) db[carryRow] = add_rn(db[carryRow], carry);
                XT c = head ? add_rn(cont ? carry : XT(0), cp) : XT(0);
                bool ext = head;  // still extending its segment
                for (int t = 1; __any_sync(kFull, ext); ++t) {
                    const int32_t rt = __shfl_down_sync(kFull, cr, t & 31);
                    const XT pt = __shfl_down_sync(kFull, cp, t & 31);
                    ext = ext && lane + t < 32 && rt == cr;
                    if (ext) c = add_rn(c, pt);
                }
                const bool last = base + 32 >= c4;
                const unsigned heads = __ballot_sync(kFull, head);
                const int lastHead = 31 - __clz(heads);
                if (!last) {  // the chunk's last segment may continue in the next chunk
                    carry = __shfl_sync(kFull, c, lastHead);
                    carryRow = __shfl_sync(kFull, cr, lastHead);
                }
                if (head && (last || lane != lastHead)) db[cr] = add_rn(db[cr], c);
                __syncwarp();
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int32_t r = row + 32 * q;
            if (r < a.n) __stcs(y + r, db[lane + 32 * q]);
        }
        __syncwarp();
        finishBody(nxt);
        cur = nxt;
        nxt = nn;
    }
}

}  // namespace dev
}  // namespace hbdia
