// Staged HBDIA SpMV for blockWidth 32 on sm_100a: the x window of every row
// tile is staged in shared memory by bulk copies, one tile ahead.
//
// The HBDIA kernel's x reads (src/Operations/HBDIASpMV.cu:42-71) are one
// gather per stored value: for a 32-row tile and offset o, lanes read
// x[row0 + o + lane].  Neighbouring diagonals (o, o+1, o+2 of a stencil) read
// nearly the same 32 elements, so a tile's x reads collapse into a few runs:
// the union of [row0 + o, row0 + o + 32) over the tile's offsets, merged where
// windows overlap or touch (9 runs of 34 elements for a 27-point stencil
// instead of 27 gathers of 32).  The kernel copies those runs once into
// shared memory and reads x from there.
//
// Persistent: warp g of W walks tiles g, g + W, ... (neighbouring warps on
// neighbouring tiles).  Per tile i the warp
//   * issues the bulk copies of tile i+1's x runs (one cp.async.bulk per run,
//     issued by the run's first lane; an unaligned end of x by plain loads)
//     and the cp.async gathers of x for tile i+1's COO entries into the other
//     of its two stages, all completing on that stage's mbarrier, and asks L2
//     for tile i+1's value rows (cp.async.bulk.prefetch.L2);
//   * loads tile i's stored values into registers, all of the tile's offsets
//     (up to U) in flight at once, and meanwhile the offsets, COO entries and
//     block pointers of tiles i+2 and i+3;
//   * waits for tile i's stage (issued one tile earlier) and runs the FMA
//     chain with x from shared memory, then the COO remainder.
// So a tile costs one round trip (its value loads, from L2 after the
// prefetch) instead of one per group of offsets and x gathers, and the x
// reads leave the L1/LSU path.  A stage is small (the x runs, 32 COO entries),
// which keeps 24-32 warps per SM.
//
// Tiles with more than 32 offsets or a window larger than a stage run from
// global memory (same arithmetic); COO entries past the first 32 of a tile are
// read from global memory too.
//
// Arithmetic is the reference's, in the reference's order (spmv_kernels.cuh):
// per row, offsets ascending, stored zeros and columns outside [0, xn)
// skipped, fma; then the COO remainder in list order with separately rounded
// multiply and add; y = dia + coo.  Interior tiles (every column of every
// offset inside [0, xn)) skip the column bound check, which cannot fail there.
//
// Every wait is bounded by a time limit; on expiry the kernel records an error
// bit in *status, waits (again bounded) for the copies it has in flight and
// returns.  No multicast anywhere: each CTA copies into its own shared memory.
#pragma once

#include "spmv_kernels.cuh"

namespace hbdia {
namespace dev {

enum : int { kErrConsumerWait = 1, kErrProducerWait = 2, kErrDrain = 4 };

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase of parity `parity` to complete, for at most timeoutNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t timeoutNs) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (global_ns() - t0 > timeoutNs) return false;
        __nanosleep(20);
    }
}
// 1-D bulk copy global -> this CTA's shared memory (16-byte aligned
// addresses, size a multiple of 16), completing on `bar`'s transaction count.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
template <int B>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// The mbarrier's pending count drops by one when this thread's earlier
// cp.async copies have landed (the count includes these arrivals).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Order this thread's earlier shared-memory reads before later async-proxy
// (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------- layout
constexpr int kXsCoo = 32;       // COO entries a stage holds
constexpr int kXsWarps = 8;      // warps per CTA

template <typename XT>
struct XsStageHead {
    int32_t crow[kXsCoo];  // local row of each staged COO entry
    XT cval[kXsCoo];
    XT cx[kXsCoo];         // x[col] of the staged COO entries
};

template <typename VT, typename XT>
struct XsArgs {
    SpmvArgs<VT, XT> a;
    int32_t *status;     // error bits (0 = fine)
    uint64_t timeoutNs;  // limit of every wait
    int32_t skipTile;    // test hook: this tile's copies are never issued (-1: off)
};

// Bytes of dynamic shared memory of one CTA: two stages of SB bytes per warp
// plus their mbarriers.
__host__ __device__ constexpr size_t xs_smem_bytes(int stageBytes) {
    return static_cast<size_t>(kXsWarps) * 2 * stageBytes + static_cast<size_t>(kXsWarps) * 2 * sizeof(uint64_t);
}

// The DIA part of one tile from global memory (tiles that are not staged):
// offsets in masked groups of 8 (loads in flight together), ascending order.
template <typename VT, typename XT>
__device__ __forceinline__ XT tile_dia_global(const SpmvArgs<VT, XT> &a, const XT *__restrict__ x, int32_t k0,
                                              int32_t K, int32_t row, float s) {
    const uint32_t n = static_cast<uint32_t>(a.xn);
    const int lane = row & 31;
    XT sum = XT(0);
    for (int32_t j = 0; j < K; j += 8) {
        const int rem = K - j;
        VT v[8];
        XT xv[8];
        bool ok[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const bool in = u < rem;  // warp-uniform
            const int32_t col = in ? row + __ldg(a.offs + k0 + j + u) : -1;
            ok[u] = in && static_cast<uint32_t>(col) < n;
            v[u] = in ? ld_stream(a.vals + static_cast<int64_t>(k0 + j + u) * 32 + lane) : VT(0);
            xv[u] = ok[u] ? __ldg(x + col) : XT(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const XT vv = widen<XT>(v[u], s);
            if (ok[u] && vv != XT(0)) sum = fma_rn(vv, xv[u], sum);
        }
    }
    return sum;
}

// Where a tile's x reads live in its stage.
struct XsPlace {
    int32_t xpos;   // this lane's offset: stage element index of x[row0 + off]
    bool staged;    // K <= 32 and the runs fit the stage (warp-uniform)
    bool interior;  // every column of the tile inside [0, xn) (warp-uniform)
};

// U: stored values in flight per lane (one group per U offsets);
// SB: bytes of one stage (head + x runs).
template <typename VT, typename XT, int U, int SB>
__global__ void __launch_bounds__(kXsWarps * 32)
spmv_bw32_xs(const XsArgs<VT, XT> A, const XT *__restrict__ x, XT *__restrict__ y) {
    static_assert(SB % 128 == 0 && SB > static_cast<int>(sizeof(XsStageHead<XT>)), "bad stage size");
    static_assert(U >= 8 && U <= 32, "bad group size");
    constexpr int al = 16 / static_cast<int>(sizeof(XT));  // x elements per 16 bytes
    constexpr int kHead = (static_cast<int>(sizeof(XsStageHead<XT>)) + 127) & ~127;
    constexpr int kWinElems = (SB - kHead) / static_cast<int>(sizeof(XT));
    extern __shared__ __align__(128) unsigned char smraw[];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const SpmvArgs<VT, XT> &a = A.a;
    unsigned char *mine = smraw + static_cast<size_t>(w) * 2 * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw + static_cast<size_t>(kXsWarps) * 2 * SB) + w * 2;

    const int32_t W = static_cast<int32_t>(gridDim.x) * kXsWarps;
    const int32_t gw = static_cast<int32_t>(blockIdx.x) * kXsWarps + w;
    if (gw >= a.numTiles) return;  // warp-uniform; this warp's barriers stay unused
    const int32_t nT = (a.numTiles - gw + W - 1) / W;  // tiles of this warp
    if (lane == 0) {
        // lane 0's arrive.expect_tx + 32 cp.async arrivals per phase
        mbar_init(&bars[0], 1 + 32);
        mbar_init(&bars[1], 1 + 32);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    const uint32_t xn = static_cast<uint32_t>(a.xn);
    const int32_t xnAl = a.xn & ~(al - 1);
    auto tileOf = [&](int32_t j) { return gw + j * W; };

    // Stage tile j (meta m, this lane's offset `off`, COO entry (cr, cc, cv))
    // into stage j & 1.
    auto issue = [&](int32_t j, const TileMeta &m, int32_t off, int32_t cr, int32_t cc, XT cv) -> XsPlace {
        const int32_t t = tileOf(j);
        unsigned char *B = mine + (j & 1) * SB;
        uint64_t *bar = &bars[j & 1];
        XsStageHead<XT> &H = *reinterpret_cast<XsStageHead<XT> *>(B);
        XT *win = reinterpret_cast<XT *>(B + kHead);
        const int32_t row0 = t * 32;
        const int32_t K = m.k1 - m.k0;
        const bool act = lane < K;
        off = act ? off : 0;
        // runs of merged windows [off, off + 32)
        const int32_t prev = __shfl_up_sync(kFull, off, 1);
        const bool isStart = act && (lane == 0 || off > prev + 32);
        const unsigned starts = __ballot_sync(kFull, isStart);
        const unsigned le = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
        const unsigned after = starts & ~le;
        const int endLane = after ? __ffs(after) - 2 : min(K, 32) - 1;
        const int32_t endOff = __shfl_sync(kFull, off, endLane < 0 ? 0 : endLane);
        int32_t alo = 0, len = 0, bhi = 0, hi = 0;
        if (isStart) {
            const int64_t lo64 = max(int64_t(0), int64_t(row0) + off);
            const int64_t hi64 = min(int64_t(a.xn), int64_t(row0) + endOff + 32);
            if (hi64 > lo64) {
                hi = static_cast<int32_t>(hi64);
                alo = static_cast<int32_t>(lo64) & ~(al - 1);
                len = (hi - alo + al - 1) & ~(al - 1);
                bhi = min((hi + al - 1) & ~(al - 1), xnAl);
                if (bhi < alo) bhi = alo;
            }
        }
        int32_t incl = len;  // inclusive scan of run lengths (start lanes only)
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t u = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += u;
        }
        const int32_t P = incl - len;
        const int32_t xElems = __shfl_sync(kFull, incl, 31);
        XsPlace pl;
        pl.staged = K <= 32 && xElems <= kWinElems;
        const int myStart = act ? 31 - __clz(starts & le) : 0;
        const int32_t Pk = __shfl_sync(kFull, P, myStart);
        const int32_t alok = __shfl_sync(kFull, alo, myStart);
        pl.xpos = Pk + (row0 + off - alok);
        const int32_t offFirst = __shfl_sync(kFull, off, 0);
        const int32_t offLast = __shfl_sync(kFull, off, K > 0 && K <= 32 ? K - 1 : 0);
        pl.interior = K > 0 && int64_t(row0) + offFirst >= 0 && int64_t(row0) + 31 + offLast < int64_t(a.xn);
        const int32_t ncoo = min(m.c1 - m.c0, kXsCoo);
        if (lane < ncoo) {
            H.crow[lane] = cr;
            H.cval[lane] = cv;
            cp_async<sizeof(XT)>(&H.cx[lane], x + cc);
        }
        // an unaligned end of x (at most al - 1 elements): plain loads
        if (pl.staged && isStart && hi > bhi) {
            for (int32_t e = max(bhi, alo); e < hi; ++e) win[P + (e - alo)] = __ldg(x + e);
        }
        const bool skip = t == A.skipTile;
        if (!skip) cp_async_arrive_noinc(bar);
        int32_t tot = pl.staged && isStart ? (bhi - alo) * static_cast<int32_t>(sizeof(XT)) : 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) tot += __shfl_xor_sync(kFull, tot, d);
        if (lane == 0 && !skip) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(tot));
        __syncwarp();
        if (pl.staged && !skip && isStart && bhi > alo)
            bulk_g2s(win + P, x + alo, static_cast<uint32_t>(bhi - alo) * sizeof(XT), bar);
        return pl;
    };
    auto loadOffs = [&](const TileMeta &m) { return lane < m.k1 - m.k0 ? __ldg(a.offs + m.k0 + lane) : 0; };
    struct CooE {
        int32_t r, c;
        XT v;
    };
    auto loadCoo = [&](const TileMeta &m, int32_t t) {
        CooE e{0, 0, XT(0)};
        const int32_t ce = m.c0 + lane;
        if (ce < min(m.c1, m.c0 + kXsCoo)) {
            e.r = __ldg(a.cooRow + ce) - t * 32;
            e.c = __ldg(a.cooCol + ce);
            e.v = __ldg(a.cooVal + ce);
        }
        return e;
    };
    auto loadScale = [&](int32_t t) { return (a.scale && t < a.numBlocks) ? __ldg(a.scale + t) : 1.0f; };
    const TileMeta zero{0, 0, 0, 0};

    // tile 0: staged now; tile 1: frontier registers; tile 2: meta
    TileMeta mC = load_meta(a, tileOf(0));
    float sC = loadScale(tileOf(0));
    XsPlace pC;
    int32_t offC;
    {
        offC = loadOffs(mC);
        const CooE e = loadCoo(mC, tileOf(0));
        pC = issue(0, mC, offC, e.r, e.c, e.v);
    }
    TileMeta mN = nT > 1 ? load_meta(a, tileOf(1)) : zero;
    int32_t offN = loadOffs(mN);
    CooE eN = nT > 1 ? loadCoo(mN, tileOf(1)) : CooE{0, 0, XT(0)};
    float sN = nT > 1 ? loadScale(tileOf(1)) : 1.0f;
    TileMeta mNN = nT > 2 ? load_meta(a, tileOf(2)) : zero;

    for (int32_t i = 0; i < nT; ++i) {
        const int32_t t = tileOf(i);
        // stage tile i+1; ask L2 for its value rows
        XsPlace pN{0, false, false};
        if (i + 1 < nT) {
            pN = issue(i + 1, mN, offN, eN.r, eN.c, eN.v);
            if (lane == 0 && mN.k1 > mN.k0) {  // values of [k0, k1) are contiguous, 64-byte aligned
                const int64_t bytes = static_cast<int64_t>(mN.k1 - mN.k0) * 32 * static_cast<int64_t>(sizeof(VT));
                prefetch_l2_bulk(a.vals + static_cast<int64_t>(mN.k0) * 32,
                                 static_cast<uint32_t>(bytes < 32768 ? bytes : 32768));
            }
        }
        // tile i's values: the first group of up to U offsets in flight
        const int32_t K = mC.k1 - mC.k0;
        const int32_t row0 = t * 32;
        const int32_t row = row0 + lane;
        const VT *vp = a.vals + static_cast<int64_t>(mC.k0) * 32 + lane;
        VT v[U];
        if (pC.staged) {
#pragma unroll
            for (int u = 0; u < U; ++u) v[u] = u < K ? ld_stream(vp + u * 32) : VT(0);
        }
        // frontier: offsets / COO entries / scale of tile i+2, meta of tile i+3
        const TileMeta m2 = mNN;
        const int32_t off2 = i + 2 < nT ? loadOffs(m2) : 0;
        const CooE e2 = i + 2 < nT ? loadCoo(m2, tileOf(i + 2)) : CooE{0, 0, XT(0)};
        const float s2 = i + 2 < nT ? loadScale(tileOf(i + 2)) : 1.0f;
        mNN = i + 3 < nT ? load_meta(a, tileOf(i + 3)) : zero;

        unsigned char *B = mine + (i & 1) * SB;
        if (!mbar_wait(&bars[i & 1], static_cast<uint32_t>(i >> 1) & 1u, A.timeoutNs)) {
            // give up: record it, let the copies in flight land, return
            if (lane == 0) atomicOr(A.status, kErrConsumerWait);
            cp_async_wait_all();
            bool drained = true;
            for (int32_t j = i; j < min(nT, i + 2) && drained; ++j) {
                if (tileOf(j) == A.skipTile) continue;
                drained = mbar_wait(&bars[j & 1], static_cast<uint32_t>(j >> 1) & 1u, A.timeoutNs);
            }
            if (!drained && lane == 0) atomicOr(A.status, kErrDrain);
            __syncwarp();
            return;
        }
        const XsStageHead<XT> &H = *reinterpret_cast<const XsStageHead<XT> *>(B);
        const XT *win = reinterpret_cast<const XT *>(B + kHead) + lane;
        XT sum = XT(0);
        if (pC.staged) {
            // groups of U offsets (K <= 32): the first group's loads were
            // issued before the wait, later groups' loads go here
            for (int32_t g = 0; g < K; g += U) {
                if (g > 0) {
#pragma unroll
                    for (int u = 0; u < U; ++u) v[u] = g + u < K ? ld_stream(vp + (g + u) * 32) : VT(0);
                }
                if (pC.interior) {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        if (g + u < K) {
                            const XT xv = win[__shfl_sync(kFull, pC.xpos, g + u)];
                            const XT vv = widen<XT>(v[u], sC);
                            if (vv != XT(0)) sum = fma_rn(vv, xv, sum);
                        }
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        if (g + u < K) {
                            const int32_t col = row + __shfl_sync(kFull, offC, g + u);
                            const int32_t p = __shfl_sync(kFull, pC.xpos, g + u);
                            const XT vv = widen<XT>(v[u], sC);
                            if (static_cast<uint32_t>(col) < xn && vv != XT(0)) sum = fma_rn(vv, win[p], sum);
                        }
                    }
                }
            }
        } else if (K > 0) {
            sum = tile_dia_global<VT, XT>(a, x, mC.k0, K, row, sC);
        }
        if (a.hasCoo) {
            const int32_t nc = min(mC.c1 - mC.c0, kXsCoo);
            int lr = -1;
            XT p = XT(0);
            if (lane < nc) {
                lr = H.crow[lane];
                p = mul_rn(H.cval[lane], H.cx[lane]);
            }
            XT c = XT(0);
            for (int q = 0; q < nc; ++q) {
                const int rt = __shfl_sync(kFull, lr, q);
                const XT pt = __shfl_sync(kFull, p, q);
                if (rt == lane) c = add_rn(c, pt);
            }
            if (mC.c1 - mC.c0 > kXsCoo)  // rare: continue in list order from global memory
                c = tile_coo<XT>(a.cooRow, a.cooCol, a.cooVal, mC.c0 + kXsCoo, mC.c1, row0, lane, x, c);
            sum = add_rn(sum, c);
        }
        if (row < a.n) __stcs(y + row, sum);
        // this stage is refilled next iteration: reads before the async writes
        fence_proxy_async_smem();
        __syncwarp();
        // rotate the frontier
        mC = mN;
        sC = sN;
        offC = offN;
        pC = pN;
        mN = m2;
        offN = off2;
        eN = e2;
        sN = s2;
    }
}

}  // namespace dev
}  // namespace hbdia
