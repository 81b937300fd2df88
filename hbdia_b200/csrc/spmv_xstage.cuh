// Staged HBDIA SpMV for blockWidth 32 on sm_100a: each warp bulk-copies the
// value rows of its next tiles into its own shared-memory stages and gathers
// a tile's x values all at once.
//
// A 32-row tile's work in the reference's kernel (src/Operations/HBDIASpMV.cu:42-71)
// is one value load and one x gather per stored offset.  With values and x
// loaded into registers in groups (the pipelined kernel), a tile costs a few
// dependent round trips whatever the value width, so 4- and 2-byte value
// storage gains little over 8-byte: that kernel is latency-bound there.  Here
// a tile's value rows -- contiguous in the layout: [k0, k1) x 32 values --
// arrive by ONE bulk copy issued D - 1 tiles ahead into a ring of D stages per
// warp, completing on the stage's mbarrier, so the value stream is in flight
// without holding registers; the tile's x gathers (one per offset, up to 32)
// are then issued together, one round trip, and the FMA chain reads the
// values from shared memory.
//
// (A variant that also staged the tile's merged x runs -- about 9 bulk copies
// of ~272 bytes per 27-point tile -- measured 0.57 / 0.33 of the byte
// roofline in FP64 / FP32 at 256^3: the many small copies and the run
// bookkeeping made every tile slow, and its time fell only with more warps.)
//
// Persistent: warp g of W walks tiles g, g + W, ... (neighbouring warps on
// neighbouring tiles, so x lines are shared through L1/L2).  Per tile i the
// warp
//   * issues the value copy of tile i + D - 1 and the cp.async gathers of x for
//     that tile's first 32 COO entries, and records the tile's offsets and
//     block pointers in the stage head;
//   * loads the offsets / COO entries / scale of tile i + D and the block
//     pointers of tile i + D + 1 (registers, consumed next iteration);
//   * gathers tile i's x values, waits for its stage and runs the FMA chain,
//     then the COO remainder.
// Tiles with more than 32 offsets run from global memory (same arithmetic);
// COO entries past the first 32 of a tile are read from global memory too.
//
// Arithmetic is the reference's, in the reference's order (spmv_kernels.cuh):
// per row, offsets ascending, stored zeros and columns outside [0, xn)
// skipped, fma; then the COO remainder in list order with separately rounded
// multiply and add; y = dia + coo.  Interior tiles (every column of every
// offset inside [0, xn)) skip the column bound check, which cannot fail there.
//
// Every wait is bounded by a time limit; on expiry the kernel records an error
// bit in *status, waits (again bounded) for the copies it has in flight and
// returns.  No multicast anywhere: each warp copies into its own CTA's shared
// memory.
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
constexpr int kXsCoo = 32;    // COO entries a stage holds
constexpr int kXsHead = 896;  // bytes of a stage's head (below)

// A stage's head: what the warp knew about the tile when it issued its copy,
// read back when it computes the tile.
template <typename XT>
struct XsStageHead {
    int32_t off[32];       // offset k of the tile (k < min(K, 32))
    int32_t crow[kXsCoo];  // local row of each staged COO entry
    int32_t meta[8];       // K, k0, c0, c1, scale bits
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

// Bytes of one stage: head and the value rows of up to 32 offsets.
template <typename VT>
__host__ __device__ constexpr int xs_stage_bytes() {
    return kXsHead + 32 * 32 * static_cast<int>(sizeof(VT));
}

// Bytes of dynamic shared memory of one CTA: NW warps x D stages of SB bytes
// plus one mbarrier per stage.
__host__ __device__ constexpr size_t xs_smem_bytes(int NW, int D, int SB) {
    return static_cast<size_t>(NW) * D * SB + static_cast<size_t>(NW) * D * sizeof(uint64_t);
}

// The DIA part of one tile from global memory (tiles with more than 32
// offsets): offsets in masked groups of 8 (loads in flight together),
// ascending order.
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

// NW warps per CTA, D stages of SB bytes per warp (head, then the value rows).
template <typename VT, typename XT, int NW, int D, int SB>
__global__ void __launch_bounds__(NW * 32, 1)
spmv_bw32_xs(const XsArgs<VT, XT> A, const XT *__restrict__ x, XT *__restrict__ y) {
    constexpr int kVal = 32 * 32 * static_cast<int>(sizeof(VT));  // value rows of 32 offsets
    static_assert(sizeof(XsStageHead<XT>) <= kXsHead, "stage head too large");
    static_assert(SB % 128 == 0 && SB >= kXsHead + kVal, "bad stage size");
    static_assert(D >= 2, "need at least two stages");
    extern __shared__ __align__(128) unsigned char smraw[];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const SpmvArgs<VT, XT> &a = A.a;
    unsigned char *mine = smraw + static_cast<size_t>(w) * D * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw + static_cast<size_t>(NW) * D * SB) + w * D;

    const int32_t W = static_cast<int32_t>(gridDim.x) * NW;
    const int32_t gw = static_cast<int32_t>(blockIdx.x) * NW + w;
    if (gw >= a.numTiles) return;  // warp-uniform; this warp's barriers stay unused
    const int32_t nT = (a.numTiles - gw + W - 1) / W;  // tiles of this warp
    if (lane == 0) {
        // lane 0's arrive.expect_tx + 32 cp.async arrivals per phase
#pragma unroll
        for (int d = 0; d < D; ++d) mbar_init(&bars[d], 1 + 32);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    const uint32_t xn = static_cast<uint32_t>(a.xn);
    auto tileOf = [&](int32_t j) { return gw + j * W; };

    struct Front {  // what issuing a tile needs, loaded one iteration ahead
        TileMeta m;
        int32_t off;  // lane k: offset k of the tile (k < min(K, 32))
        int32_t cr, cc;
        XT cv;
        float s;
    };
    auto loadFront = [&](const TileMeta &m, int32_t t) {
        Front f;
        f.m = m;
        f.off = lane < m.k1 - m.k0 ? __ldg(a.offs + m.k0 + lane) : 0;
        f.cr = 0;
        f.cc = 0;
        f.cv = XT(0);
        const int32_t ce = m.c0 + lane;
        if (ce < min(m.c1, m.c0 + kXsCoo)) {
            f.cr = __ldg(a.cooRow + ce) - t * 32;
            f.cc = __ldg(a.cooCol + ce);
            f.cv = __ldg(a.cooVal + ce);
        }
        f.s = (a.scale && t < a.numBlocks) ? __ldg(a.scale + t) : 1.0f;
        return f;
    };

    // Stage tile j: its head, its COO x values (cp.async) and its value rows
    // (one bulk copy), completing on stage j % D's barrier.
    auto issue = [&](int32_t j, const Front &f) {
        const int32_t t = tileOf(j);
        unsigned char *B = mine + (j % D) * SB;
        uint64_t *bar = &bars[j % D];
        XsStageHead<XT> &H = *reinterpret_cast<XsStageHead<XT> *>(B);
        const int32_t K = f.m.k1 - f.m.k0;
        if (lane < K) H.off[lane] = f.off;
        if (lane == 0) {
            H.meta[0] = K;
            H.meta[1] = f.m.k0;
            H.meta[2] = f.m.c0;
            H.meta[3] = f.m.c1;
            H.meta[4] = __float_as_int(f.s);
        }
        const int32_t ncoo = min(f.m.c1 - f.m.c0, kXsCoo);
        if (lane < ncoo) {
            H.crow[lane] = f.cr;
            H.cval[lane] = f.cv;
            cp_async<sizeof(XT)>(&H.cx[lane], x + f.cc);
        }
        const bool skip = t == A.skipTile;
        if (!skip) cp_async_arrive_noinc(bar);
        __syncwarp();
        if (lane == 0 && !skip) {
            // the tile's value rows: contiguous, 64-byte aligned
            const uint32_t valBytes = K > 0 && K <= 32 ? static_cast<uint32_t>(K) * 32u * sizeof(VT) : 0u;
            mbar_arrive_expect_tx(bar, valBytes);
            if (valBytes) bulk_g2s(B + kXsHead, a.vals + static_cast<int64_t>(f.m.k0) * 32, valBytes, bar);
        }
    };

    // prologue: tiles 0 .. D-2 staged, tile D-1's front in registers
    TileMeta mNext = load_meta(a, tileOf(0));
    for (int32_t j = 0; j < D - 1; ++j) {
        if (j < nT) {
            const Front f = loadFront(mNext, tileOf(j));
            mNext = j + 1 < nT ? load_meta(a, tileOf(j + 1)) : TileMeta{0, 0, 0, 0};
            issue(j, f);
        }
    }
    Front F = D - 1 < nT ? loadFront(mNext, tileOf(D - 1)) : Front{};
    mNext = D < nT ? load_meta(a, tileOf(D)) : TileMeta{0, 0, 0, 0};

    for (int32_t i = 0; i < nT; ++i) {
        const int32_t t = tileOf(i);
        // stage tile i + D - 1, then fetch the front of the tile after it
        if (i + D - 1 < nT) issue(i + D - 1, F);
        if (i + D < nT) {
            F = loadFront(mNext, tileOf(i + D));
            mNext = i + D + 1 < nT ? load_meta(a, tileOf(i + D + 1)) : TileMeta{0, 0, 0, 0};
        }
        unsigned char *B = mine + (i % D) * SB;
        const XsStageHead<XT> &H = *reinterpret_cast<const XsStageHead<XT> *>(B);
        // the head was written by this warp when the tile was issued
        const int32_t K = H.meta[0];
        const int32_t row0 = t * 32;
        const int32_t row = row0 + lane;
        // interior tile (every column of every offset inside [0, xn), at most
        // 32 offsets): no column checks, x read at x + row + offset
        const bool interior = K > 0 && K <= 32 && int64_t(row0) + H.off[0] >= 0 &&
                              int64_t(row0) + 31 + H.off[K - 1] < int64_t(a.xn);
        // this tile's x gathers, all in flight before the wait
        XT xv[32];
        uint32_t okMask = 0;
        if (interior) {
            const XT *xr = x + row;
#pragma unroll
            for (int k = 0; k < 32; ++k)
                if (k < K) xv[k] = __ldg(xr + H.off[k]);  // warp-uniform bound; broadcast read of the offset
        } else if (K <= 32) {
            const int32_t myoff = lane < K ? H.off[lane] : 0;
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                if (k < K) {  // warp-uniform
                    const int32_t col = row + __shfl_sync(kFull, myoff, k);
                    const bool ok = static_cast<uint32_t>(col) < xn;
                    okMask |= ok ? (1u << k) : 0u;
                    xv[k] = ok ? __ldg(x + col) : XT(0);
                }
            }
        }
        if (!mbar_wait(&bars[i % D], static_cast<uint32_t>(i / D) & 1u, A.timeoutNs)) {
            // give up: record it, let the copies in flight land, return
            if (lane == 0) atomicOr(A.status, kErrConsumerWait);
            cp_async_wait_all();
            bool drained = true;
            for (int32_t j = i; j < min(nT, i + D) && drained; ++j) {
                if (tileOf(j) == A.skipTile) continue;
                drained = mbar_wait(&bars[j % D], static_cast<uint32_t>(j / D) & 1u, A.timeoutNs);
            }
            if (!drained && lane == 0) atomicOr(A.status, kErrDrain);
            __syncwarp();
            return;
        }
        const int32_t c0 = H.meta[2], c1 = H.meta[3];
        const float s = __int_as_float(H.meta[4]);
        const VT *vals = reinterpret_cast<const VT *>(B + kXsHead) + lane;
        XT sum = XT(0);
        if (interior) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                if (k < K) {  // warp-uniform
                    const XT vv = widen<XT>(vals[k * 32], s);
                    if (vv != XT(0)) sum = fma_rn(vv, xv[k], sum);
                }
            }
        } else if (K <= 32) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                if (k < K) {  // warp-uniform
                    const XT vv = widen<XT>(vals[k * 32], s);
                    if (((okMask >> k) & 1u) && vv != XT(0)) sum = fma_rn(vv, xv[k], sum);
                }
            }
        } else {
            sum = tile_dia_global<VT, XT>(a, x, H.meta[1], K, row, s);
        }
        if (a.hasCoo) {
            const int32_t nc = min(c1 - c0, kXsCoo);
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
            if (c1 - c0 > kXsCoo)  // rare: continue in list order from global memory
                c = tile_coo<XT>(a.cooRow, a.cooCol, a.cooVal, c0 + kXsCoo, c1, row0, lane, x, c);
            sum = add_rn(sum, c);
        }
        if (row < a.n) __stcs(y + row, sum);
        // this stage is refilled D - 1 iterations from now: reads before the async writes
        fence_proxy_async_smem();
        __syncwarp();
    }
}

}  // namespace dev
}  // namespace hbdia
