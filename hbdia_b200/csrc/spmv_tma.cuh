// Staged HBDIA SpMV for blockWidth 32 on sm_100a: a persistent,
// warp-specialised kernel.
//
// One CTA per SM walks the chunks (kTilesPerChunk consecutive 32-row tiles)
// blockIdx.x, blockIdx.x + gridDim.x, ...  A producer warp fills a ring of
// kStages shared-memory stages, one chunk per stage:
//   * the chunk's values (one contiguous cp.async.bulk with an L2 evict-first
//     hint: they are read once), its offsets and its COO remainder (rows,
//     values), each one cp.async.bulk completing on the stage's "full"
//     mbarrier through the transaction count;
//   * the x values its COO entries gather, with per-lane cp.async copies that
//     the same mbarrier tracks (cp.async.mbarrier.arrive.noinc);
//   * an L2 prefetch (cp.async.bulk.prefetch.L2) of the x windows the chunk's
//     diagonals read, so the consumers' x loads find their lines on chip.
// The producer's own metadata (chunk records, window tables, COO columns) is
// bulk-copied 2-4 chunks ahead onto per-slot mbarriers, so no producer step
// waits on a global-memory round trip (nor on the COO gathers in flight).
//
// kGroups groups of kTilesPerChunk consumer warps take the stages in turn
// (group g handles local steps g, g + kGroups, ...); within a group, warp w
// computes tile w of the chunk -- the reference's arithmetic in the
// reference's order (spmv_kernels.cuh) -- and the group releases the stage on
// its "empty" mbarrier.
//
// Chunks whose rows do not fit a stage and COO entries beyond a stage's
// capacity are read straight from global memory.
//
// Every wait is bounded by a time limit; on expiry the kernel records an error
// bit in *status, drains the copies it has in flight (again bounded) and
// returns.
#pragma once

#include "chunks.hpp"
#include "spmv_kernels.cuh"

namespace hbdia {
namespace dev {

constexpr int kStages = 6;
constexpr int kGroups = 3;                   // consumer groups (stages computed at once)
constexpr int kVRows = kTilesPerChunk * 32;  // stored offsets a stage holds
constexpr int kCCap = 128;                   // COO entries a stage holds
constexpr int kRecRing = 5;                  // chunk records in flight (distance 4)
constexpr int kMetaRing = 3;                 // window tables / COO columns in flight (distance 2)
constexpr int kConsumerWarps = kGroups * kTilesPerChunk;
constexpr int kTmaThreads = (kConsumerWarps + 1) * 32;
static_assert(kStages > kGroups, "stages must outnumber consumer groups");
// Each slot is then always consumed by the same group, which has finished the
// slot's previous phase before it waits on the next one, so a parity wait can
// never match a phase two uses old.
static_assert(kStages % kGroups == 0, "a slot must always belong to the same consumer group");

enum : int { kErrConsumerWait = 1, kErrProducerWait = 2, kErrDrain = 4 };

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// ---------------------------------------------------------------- layout
template <typename VT, typename XT>
struct __align__(16) Stage {
    VT vals[kVRows * 32];
    XT cval[kCCap + 16 / sizeof(XT)];
    XT xg[kCCap];
    int32_t offs[kVRows + 8];
    int32_t crow[kCCap + 8];
    int32_t hdr[kRecInts];
};

template <typename VT, typename XT>
struct __align__(16) TmaSmem {
    Stage<VT, XT> stage[kStages];
    int32_t rec[kRecRing][kRecInts];
    XWindow win[kMetaRing][kMaxWindows];
    int32_t cols[kMetaRing][kCCap + 8];
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t recBar[kRecRing];    // chunk record landed (bulk copy)
    uint64_t metaBar[kMetaRing];  // window table + COO columns landed (bulk copies)
};

template <typename VT, typename XT>
struct TmaArgs {
    SpmvArgs<VT, XT> a;
    const int32_t *rec;     // chunk records, kRecInts per chunk
    const XWindow *win;     // window lists (x ranges to prefetch into L2)
    int32_t numChunks;
    int32_t *status;        // error bits (0 = fine)
    uint64_t timeoutNs;     // limit of every wait
    int32_t skipChunk;      // test hook: the producer never publishes this chunk (-1: off)
};

// One tile straight from global memory (chunks that are not staged).
template <typename VT, typename XT>
__device__ __forceinline__ XT tile_direct(const SpmvArgs<VT, XT> &a, int32_t tile, int lane,
                                          const XT *__restrict__ x) {
    const int64_t row0 = static_cast<int64_t>(tile) * 32;
    const int64_t row = row0 + lane;
    XT sum = XT(0);
    if (tile < a.numBlocks) {
        const int32_t k0 = __ldg(a.blkOff + tile), k1 = __ldg(a.blkOff + tile + 1);
        const float s = a.scale ? __ldg(a.scale + tile) : 1.0f;
        for (int32_t k = k0; k < k1; ++k) {
            const XT v = widen<XT>(ld_stream(a.vals + static_cast<int64_t>(k) * 32 + lane), s);
            const int64_t col = row + __ldg(a.offs + k);
            if (v != XT(0) && col >= 0 && col < a.xn) sum = fma_rn(v, __ldg(x + col), sum);
        }
    }
    if (a.hasCoo) {
        const int32_t e0 = __ldg(a.cooTile + tile), e1 = __ldg(a.cooTile + tile + 1);
        sum = add_rn(sum, tile_coo<XT>(a.cooRow, a.cooCol, a.cooVal, e0, e1, row0, lane, x));
    }
    return sum;
}

// One tile from a staged chunk: values, offsets and the COO remainder from
// shared memory, x through L1 (its lines were prefetched into L2).
template <typename VT, typename XT, int U>
__device__ __forceinline__ XT tile_staged(const SpmvArgs<VT, XT> &a, const Stage<VT, XT> &S, int w, int lane,
                                          const XT *__restrict__ x) {
    const int32_t *H = S.hdr;
    const int32_t tile = H[kRecT0] + w;
    // 32-bit row/column arithmetic: the staged kernel runs only for n <= 2^30,
    // so row + offset (offsets lie in (-n, n)) cannot overflow
    const int32_t row0 = tile * 32;
    const int32_t row = row0 + lane;
    const int32_t k0c = H[kRecK0];
    const int32_t kt0 = H[kRecTileK + w], kt1 = H[kRecTileK + w + 1];
    const float s = (a.scale && tile < a.numBlocks) ? __ldg(a.scale + tile) : 1.0f;
    const int32_t *offs = S.offs + (kt0 - (k0c & ~3));
    const VT *vrow = S.vals + (kt0 - k0c) * 32 + lane;
    const int cnt = kt1 - kt0;
    const uint32_t n = static_cast<uint32_t>(a.xn);  // column bound
    XT sum = XT(0);
    int j = 0;
    // full groups of U offsets: U independent x loads in flight, then the
    // FMA chain in ascending offset order
    for (; j + U <= cnt; j += U) {
        int32_t col[U];
        bool ok[U];
        VT v[U];
        XT xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            col[u] = row + offs[j + u];
            ok[u] = static_cast<uint32_t>(col[u]) < n;
            v[u] = vrow[(j + u) * 32];
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
    for (; j < cnt; ++j) {
        const int32_t col = row + offs[j];
        const XT vv = widen<XT>(vrow[j * 32], s);
        if (static_cast<uint32_t>(col) < n && vv != XT(0)) sum = fma_rn(vv, __ldg(x + col), sum);
    }
    if (a.hasCoo) {
        const int32_t c0 = H[kRecC0], c1 = H[kRecC1];
        const int32_t crAl = c0 & ~3;
        const int32_t cvAl = c0 & ~(16 / static_cast<int>(sizeof(XT)) - 1);
        const int32_t ncs = min(c1 - c0, kCCap);
        const int32_t ct0 = H[kRecTileC + w], ct1 = H[kRecTileC + w + 1];
        XT c = XT(0);
        for (int32_t base = ct0; base < ct1; base += 32) {
            const int32_t e = base + lane;
            int lr = -1;
            XT p = XT(0);
            if (e < ct1) {
                int32_t r;
                XT v, xg;
                if (e - c0 < ncs) {
                    r = S.crow[e - crAl];
                    v = S.cval[e - cvAl];
                    xg = S.xg[e - c0];
                } else {
                    r = __ldg(a.cooRow + e);
                    v = __ldg(a.cooVal + e);
                    xg = __ldg(x + __ldg(a.cooCol + e));
                }
                lr = static_cast<int>(r - row0);
                p = mul_rn(v, xg);
            }
            const int m = min(32, ct1 - base);
            for (int t = 0; t < m; ++t) {
                const int rt = __shfl_sync(kFull, lr, t);
                const XT pt = __shfl_sync(kFull, p, t);
                if (rt == lane) c = add_rn(c, pt);
            }
        }
        sum = add_rn(sum, c);
    }
    return sum;
}

template <typename VT, typename XT, int U>
__global__ void __launch_bounds__(kTmaThreads, 1)
spmv_bw32_tma(const TmaArgs<VT, XT> T, const XT *__restrict__ x, XT *__restrict__ y) {
    extern __shared__ __align__(128) unsigned char smemRaw[];
    TmaSmem<VT, XT> &sm = *reinterpret_cast<TmaSmem<VT, XT> *>(smemRaw);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const SpmvArgs<VT, XT> &a = T.a;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sm.full[s], 1 + 32);            // producer arrive.expect_tx + 32 cp.async arrivals
            mbar_init(&sm.empty[s], kTilesPerChunk);   // one arrival per warp of the consuming group
        }
        for (int r = 0; r < kRecRing; ++r) mbar_init(&sm.recBar[r], 1);
        for (int r = 0; r < kMetaRing; ++r) mbar_init(&sm.metaBar[r], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int32_t G = gridDim.x;
    const int32_t first = blockIdx.x;
    // local step i handles chunk first + i * G
    const int32_t nSteps = first < T.numChunks ? (T.numChunks - first + G - 1) / G : 0;

    if (warp == kConsumerWarps) {
        // ------------------------------------------------------------ producer
        const uint64_t policy = l2_evict_first_policy();
        auto chunkOf = [&](int32_t i) { return first + i * G; };
        // The producer's own metadata arrives by bulk copies on per-slot
        // mbarriers, never through cp.async groups: waiting on a group would
        // also wait for the (older) COO x gathers, which are random DRAM reads.
        int32_t recIssued = 0, metaIssued = 0;
        auto prefetchRec = [&](int32_t i) {  // chunk record of step i
            if (i >= nSteps) return;
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive_expect_tx(&sm.recBar[i % kRecRing], kRecInts * 4);
                bulk_g2s(sm.rec[i % kRecRing], T.rec + static_cast<int64_t>(chunkOf(i)) * kRecInts, kRecInts * 4,
                         &sm.recBar[i % kRecRing]);
            }
            recIssued = i + 1;
        };
        auto waitRec = [&](int32_t i) {
            return mbar_wait(&sm.recBar[i % kRecRing], static_cast<uint32_t>(i / kRecRing) & 1u, T.timeoutNs);
        };
        auto waitMeta = [&](int32_t i) {
            return mbar_wait(&sm.metaBar[i % kMetaRing], static_cast<uint32_t>(i / kMetaRing) & 1u, T.timeoutNs);
        };
        auto prefetchMeta = [&](int32_t i) {  // window table + COO columns of step i; rec(i) has landed
            if (i >= nSteps) return;
            const int32_t *R = sm.rec[i % kRecRing];
            const bool staged = R[kRecFlags] & 1;
            const int32_t nWin = staged ? R[kRecNWin] : 0;
            const int32_t c0 = R[kRecC0];
            const int32_t ncs = staged ? min(R[kRecC1] - c0, kCCap) : 0;
            const int32_t colAl = c0 & ~3;
            const int32_t colEnd = ncs > 0 ? (c0 + ncs + 3) & ~3 : colAl;
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive_expect_tx(&sm.metaBar[i % kMetaRing],
                                      static_cast<uint32_t>(nWin) * 16u + static_cast<uint32_t>(colEnd - colAl) * 4u);
                if (nWin > 0)
                    bulk_g2s(sm.win[i % kMetaRing], T.win + R[kRecWin0], static_cast<uint32_t>(nWin) * 16u,
                             &sm.metaBar[i % kMetaRing]);
                if (colEnd > colAl)
                    bulk_g2s(sm.cols[i % kMetaRing], a.cooCol + colAl, static_cast<uint32_t>(colEnd - colAl) * 4u,
                             &sm.metaBar[i % kMetaRing]);
            }
            metaIssued = i + 1;
        };
        bool ok = true;
        for (int32_t i = 0; i < 4; ++i) prefetchRec(i);
        for (int32_t i = 0; i < 2 && i < nSteps && ok; ++i) {
            ok = waitRec(i);
            if (ok) prefetchMeta(i);
        }
        __syncwarp();
        int32_t issued = 0;
        for (int32_t i = 0; i < nSteps && ok; ++i) {
            const int slot = i % kStages;
            const uint32_t use = static_cast<uint32_t>(i / kStages);
            if (!waitRec(i) || !waitMeta(i) || !mbar_wait(&sm.empty[slot], (use & 1u) ^ 1u, T.timeoutNs)) {
                ok = false;
                break;
            }
            Stage<VT, XT> &S = sm.stage[slot];
            const int32_t *R = sm.rec[i % kRecRing];
            const XWindow *W = sm.win[i % kMetaRing];
            const bool staged = R[kRecFlags] & 1;
            if (lane < kRecInts) S.hdr[lane] = R[lane];
            __syncwarp();
            uint32_t bytes = 0;
            int32_t k0 = 0, k1 = 0, kAl = 0, kEnd = 0, c0 = 0, ncs = 0, crAl = 0, crEnd = 0, cvAl = 0, cvEnd = 0;
            if (staged) {
                k0 = R[kRecK0];
                k1 = R[kRecK1];
                kAl = k0 & ~3;
                kEnd = k1 > k0 ? (k1 + 3) & ~3 : kAl;
                c0 = R[kRecC0];
                ncs = min(R[kRecC1] - c0, kCCap);
                constexpr int vAl = 16 / static_cast<int>(sizeof(XT));
                crAl = c0 & ~3;
                crEnd = ncs > 0 ? (c0 + ncs + 3) & ~3 : crAl;
                cvAl = c0 & ~(vAl - 1);
                cvEnd = ncs > 0 ? (c0 + ncs + vAl - 1) & ~(vAl - 1) : cvAl;
                bytes = static_cast<uint32_t>(k1 - k0) * 32u * sizeof(VT) + static_cast<uint32_t>(kEnd - kAl) * 4u +
                        static_cast<uint32_t>(crEnd - crAl) * 4u + static_cast<uint32_t>(cvEnd - cvAl) * sizeof(XT);
            }
            const bool skip = chunkOf(i) == T.skipChunk;
            if (lane == 0 && !skip) mbar_arrive_expect_tx(&sm.full[slot], bytes);
            __syncwarp();
            if (staged && !skip) {
                if (lane == 0 && k1 > k0)
                    bulk_g2s_hint(S.vals, a.vals + static_cast<int64_t>(k0) * 32,
                                  static_cast<uint32_t>(k1 - k0) * 32u * sizeof(VT), &sm.full[slot], policy);
                if (lane == 1 && kEnd > kAl)
                    bulk_g2s(S.offs, a.offs + kAl, static_cast<uint32_t>(kEnd - kAl) * 4u, &sm.full[slot]);
                if (lane == 2 && crEnd > crAl)
                    bulk_g2s(S.crow, a.cooRow + crAl, static_cast<uint32_t>(crEnd - crAl) * 4u, &sm.full[slot]);
                if (lane == 3 && cvEnd > cvAl)
                    bulk_g2s(S.cval, a.cooVal + cvAl, static_cast<uint32_t>(cvEnd - cvAl) * sizeof(XT),
                             &sm.full[slot]);
                if (lane < R[kRecNWin]) {
                    const XWindow w = W[lane];
                    if (w.stagedEnd > w.alignedStart)
                        bulk_prefetch_l2(x + w.alignedStart,
                                         static_cast<uint32_t>(w.stagedEnd - w.alignedStart) * sizeof(XT));
                }
                const int32_t *cols = sm.cols[i % kMetaRing] + (c0 - (c0 & ~3));
                for (int32_t e = lane; e < ncs; e += 32) cp_async<sizeof(XT)>(&S.xg[e], x + cols[e]);
            }
            if (!skip) cp_async_arrive_noinc(&sm.full[slot]);
            __syncwarp();
            issued = i + 1;
            if (i + 2 < nSteps) {
                if (!waitRec(i + 2)) {
                    ok = false;
                    break;
                }
                prefetchMeta(i + 2);
            }
            prefetchRec(i + 4);
            __syncwarp();
        }
        if (!ok && lane == 0) atomicOr(T.status, kErrProducerWait);
        // drain: every copy this warp started has landed before the CTA exits
        cp_async_commit();
        cp_async_wait<0>();
        __syncwarp();
        bool drained = true;
        for (int32_t j = max(0, issued - kStages); j < issued && drained; ++j) {
            if (chunkOf(j) == T.skipChunk) continue;
            drained = mbar_wait(&sm.full[j % kStages], static_cast<uint32_t>(j / kStages) & 1u, T.timeoutNs);
        }
        for (int32_t j = max(0, recIssued - kRecRing); j < recIssued && drained; ++j) drained = waitRec(j);
        for (int32_t j = max(0, metaIssued - kMetaRing); j < metaIssued && drained; ++j) drained = waitMeta(j);
        if (!drained && lane == 0) atomicOr(T.status, kErrDrain);
    } else {
        // ------------------------------------------------------------ consumers
        const int group = warp / kTilesPerChunk;
        const int w = warp % kTilesPerChunk;
        for (int32_t i = group; i < nSteps; i += kGroups) {
            const int slot = i % kStages;
            const uint32_t use = static_cast<uint32_t>(i / kStages);
            if (!mbar_wait(&sm.full[slot], use & 1u, T.timeoutNs)) {
                if (lane == 0) atomicOr(T.status, kErrConsumerWait);
                break;
            }
            const Stage<VT, XT> &S = sm.stage[slot];
            const int32_t tile = S.hdr[kRecT0] + w;
            if (tile < a.numTiles) {
                const XT sum = (S.hdr[kRecFlags] & 1) ? tile_staged<VT, XT, U>(a, S, w, lane, x)
                                                      : tile_direct<VT, XT>(a, tile, lane, x);
                const int64_t row = static_cast<int64_t>(tile) * 32 + lane;
                if (row < a.n) __stcs(y + row, sum);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.empty[slot]);
        }
    }
}

}  // namespace dev
}  // namespace hbdia
