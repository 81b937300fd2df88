// Device layout (prepareForGPU, src/Format/HBDIA.cpp:720-816, in this
// library's form) and the SpMV launchers.
//
// HBM layout of one plan, a single allocation with 256-byte aligned parts:
//   vals      storage-type values, [block][offsetIdx][lane]   (slots)
//   scale     float per block (bf16 storage only)
//   offs      int32 kept offsets, ascending per block           (totalOffsets)
//   blkOff    int32 block -> first offset index                 (numBlocks + 1)
//   cooRow/cooCol int32, cooVal T: the COO remainder, row-sorted (nCoo)
//   cooRowPtr int32 CSR row pointer of the remainder            (numRows + 1)
//   cooTile   int32 first remainder entry of each 32-row tile   (numTiles + 1)

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "args.cuh"
#include "hbdia_internal.hpp"
#include "spmv_kernels.cuh"
#include "spmv_quad.cuh"
#include "spmv_xstage.cuh"
#include "spmm_kernels.cuh"

namespace hbdia {

void check_cuda(int err, const char *what) {
    if (err != cudaSuccess) {
        throw Error(err == cudaErrorMemoryAllocation ? HBDIA_ERR_NO_MEMORY : HBDIA_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(static_cast<cudaError_t>(err)));
    }
}

std::atomic<int64_t> g_deviceAllocs{0}, g_pinnedAllocs{0};

int dev_alloc_bytes(void **p, size_t bytes) {
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) g_deviceAllocs.fetch_add(1, std::memory_order_relaxed);
    return e;
}

int pinned_alloc_bytes(void **p, size_t bytes) {
    const cudaError_t e = cudaMallocHost(p, bytes);
    if (e == cudaSuccess) g_pinnedAllocs.fetch_add(1, std::memory_order_relaxed);
    return e;
}

void allocation_counts(int64_t *device, int64_t *pinned) {
    *device = g_deviceAllocs.load();
    *pinned = g_pinnedAllocs.load();
}

namespace {

constexpr int kUnroll = 9;  // offsets in flight per lane in the bw == 32 kernels

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t storage_bytes(int storage, int dtype) {
    if (storage == HBDIA_STORE_F32) return 4;
    if (storage == HBDIA_STORE_BF16_SCALED) return 2;
    return dtype == HBDIA_F32 ? 4 : 8;
}

}  // namespace

bool tail_heavy(const std::vector<int32_t> &hist) {
    // a block's offsets go in chunks of 32, each in groups of kUnroll
    int64_t tail = 0, total = 0;
    for (size_t d = 0; d < hist.size(); ++d) {
        const int64_t dd = static_cast<int64_t>(d);
        tail += hist[d] * ((dd / 32) * (32 % kUnroll) + (dd % 32) % kUnroll);
        total += hist[d] * dd;
    }
    return total > 0 && 2 * tail >= total;
}

void free_plan(DevicePlan &P) {
    if (P.stream) {
        cudaStreamSynchronize(static_cast<cudaStream_t>(P.stream));
        cudaStreamDestroy(static_cast<cudaStream_t>(P.stream));
    }
    if (P.base) cudaFree(P.base);
    if (P.xScratch) cudaFree(P.xScratch);
    if (P.yScratch) cudaFree(P.yScratch);
    P = DevicePlan();
}

template <typename T>
void build_plan(const HostLayout<T> &L, int storage, DevicePlan &P, const ColumnWindow *W) {
    DevicePlan Q;
    Q.kernel = P.kernel;  // settings survive a rebuild
    Q.waitTimeoutNs = P.waitTimeoutNs;
    Q.skipTile = P.skipTile;
    Q.xsConfig = P.xsConfig;
    Q.quadGroup = P.quadGroup;
    Q.unroll = P.unroll;
    Q.prefetchL2 = P.prefetchL2;
    Q.maskedTail = P.maskedTail;
    Q.tailHeavy = tail_heavy(L.histBlocks);
    free_plan(P);
    Q.dtype = std::is_same<T, float>::value ? HBDIA_F32 : HBDIA_F64;
    if (storage != HBDIA_STORE_NATIVE && Q.dtype != HBDIA_F64)
        throw Error(HBDIA_ERR_UNSUPPORTED, "reduced value storage needs a double matrix");
    if (storage < HBDIA_STORE_NATIVE || storage > HBDIA_STORE_BF16_QUAD)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown value storage");
    // the quad-interleaved storages hold F32 / BF16 values for the quad kernel
    Q.quadLayout = storage == HBDIA_STORE_F32_QUAD || storage == HBDIA_STORE_BF16_QUAD;
    if (Q.quadLayout) {
        if (L.blockWidth != 32 || L.numRows > (1 << 30))
            throw Error(HBDIA_ERR_UNSUPPORTED, "quad-interleaved storage needs blockWidth 32 and numRows <= 2^30");
        storage = storage == HBDIA_STORE_F32_QUAD ? HBDIA_STORE_F32 : HBDIA_STORE_BF16_SCALED;
    }
    Q.storage = storage;
    Q.n = L.numRows;
    Q.numCols = W ? W->len : L.numCols;
    Q.xn = W ? W->len : L.numRows;
    Q.bw = L.blockWidth;
    Q.numBlocks = L.numBlocks;
    Q.numTiles = static_cast<int32_t>((static_cast<int64_t>(L.numRows) + 31) / 32);
    Q.totalOffsets = static_cast<int64_t>(L.offsets.size());
    Q.slots = static_cast<int64_t>(L.data.size());
    Q.nCoo = static_cast<int64_t>(L.cooRow.size());

    // The fused kernels walk the COO remainder row by row: use a stable
    // row-sorted copy when the input order was not row-sorted (the reference
    // assumes row-sorted input here, src/Format/HBDIA.cpp:671-703).
    const int32_t *cr = L.cooRow.data(), *cc = L.cooCol.data();
    const T *cv = L.cooVal.data();
    const int32_t *crp = L.cooRowPtr.data();
    // a partial matrix's plan works in x-window coordinates: offsets become
    // col - lo - localRow, COO columns col - lo
    const int32_t *ko = L.offsets.data();
    std::vector<int32_t> wOffs, wCols;
    if (W) {
        wOffs.resize(L.offsets.size());
        for (size_t k = 0; k < wOffs.size(); ++k) wOffs[k] = L.offsets[k] + (W->rowBase - W->lo);
        wCols.resize(L.cooCol.size());
        for (size_t e = 0; e < wCols.size(); ++e) wCols[e] = L.cooCol[e] - W->lo;
        ko = wOffs.data();
        cc = wCols.data();
    }
    std::vector<int32_t> sr, sc, srp;
    std::vector<T> sv;
    for (int64_t e = 0; e < Q.nCoo; ++e) {
        if (cr[e] < 0 || cr[e] >= Q.n || cc[e] < 0 || cc[e] >= Q.numCols)
            throw Error(HBDIA_ERR_OUT_OF_RANGE, "COO entry (" + std::to_string(cr[e]) + ", " +
                                                     std::to_string(cc[e]) + ") outside the matrix");
    }
    if (!L.cooRowSorted) {
        std::vector<int64_t> order = stable_row_order(L.cooRow, Q.n);
        sr.resize(Q.nCoo);
        sc.resize(Q.nCoo);
        sv.resize(Q.nCoo);
        for (int64_t e = 0; e < Q.nCoo; ++e) {
            sr[e] = cr[order[e]];
            sc[e] = cc[order[e]];
            sv[e] = cv[order[e]];
        }
        srp.assign(static_cast<size_t>(Q.n) + 1, 0);
        for (int64_t e = 0; e < Q.nCoo; ++e) srp[sr[e] + 1]++;
        for (int32_t r = 0; r < Q.n; ++r) srp[r + 1] += srp[r];
        cr = sr.data();
        cc = sc.data();
        cv = sv.data();
        crp = srp.data();
    }
    std::vector<int32_t> tile(static_cast<size_t>(Q.numTiles) + 1);
    for (int64_t t = 0; t <= Q.numTiles; ++t) tile[t] = crp[std::min<int64_t>(t * 32, Q.n)];

    // host-side value conversion for reduced storage
    const size_t vsz = storage_bytes(storage, Q.dtype);
    std::vector<float> vf, sf;
    std::vector<__nv_bfloat16> vb;
    const void *valSrc = L.data.data();
    if (storage == HBDIA_STORE_F32) {
        vf.resize(Q.slots);
        for (int64_t i = 0; i < Q.slots; ++i) vf[i] = static_cast<float>(L.data[i]);
        valSrc = vf.data();
    } else if (storage == HBDIA_STORE_BF16_SCALED) {
        vb.resize(Q.slots);
        sf.assign(static_cast<size_t>(Q.numBlocks), 1.0f);
        for (int32_t b = 0; b < Q.numBlocks; ++b) {
            const int64_t s0 = static_cast<int64_t>(L.blockStart[b]) * Q.bw;
            const int64_t s1 = static_cast<int64_t>(L.blockStart[b + 1]) * Q.bw;
            double m = 0.0;
            for (int64_t i = s0; i < s1; ++i) m = std::max(m, std::fabs(static_cast<double>(L.data[i])));
            const float s = m > 0.0 ? static_cast<float>(m) : 1.0f;
            sf[b] = s;
            for (int64_t i = s0; i < s1; ++i)
                vb[i] = __float2bfloat16_rn(static_cast<float>(static_cast<double>(L.data[i]) / s));
        }
        valSrc = vb.data();
    }
    if (Q.quadLayout) {
        // uniform quads (the quad kernel's run-time test: four blocks, one list
        // of 1-32 offsets) go [offset][lane][block]
        const int32_t *bs = L.blockStart.data();
        auto interleave = [&](auto &v) {
            using E = typename std::remove_reference<decltype(v)>::type::value_type;
            std::vector<E> tmp;
            for (int64_t b0 = 0; b0 + 4 <= Q.numBlocks; b0 += 4) {
                const int32_t K = bs[b0 + 1] - bs[b0];
                if (K < 1 || K > 32) continue;
                bool uni = bs[b0 + 2] - bs[b0 + 1] == K && bs[b0 + 3] - bs[b0 + 2] == K && bs[b0 + 4] - bs[b0 + 3] == K;
                for (int32_t q = 1; uni && q < 4; ++q)
                    for (int32_t k = 0; uni && k < K; ++k) uni = L.offsets[bs[b0 + q] + k] == L.offsets[bs[b0] + k];
                if (!uni) continue;
                const int64_t base = static_cast<int64_t>(bs[b0]) * 32;
                tmp.assign(v.begin() + base, v.begin() + base + 4 * 32 * K);
                for (int32_t q = 0; q < 4; ++q)
                    for (int32_t k = 0; k < K; ++k)
                        for (int32_t l = 0; l < 32; ++l)
                            v[base + (static_cast<int64_t>(k) * 32 + l) * 4 + q] = tmp[(static_cast<int64_t>(q) * K + k) * 32 + l];
            }
        };
        if (storage == HBDIA_STORE_F32) interleave(vf);
        else interleave(vb);
    }

    // one allocation
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += align256(bytes);
        return o;
    };
    const size_t oVals = carve(Q.slots * vsz);
    const size_t oScale = carve(storage == HBDIA_STORE_BF16_SCALED ? Q.numBlocks * sizeof(float) : 0);
    const size_t oOffs = carve(Q.totalOffsets * sizeof(int32_t));
    const size_t oBlk = carve((static_cast<size_t>(Q.numBlocks) + 1) * sizeof(int32_t));
    const size_t oCR = carve(Q.nCoo * sizeof(int32_t));
    const size_t oCC = carve(Q.nCoo * sizeof(int32_t));
    const size_t oCV = carve(Q.nCoo * sizeof(T));
    const size_t oRP = carve((static_cast<size_t>(Q.n) + 1) * sizeof(int32_t));
    const size_t oTile = carve((static_cast<size_t>(Q.numTiles) + 1) * sizeof(int32_t));
    const size_t oStatus = carve(sizeof(int32_t));
    Q.bytes = off;
    check_cuda(dev_alloc(&Q.base, Q.bytes), "cudaMalloc(matrix layout)");
    char *base = static_cast<char *>(Q.base);
    try {
        Q.vals = base + oVals;
        Q.scale = storage == HBDIA_STORE_BF16_SCALED ? reinterpret_cast<float *>(base + oScale) : nullptr;
        Q.offs = reinterpret_cast<int32_t *>(base + oOffs);
        Q.blkOff = reinterpret_cast<int32_t *>(base + oBlk);
        Q.cooRow = reinterpret_cast<int32_t *>(base + oCR);
        Q.cooCol = reinterpret_cast<int32_t *>(base + oCC);
        Q.cooVal = base + oCV;
        Q.cooRowPtr = reinterpret_cast<int32_t *>(base + oRP);
        Q.cooTile = reinterpret_cast<int32_t *>(base + oTile);
        Q.status = reinterpret_cast<int32_t *>(base + oStatus);
        check_cuda(cudaMemset(Q.status, 0, sizeof(int32_t)), "cudaMemset(status)");
        auto up = [](void *dst, const void *src, size_t bytes) {
            if (bytes) check_cuda(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(layout)");
        };
        up(Q.vals, valSrc, Q.slots * vsz);
        if (Q.scale) up(Q.scale, sf.data(), Q.numBlocks * sizeof(float));
        up(Q.offs, ko, Q.totalOffsets * sizeof(int32_t));
        up(Q.blkOff, L.blockStart.data(), (static_cast<size_t>(Q.numBlocks) + 1) * sizeof(int32_t));
        up(Q.cooRow, cr, Q.nCoo * sizeof(int32_t));
        up(Q.cooCol, cc, Q.nCoo * sizeof(int32_t));
        up(Q.cooVal, cv, Q.nCoo * sizeof(T));
        up(Q.cooRowPtr, crp, (static_cast<size_t>(Q.n) + 1) * sizeof(int32_t));
        up(Q.cooTile, tile.data(), (static_cast<size_t>(Q.numTiles) + 1) * sizeof(int32_t));
        cudaStream_t s;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        Q.stream = s;
        check_cuda(cudaGetDevice(&Q.device), "cudaGetDevice");
    } catch (...) {
        free_plan(Q);
        throw;
    }

    // Algorithmic HBM bytes of one SpMV: every stored value, offset and index
    // read once, x read once, y written once, one x gather per COO entry.
    const int64_t xs = static_cast<int64_t>(sizeof(T));
    int64_t bytes = Q.slots * static_cast<int64_t>(vsz) + 4 * Q.totalOffsets +
                    4 * (static_cast<int64_t>(Q.numBlocks) + 1) + 2 * xs * Q.n +
                    (8 + xs) * Q.nCoo + xs * Q.nCoo;
    if (Q.scale) bytes += 4 * static_cast<int64_t>(Q.numBlocks);
    if (Q.nCoo > 0) bytes += Q.bw == 32 ? 4 * (static_cast<int64_t>(Q.numTiles) + 1)
                                        : 4 * (static_cast<int64_t>(Q.n) + 1);
    Q.bytesPerSpmv = bytes;
    P = Q;
}

template void build_plan<double>(const HostLayout<double> &, int, DevicePlan &, const ColumnWindow *);
template void build_plan<float>(const HostLayout<float> &, int, DevicePlan &, const ColumnWindow *);

namespace {

// The device a plan's kernels run on: the one its layout lives on (a stream
// query would fail while the stream is being captured into a graph).
int plan_device(const DevicePlan &P) {
    if (P.device >= 0) return P.device;
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    return dev;
}

// The staged kernel with NW warps per CTA and D stages per warp; as many
// CTAs as fit on all SMs at once (shared memory decides: one per SM).
template <typename VT, typename XT, int NW, int D>
void launch_xs_cfg(const dev::XsArgs<VT, XT> &A, const XT *x, XT *y, cudaStream_t s, int device) {
    constexpr int SB = dev::xs_stage_bytes<VT>();
    auto kernel = dev::spmv_bw32_xs<VT, XT, NW, D, SB>;
    constexpr size_t smem = dev::xs_smem_bytes(NW, D, SB);
    static_assert(smem <= 232448, "staged SpMV stages too large for one CTA");
    constexpr int threads = NW * 32;
    // bit d: the shared-memory opt-in is in place on device d.  Several host
    // threads (a server's scheduler and solver threads) launch at once.
    static std::atomic<uint64_t> configured{0};
    const uint64_t bit = uint64_t(1) << (device < 63 ? device : 63);
    if (device >= 63 || !(configured.load(std::memory_order_acquire) & bit)) {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "cudaFuncSetAttribute(staged SpMV)");
        if (device < 63) configured.fetch_or(bit, std::memory_order_acq_rel);
    }
    int sms = 0, perSm = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t ctasNeeded = (static_cast<int64_t>(A.a.numTiles) + NW - 1) / NW;
    const unsigned grid = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>(ctasNeeded, int64_t(sms) * std::max(1, perSm))));
    kernel<<<grid, threads, smem, s>>>(A, x, y);
}

// Staged kernel shapes (HBDIA_TUNE_STAGES), warps per CTA x stages per warp:
// 1 = 8 x 2, 2 = 12 x 2, 3 = 16 x 2, 4 = 12 x 3, 5 = 16 x 4; 0 = the default:
// 12 x 2 for 8-byte values, 16 x 2 for 4-byte, 16 x 3 for 2-byte.  A shape
// whose stages do not fit one CTA's shared memory runs the default.
template <typename VT, typename XT, int NW, int D>
constexpr bool xs_fits() {
    return dev::xs_smem_bytes(NW, D, dev::xs_stage_bytes<VT>()) <= 232448;
}

template <typename VT, typename XT>
void launch_xs(const dev::XsArgs<VT, XT> &A, int32_t cfg, const XT *x, XT *y, cudaStream_t s, int device) {
    switch (cfg) {
        case 1: return launch_xs_cfg<VT, XT, 8, 2>(A, x, y, s, device);
        case 2: return launch_xs_cfg<VT, XT, 12, 2>(A, x, y, s, device);
        case 3:
            if constexpr (xs_fits<VT, XT, 16, 2>()) return launch_xs_cfg<VT, XT, 16, 2>(A, x, y, s, device);
            break;
        case 4:
            if constexpr (xs_fits<VT, XT, 12, 3>()) return launch_xs_cfg<VT, XT, 12, 3>(A, x, y, s, device);
            break;
        case 5:
            if constexpr (xs_fits<VT, XT, 16, 4>()) return launch_xs_cfg<VT, XT, 16, 4>(A, x, y, s, device);
            break;
        default: break;
    }
    if constexpr (sizeof(VT) == 8) return launch_xs_cfg<VT, XT, 12, 2>(A, x, y, s, device);
    else if constexpr (sizeof(VT) == 4) return launch_xs_cfg<VT, XT, 16, 2>(A, x, y, s, device);
    else return launch_xs_cfg<VT, XT, 16, 3>(A, x, y, s, device);
}

// Persistent grid: as many 256-thread CTAs as fit on all SMs at once (the
// warps then walk the tiles grid-stride).
template <typename VT, typename XT, typename Kernel>
void launch_pipe(Kernel kernel, const dev::SpmvArgs<VT, XT> &a, int32_t numTiles, const XT *x, XT *y,
                 cudaStream_t s, int device, int threads = 256) {
    int sms = 0, perSm = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, 0),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t warpsPerCta = threads / 32;
    const int64_t ctasNeeded = (static_cast<int64_t>(numTiles) + warpsPerCta - 1) / warpsPerCta;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(ctasNeeded,
                                                                                       int64_t(sms) * std::max(1, perSm))));
    kernel<<<grid, threads, 0, s>>>(a, x, y);
}

// The quad kernel: U offsets of four blocks in flight per lane (default 4
// for 4- and 2-byte values, 2 for 8-byte ones), L2 prefetch of the next
// quad's values when x exceeds L2 (the pipelined kernel's rule).
template <typename VT, typename XT>
void launch_quad(const DevicePlan &P, const dev::SpmvArgs<VT, XT> &a, const XT *x, XT *y, cudaStream_t s) {
    int l2 = 0;
    const int device = plan_device(P);
    check_cuda(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device), "cudaDeviceGetAttribute(L2)");
    // default prefetch, measured on B200 (27-point 128^3 / 256^3): always for
    // 2-byte values (+5-33 %), never for 4-byte ones (-2 to -9 %), for 8-byte
    // ones when x exceeds L2
    const bool xBig = static_cast<int64_t>(std::max(P.n, P.numCols)) * static_cast<int64_t>(sizeof(XT)) > l2;
    const bool pfAuto = sizeof(VT) == 2 || (sizeof(VT) == 8 && xBig);
    const bool pf = P.prefetchL2 > 0 || (P.prefetchL2 < 0 && pfAuto);
    // default: 4 offsets in flight, the fastest or within run-to-run noise of
    // it for every value storage on B200 (27-point 128^3 / 256^3, banded 8M)
    const int32_t g = P.quadGroup ? P.quadGroup : 4;
    const int32_t quads = (P.numTiles + 3) / 4 * 4;  // tiles covered by whole quads (4 per warp)
#define HBDIA_QUAD(U)                                                                                  \
    return pf ? launch_pipe(dev::spmv_bw32_quad<VT, XT, U, true>, a, quads / 4, x, y, s, device)              \
              : launch_pipe(dev::spmv_bw32_quad<VT, XT, U, false>, a, quads / 4, x, y, s, device)
    switch (g) {
        case 1: HBDIA_QUAD(1);
        case 2: HBDIA_QUAD(2);
        case 8: HBDIA_QUAD(8);
        default: HBDIA_QUAD(4);
    }
#undef HBDIA_QUAD
}

template <typename VT, typename XT>
void launch_pipe_tuned(const DevicePlan &P, const dev::SpmvArgs<VT, XT> &a, const XT *x, XT *y, cudaStream_t s) {
    // Forcing 4-6 CTAs per SM through __launch_bounds__ made ptxas spill and
    // ran 3-45% slower on B200; the compiler's own register choice is kept.
    // The prefetch pays when x does not fit in L2 (measured on B200: +1.5 % FP64
    // and +8 % FP32 storage with a 134 MB x); with x resident in L2 the
    // prefetched value rows evict x lines that would have been reused (-2 to
    // -10 % at 57 MB and below).
    const int device = plan_device(P);
    bool pf = P.prefetchL2 > 0;
    if (P.prefetchL2 < 0) {
        int l2 = 0;
        check_cuda(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device), "cudaDeviceGetAttribute(L2)");
        pf = static_cast<int64_t>(std::max(P.n, P.numCols)) * static_cast<int64_t>(sizeof(XT)) > l2;
    }
    if (P.unroll != 27 && (P.maskedTail > 0 || (P.maskedTail < 0 && P.tailHeavy))) {
        if (pf) return launch_pipe(dev::spmv_bw32_pipe<VT, XT, kUnroll, true, true>, a, P.numTiles, x, y, s, device);
        return launch_pipe(dev::spmv_bw32_pipe<VT, XT, kUnroll, false, true>, a, P.numTiles, x, y, s, device);
    }
    if (pf) {
        if (P.unroll == 27) return launch_pipe(dev::spmv_bw32_pipe<VT, XT, 27, true>, a, P.numTiles, x, y, s, device);
        return launch_pipe(dev::spmv_bw32_pipe<VT, XT, kUnroll, true>, a, P.numTiles, x, y, s, device);
    }
    if (P.unroll == 27) return launch_pipe(dev::spmv_bw32_pipe<VT, XT, 27>, a, P.numTiles, x, y, s, device);
    return launch_pipe(dev::spmv_bw32_pipe<VT, XT, kUnroll>, a, P.numTiles, x, y, s, device);
}

template <typename VT, typename XT>
void launch_typed(const DevicePlan &P, const void *x, void *y, cudaStream_t s) {
    const dev::SpmvArgs<VT, XT> a = make_args<VT, XT>(P);
    const XT *xp = static_cast<const XT *>(x);
    XT *yp = static_cast<XT *>(y);
    const int32_t kern = select_kernel(P, x);
    if (kern == HBDIA_KERNEL_STAGED) {
        dev::XsArgs<VT, XT> A;
        A.a = a;
        A.status = P.status;
        A.timeoutNs = P.waitTimeoutNs;
        A.skipTile = P.skipTile;
        launch_xs<VT, XT>(A, P.xsConfig, xp, yp, s, plan_device(P));
    } else if (kern == HBDIA_KERNEL_PIPE) {
        launch_pipe_tuned<VT, XT>(P, a, xp, yp, s);
    } else if (kern == HBDIA_KERNEL_QUAD) {
        launch_quad<VT, XT>(P, a, xp, yp, s);

    } else if (kern == HBDIA_KERNEL_WARP) {
        const int64_t warpsPerCta = 8;
        const unsigned grid = static_cast<unsigned>((P.numTiles + warpsPerCta - 1) / warpsPerCta);
        dev::spmv_bw32<VT, XT, kUnroll><<<grid, 256, 0, s>>>(a, xp, yp);
    } else {
        const unsigned grid = static_cast<unsigned>((static_cast<int64_t>(P.n) + 255) / 256);
        dev::spmv_rowwise<VT, XT><<<grid, 256, 0, s>>>(a, xp, yp);
    }
    check_cuda(cudaGetLastError(), "SpMV launch");
}

}  // namespace

int32_t iteration_storage(const HostLayout<double> &L, int32_t storage) {
    const bool quad = storage == HBDIA_STORE_F32_QUAD || storage == HBDIA_STORE_BF16_QUAD;
    if (quad && (L.blockWidth != 32 || L.numRows > (1 << 30)))
        return storage == HBDIA_STORE_F32_QUAD ? HBDIA_STORE_F32 : HBDIA_STORE_BF16_SCALED;
    return storage;
}

int32_t select_kernel(const DevicePlan &P, const void *x) {
    if (P.quadLayout) return HBDIA_KERNEL_QUAD;  // the only kernel that reads that layout
    const bool bw32 = P.bw == 32;
    // the staged kernel bulk-copies x and the value slabs (16-byte aligned
    // starts), needs a status word for its bounded waits, and does row/column
    // arithmetic in 32 bits (n <= 2^30)
    const bool aligned = (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (reinterpret_cast<uintptr_t>(P.vals) & 15) == 0;
    // (x holds numCols >= the column bound entries: the runs never pass its end)
    const bool stagedOk = bw32 && aligned && P.status && P.numCols >= P.xn && P.n <= (1 << 30);
    const bool pipeOk = bw32 && P.n <= (1 << 30);  // 32-bit row/column arithmetic
    switch (P.kernel) {
        case HBDIA_KERNEL_ROWWISE: return HBDIA_KERNEL_ROWWISE;
        case HBDIA_KERNEL_STAGED:
            if (stagedOk) return HBDIA_KERNEL_STAGED;
            return bw32 ? HBDIA_KERNEL_WARP : HBDIA_KERNEL_ROWWISE;
        case HBDIA_KERNEL_PIPE:
            if (pipeOk) return HBDIA_KERNEL_PIPE;
            return bw32 ? HBDIA_KERNEL_WARP : HBDIA_KERNEL_ROWWISE;
        case HBDIA_KERNEL_QUAD:
            if (pipeOk) return HBDIA_KERNEL_QUAD;
            return bw32 ? HBDIA_KERNEL_WARP : HBDIA_KERNEL_ROWWISE;
        case HBDIA_KERNEL_WARP: return bw32 ? HBDIA_KERNEL_WARP : HBDIA_KERNEL_ROWWISE;
        default:  // AUTO: the fastest measured on B200 for blockWidth 32
            // (4- and 2-byte values: the quad kernel, 2-10 % ahead of the
            // pipelined one on the 27-point 128^3 and 256^3 workloads; FP64
            // values: the pipelined kernel, which the quad one trails there)
            if (pipeOk) return P.storage == HBDIA_STORE_NATIVE ? HBDIA_KERNEL_PIPE : HBDIA_KERNEL_QUAD;
            return bw32 ? HBDIA_KERNEL_WARP : HBDIA_KERNEL_ROWWISE;
    }
}

void launch_spmv(const DevicePlan &P, const void *x, void *y, void *stream) {
    if (!P.base) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
    if (!x || !y) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null vector pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : P.stream);
    if (P.dtype == HBDIA_F32) {
        launch_typed<float, float>(P, x, y, s);
    } else if (P.storage == HBDIA_STORE_F32) {
        launch_typed<float, double>(P, x, y, s);
    } else if (P.storage == HBDIA_STORE_BF16_SCALED) {
        launch_typed<__nv_bfloat16, double>(P, x, y, s);
    } else {
        launch_typed<double, double>(P, x, y, s);
    }
}

namespace {

template <typename VT, typename XT, int KT, bool CM>
void launch_spmm_kt(const DevicePlan &P, const dev::SpmvArgs<VT, XT> &a, const XT *X, int64_t ldx, XT *Y,
                    int64_t ldy, int32_t k, cudaStream_t s) {
    if (P.bw == 32) {
        const unsigned grid = static_cast<unsigned>((static_cast<int64_t>(P.numTiles) + 7) / 8);
        // The full passes in one launch, a partial last pass (k not a multiple
        // of KT) in a second one on the remaining columns; 32-bit gather
        // indices when every pass's block has fewer than 2^31 elements.
        const int64_t rowsX = std::max(P.n, P.numCols);
        const bool i32 = (CM ? int64_t(KT) * ldx + rowsX : rowsX * ldx + KT) < (int64_t(1) << 31);
        const int32_t kfull = k - k % KT, krest = k % KT;
        const XT *Xr = CM ? X + static_cast<int64_t>(kfull) * ldx : X + kfull;
        XT *Yr = CM ? Y + static_cast<int64_t>(kfull) * ldy : Y + kfull;
        if (i32) {
            if (kfull) dev::spmm_bw32<VT, XT, KT, CM, int32_t, true><<<grid, 256, 0, s>>>(a, X, ldx, Y, ldy, kfull);
            if (krest) dev::spmm_bw32<VT, XT, KT, CM, int32_t, false><<<grid, 256, 0, s>>>(a, Xr, ldx, Yr, ldy, krest);
        } else {
            if (kfull) dev::spmm_bw32<VT, XT, KT, CM, int64_t, true><<<grid, 256, 0, s>>>(a, X, ldx, Y, ldy, kfull);
            if (krest) dev::spmm_bw32<VT, XT, KT, CM, int64_t, false><<<grid, 256, 0, s>>>(a, Xr, ldx, Yr, ldy, krest);
        }
    } else {
        const unsigned grid = static_cast<unsigned>((static_cast<int64_t>(P.n) + 255) / 256);
        dev::spmm_rowwise<VT, XT, KT, CM><<<grid, 256, 0, s>>>(a, X, ldx, Y, ldy, k);
    }
}

template <typename VT, typename XT, bool CM>
void launch_spmm_layout(const DevicePlan &P, const dev::SpmvArgs<VT, XT> &a, const XT *xp, int64_t ldx, XT *yp,
                        int64_t ldy, int32_t k, int32_t tile, cudaStream_t s) {
    switch (tile) {
        case 2: launch_spmm_kt<VT, XT, 2, CM>(P, a, xp, ldx, yp, ldy, k, s); break;
        case 4: launch_spmm_kt<VT, XT, 4, CM>(P, a, xp, ldx, yp, ldy, k, s); break;
        case 8: launch_spmm_kt<VT, XT, 8, CM>(P, a, xp, ldx, yp, ldy, k, s); break;
        case 16: launch_spmm_kt<VT, XT, 16, CM>(P, a, xp, ldx, yp, ldy, k, s); break;
        default: launch_spmm_kt<VT, XT, 32, CM>(P, a, xp, ldx, yp, ldy, k, s); break;
    }
}

template <typename VT, typename XT>
void launch_spmm_typed(const DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                       int32_t tile, bool colMajor, cudaStream_t s) {
    dev::SpmvArgs<VT, XT> a = make_args<VT, XT>(P);
    const XT *xp = static_cast<const XT *>(X);
    XT *yp = static_cast<XT *>(Y);
    if (colMajor) launch_spmm_layout<VT, XT, true>(P, a, xp, ldx, yp, ldy, k, tile, s);
    else launch_spmm_layout<VT, XT, false>(P, a, xp, ldx, yp, ldy, k, tile, s);
    check_cuda(cudaGetLastError(), "SpMM launch");
}

}  // namespace

int32_t default_spmm_tile(int32_t k, bool colMajor) {
    // Measured on B200 (27-point stencil 256^3): column-major blocks are
    // fastest in passes of 4 for every k >= 3 (each column a separate
    // coalesced gather); row-major ones in the smallest tile covering k up to
    // 8 (wider passes re-fetch the same lines of X in every pass).
    if (k <= 2) return 2;
    if (colMajor || k <= 4) return 4;
    return 8;
}

void launch_spmm_tile(const DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                      int32_t tile, void *stream, bool colMajor) {
    if (!P.base) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
    if (P.quadLayout) throw Error(HBDIA_ERR_UNSUPPORTED, "quad-interleaved value storage supports SpMV only");
    if (!X || !Y) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null matrix pointer");
    if (k <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "need k > 0");
    if (!colMajor && (ldx < k || ldy < k)) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "need ldx, ldy >= k");
    if (colMajor && (ldx < std::max(P.n, P.numCols) || ldy < P.n))
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "column-major blocks need ldx >= max(numRows, numCols), ldy >= numRows");
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : P.stream);
    if (P.dtype == HBDIA_F32) launch_spmm_typed<float, float>(P, X, ldx, Y, ldy, k, tile, colMajor, s);
    else if (P.storage == HBDIA_STORE_F32) launch_spmm_typed<float, double>(P, X, ldx, Y, ldy, k, tile, colMajor, s);
    else if (P.storage == HBDIA_STORE_BF16_SCALED)
        launch_spmm_typed<__nv_bfloat16, double>(P, X, ldx, Y, ldy, k, tile, colMajor, s);
    else launch_spmm_typed<double, double>(P, X, ldx, Y, ldy, k, tile, colMajor, s);
}

namespace {

template <typename VT, typename XT, int KT>
void launch_list_kt(const DevicePlan &P, const dev::SpmvArgs<VT, XT> &a, const void *const *x, void *const *y,
                    int32_t k, cudaStream_t s) {
    // full passes in one launch, a partial last pass in a second
    const unsigned grid = static_cast<unsigned>((static_cast<int64_t>(P.numTiles) + 7) / 8);
    const int32_t kfull = k - k % KT, krest = k % KT;
    auto fill = [&](int32_t j0, int32_t cnt) {
        dev::VecList<XT> L{};
        for (int32_t j = 0; j < cnt; ++j) {
            L.x[j] = static_cast<const XT *>(x[j0 + j]);
            L.y[j] = static_cast<XT *>(y[j0 + j]);
        }
        return L;
    };
    if (kfull) dev::spmm_bw32_list<VT, XT, KT, true><<<grid, 256, 0, s>>>(a, fill(0, kfull), kfull);
    if (krest) dev::spmm_bw32_list<VT, XT, KT, false><<<grid, 256, 0, s>>>(a, fill(kfull, krest), krest);
}

template <typename VT, typename XT>
void launch_list_typed(const DevicePlan &P, const void *const *x, void *const *y, int32_t k, int32_t tile,
                       cudaStream_t s) {
    const dev::SpmvArgs<VT, XT> a = make_args<VT, XT>(P);
    switch (tile) {
        case 2: launch_list_kt<VT, XT, 2>(P, a, x, y, k, s); break;
        case 4: launch_list_kt<VT, XT, 4>(P, a, x, y, k, s); break;
        case 8: launch_list_kt<VT, XT, 8>(P, a, x, y, k, s); break;
        case 16: launch_list_kt<VT, XT, 16>(P, a, x, y, k, s); break;
        default: launch_list_kt<VT, XT, 32>(P, a, x, y, k, s); break;
    }
    check_cuda(cudaGetLastError(), "SpMV list launch");
}

}  // namespace

void launch_spmv_list(const DevicePlan &P, const void *const *x, void *const *y, int32_t k, void *stream) {
    if (!P.base) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
    if (P.quadLayout) throw Error(HBDIA_ERR_UNSUPPORTED, "quad-interleaved value storage supports SpMV only");
    if (k < 0 || (k > 0 && (!x || !y))) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad vector list");
    for (int32_t j = 0; j < k; ++j)
        if (!x[j] || !y[j]) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null vector in the list");
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : P.stream);
    if (P.bw != 32) {  // one SpMV per vector (column j of an SpMM is that SpMV)
        for (int32_t j = 0; j < k; ++j) launch_spmv(P, x[j], y[j], s);
        return;
    }
    for (int32_t j0 = 0; j0 < k; j0 += dev::kVecListMax) {
        const int32_t kk = std::min<int32_t>(dev::kVecListMax, k - j0);
        const int32_t tile = P.spmmTileForced ? P.spmmTileForced : default_spmm_tile(kk, true);
        if (P.dtype == HBDIA_F32) launch_list_typed<float, float>(P, x + j0, y + j0, kk, tile, s);
        else if (P.storage == HBDIA_STORE_F32) launch_list_typed<float, double>(P, x + j0, y + j0, kk, tile, s);
        else if (P.storage == HBDIA_STORE_BF16_SCALED)
            launch_list_typed<__nv_bfloat16, double>(P, x + j0, y + j0, kk, tile, s);
        else launch_list_typed<double, double>(P, x + j0, y + j0, kk, tile, s);
    }
}

void launch_spmm(const DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k, void *stream,
                 bool colMajor) {
    int32_t tile = P.spmmTileForced;
    if (!tile) {  // the autotuner's table is measured on row-major blocks
        auto it = colMajor ? P.spmmTile.end() : P.spmmTile.find(k);
        tile = it != P.spmmTile.end() ? it->second : default_spmm_tile(k, colMajor);
    }
    launch_spmm_tile(P, X, ldx, Y, ldy, k, tile, stream, colMajor);
}

}  // namespace hbdia
