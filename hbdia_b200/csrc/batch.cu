// Batches: many converted matrices computed by one persistent launch.
//
// A batch fixes a list of device plans (same value type and storage, block
// width 32), cut into segments of up to dev::kBatchSeg matrices.  Binding
// gives every matrix its vectors (x/y, or k right-hand sides) and writes each
// segment's parameter block on the host (the kernel reads its entry table
// from the parameter block, no device table).  A run zeroes the segments'
// work counters and launches spmv_bw32_batch once per segment -- by default
// by replaying a CUDA graph (one memset node, then one kernel node per
// segment, the segments free to overlap), built once per configuration and
// given new parameter blocks in place when the binding changes.
//
// Device memory of a batch: the segments' work counters (int32 each).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "args.cuh"
#include "batch_kernels.cuh"
#include "hbdia_internal.hpp"

namespace hbdia {

namespace {
constexpr int kBatchUnroll = 9;  // offsets in flight per lane (the single-matrix default)
static_assert(sizeof(dev::BatchSeg<double, double>) <= 32000, "batch segment exceeds the kernel parameter limit");
static_assert(sizeof(dev::BatchSeg<float, float>) <= 32000, "batch segment exceeds the kernel parameter limit");

struct Seg {
    int32_t first = 0, count = 0, tiles = 0;
};
}  // namespace

struct Batch {
    std::vector<const DevicePlan *> plans;
    int32_t dtype = HBDIA_F64, storage = HBDIA_STORE_NATIVE;
    int32_t count = 0;
    int64_t totalTiles = 0;
    std::vector<Seg> segs;
    size_t segBytes = 0;
    std::vector<std::vector<unsigned char>> segBuf;  // parameter block of each segment
    int32_t *counters = nullptr;                     // one per segment
    int64_t bytesPerRun = 0;
    bool bound = false;
    int32_t maxK = 0;
    int32_t sms = 0;
    // configuration
    int32_t threads = 256, grab = 4, rhsTile = 8, useGraph = 1;
    // graph of the current configuration
    cudaStream_t own = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphNode_t> kernNodes;
    int32_t execThreads = 0, execGrab = 0, execTile = 0, execClass = -1;
    bool paramsStale = false;
};

namespace {

void drop_graph(Batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->kernNodes.clear();
}

template <typename VT, typename XT>
void fill_entries(Batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                  const int32_t *k) {
    using SegT = dev::BatchSeg<VT, XT>;
    std::vector<std::unique_ptr<SegT>> tmp;
    int64_t bytes = 0;
    int32_t maxK = 0;
    for (size_t si = 0; si < b->segs.size(); ++si) {
        const Seg &sg = b->segs[si];
        auto S = std::make_unique<SegT>();
        std::memset(S.get(), 0, sizeof(SegT));
        int32_t tb = 0;
        for (int32_t j = 0; j < sg.count; ++j) {
            const int32_t i = sg.first + j;
            const DevicePlan &P = *b->plans[i];
            dev::BatchEntry<VT, XT> &e = S->e[j];
            e.a = make_args<VT, XT>(P);
            e.tileBase = tb;
            tb += P.numTiles;
            const int32_t ki = k ? k[i] : 1;
            if (ki < 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "negative right-hand-side count");
            e.k = ki;
            if (ki > 0) {
                if (!X || !Y || !X[i] || !Y[i])
                    throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null vector for matrix " + std::to_string(i));
                e.X = static_cast<const XT *>(X[i]);
                e.Y = static_cast<XT *>(Y[i]);
                e.ldx = ki > 1 ? (ldx ? ldx[i] : ki) : 1;
                e.ldy = ki > 1 ? (ldy ? ldy[i] : ki) : 1;
                if (ki > 1 && (e.ldx < ki || e.ldy < ki))
                    throw Error(HBDIA_ERR_INVALID_ARGUMENT, "leading dimension smaller than k for matrix " +
                                                                std::to_string(i));
                if (ki == 1 && ((ldx && ldx[i] != 1) || (ldy && ldy[i] != 1)))
                    throw Error(HBDIA_ERR_INVALID_ARGUMENT,
                                "k == 1 takes contiguous vectors (leading dimension 1) for matrix " +
                                    std::to_string(i));
                const int64_t xs = static_cast<int64_t>(sizeof(XT));
                bytes += P.bytesPerSpmv + static_cast<int64_t>(ki - 1) * (2 * xs * P.n + xs * P.nCoo);
            }
            maxK = std::max(maxK, ki);
        }
        S->next = b->counters + si;
        S->count = sg.count;
        S->totalTiles = sg.tiles;
        tmp.push_back(std::move(S));
    }
    // every entry is valid: commit the new parameter blocks
    for (size_t si = 0; si < tmp.size(); ++si)
        std::memcpy(b->segBuf[si].data(), tmp[si].get(), sizeof(SegT));
    b->bytesPerRun = bytes;
    b->maxK = maxK;
}

// Kernel of the current configuration, its grid per segment, and the
// parameter blocks with the current tiles-per-grab.
struct LaunchSpec {
    const void *func = nullptr;
    std::vector<unsigned> grid;
};

template <typename VT, typename XT, int KT>
LaunchSpec spec_kt(Batch *b) {
    auto kern = dev::spmv_bw32_batch<VT, XT, kBatchUnroll, KT>;
    int perSm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, b->threads, 0),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor(batch)");
    LaunchSpec L;
    L.func = reinterpret_cast<const void *>(kern);
    const int64_t warpsPerCta = b->threads / 32;
    const int64_t resident = static_cast<int64_t>(std::max(perSm, 1)) * b->sms;
    for (const Seg &sg : b->segs) {
        const int64_t need = (static_cast<int64_t>(sg.tiles) + warpsPerCta - 1) / warpsPerCta;
        L.grid.push_back(static_cast<unsigned>(std::max<int64_t>(1, std::min(resident, need))));
    }
    for (auto &buf : b->segBuf) reinterpret_cast<dev::BatchSeg<VT, XT> *>(buf.data())->grab = b->grab;
    return L;
}

template <typename VT, typename XT>
LaunchSpec spec_typed(Batch *b) {
    if (b->maxK <= 1) return spec_kt<VT, XT, 0>(b);
    switch (b->rhsTile) {
        case 4: return spec_kt<VT, XT, 4>(b);
        case 16: return spec_kt<VT, XT, 16>(b);
        default: return spec_kt<VT, XT, 8>(b);
    }
}

LaunchSpec spec(Batch *b) {
    if (b->dtype == HBDIA_F32) return spec_typed<float, float>(b);
    if (b->storage == HBDIA_STORE_F32) return spec_typed<float, double>(b);
    if (b->storage == HBDIA_STORE_BF16_SCALED) return spec_typed<__nv_bfloat16, double>(b);
    return spec_typed<double, double>(b);
}

cudaKernelNodeParams node_params(Batch *b, const LaunchSpec &L, size_t si, void **argSlot) {
    cudaKernelNodeParams p;
    std::memset(&p, 0, sizeof(p));
    p.func = const_cast<void *>(L.func);
    p.gridDim = dim3(L.grid[si]);
    p.blockDim = dim3(static_cast<unsigned>(b->threads));
    p.sharedMemBytes = 0;
    *argSlot = b->segBuf[si].data();
    p.kernelParams = argSlot;
    p.extra = nullptr;
    return p;
}

void launch_direct(Batch *b, cudaStream_t s) {
    const LaunchSpec L = spec(b);
    check_cuda(cudaMemsetAsync(b->counters, 0, sizeof(int32_t) * b->segs.size(), s), "cudaMemsetAsync(batch)");
    for (size_t si = 0; si < b->segs.size(); ++si) {
        void *args[1] = {b->segBuf[si].data()};
        check_cuda(cudaLaunchKernel(L.func, dim3(L.grid[si]), dim3(static_cast<unsigned>(b->threads)), args, 0, s),
                   "batch kernel launch");
    }
}

void build_graph(Batch *b) {
    drop_graph(b);
    const LaunchSpec L = spec(b);
    check_cuda(cudaGraphCreate(&b->graph, 0), "cudaGraphCreate(batch)");
    try {
        cudaMemsetParams mp;
        std::memset(&mp, 0, sizeof(mp));
        mp.dst = b->counters;
        mp.value = 0;
        mp.elementSize = sizeof(int32_t);
        mp.width = b->segs.size();
        mp.height = 1;
        cudaGraphNode_t mnode = nullptr;
        check_cuda(cudaGraphAddMemsetNode(&mnode, b->graph, nullptr, 0, &mp), "cudaGraphAddMemsetNode(batch)");
        for (size_t si = 0; si < b->segs.size(); ++si) {
            void *slot = nullptr;
            const cudaKernelNodeParams p = node_params(b, L, si, &slot);
            cudaGraphNode_t kn = nullptr;
            check_cuda(cudaGraphAddKernelNode(&kn, b->graph, &mnode, 1, &p), "cudaGraphAddKernelNode(batch)");
            b->kernNodes.push_back(kn);
        }
        check_cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate(batch)");
    } catch (...) {
        drop_graph(b);
        throw;
    }
    b->execThreads = b->threads;
    b->execGrab = b->grab;
    b->execTile = b->rhsTile;
    b->execClass = b->maxK <= 1 ? 1 : 2;
    b->paramsStale = false;
}

void refresh_graph_params(Batch *b) {
    const LaunchSpec L = spec(b);
    for (size_t si = 0; si < b->segs.size(); ++si) {
        void *slot = nullptr;
        const cudaKernelNodeParams p = node_params(b, L, si, &slot);
        check_cuda(cudaGraphExecKernelNodeSetParams(b->exec, b->kernNodes[si], &p),
                   "cudaGraphExecKernelNodeSetParams(batch)");
    }
    b->paramsStale = false;
}

cudaStream_t pick(const Batch *b, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : b->own;
}

void check_config(int32_t threads, int32_t grab, int32_t tile) {
    if (threads != 128 && threads != 256 && threads != 512)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "threads per block must be 128, 256 or 512");
    if (grab < 1 || grab > 64) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "tiles per grab must be in [1, 64]");
    if (tile != 4 && tile != 8 && tile != 16)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "right-hand-side tile must be 4, 8 or 16");
}

size_t seg_bytes(int32_t dtype, int32_t storage) {
    if (dtype == HBDIA_F32) return sizeof(dev::BatchSeg<float, float>);
    if (storage == HBDIA_STORE_F32) return sizeof(dev::BatchSeg<float, double>);
    if (storage == HBDIA_STORE_BF16_SCALED) return sizeof(dev::BatchSeg<__nv_bfloat16, double>);
    return sizeof(dev::BatchSeg<double, double>);
}

}  // namespace

Batch *batch_create(const std::vector<const DevicePlan *> &plans) {
    if (plans.empty()) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "empty batch");
    if (plans.size() > (1u << 24)) throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^24 matrices in a batch");
    const DevicePlan &P0 = *plans[0];
    std::vector<Seg> segs;
    int64_t total = 0;
    for (size_t i = 0; i < plans.size(); ++i) {
        const DevicePlan &P = *plans[i];
        if (!P.base) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix " + std::to_string(i) + " has no device layout");
        if (P.bw != 32)
            throw Error(HBDIA_ERR_UNSUPPORTED, "batches need blockWidth 32 (matrix " + std::to_string(i) + ")");
        if (P.dtype != P0.dtype || P.storage != P0.storage)
            throw Error(HBDIA_ERR_INVALID_ARGUMENT, "all matrices of a batch need the same value type and storage");
        if (segs.empty() || segs.back().count == dev::kBatchSeg ||
            static_cast<int64_t>(segs.back().tiles) + P.numTiles > (int64_t(1) << 30)) {
            Seg s;
            s.first = static_cast<int32_t>(i);
            segs.push_back(s);
        }
        segs.back().count += 1;
        segs.back().tiles += P.numTiles;
        total += P.numTiles;
    }
    auto b = new Batch;
    try {
        b->plans = plans;
        b->dtype = P0.dtype;
        b->storage = P0.storage;
        b->count = static_cast<int32_t>(plans.size());
        b->totalTiles = total;
        b->segs = segs;
        b->segBytes = seg_bytes(b->dtype, b->storage);
        b->segBuf.assign(segs.size(), std::vector<unsigned char>(b->segBytes, 0));
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&b->counters), sizeof(int32_t) * segs.size()),
                   "cudaMalloc(batch counters)");
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        check_cuda(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "cudaStreamCreate(batch)");
    } catch (...) {
        batch_free(b);
        throw;
    }
    return b;
}

void batch_free(Batch *b) {
    if (!b) return;
    drop_graph(b);
    if (b->own) {
        cudaStreamSynchronize(b->own);
        cudaStreamDestroy(b->own);
    }
    if (b->counters) cudaFree(b->counters);
    delete b;
}

void batch_bind(Batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                const int32_t *k) {
    // Launches already enqueued carry copies of the old parameter blocks, so
    // the new binding needs no synchronisation.
    if (b->dtype == HBDIA_F32) fill_entries<float, float>(b, X, ldx, Y, ldy, k);
    else if (b->storage == HBDIA_STORE_F32) fill_entries<float, double>(b, X, ldx, Y, ldy, k);
    else if (b->storage == HBDIA_STORE_BF16_SCALED) fill_entries<__nv_bfloat16, double>(b, X, ldx, Y, ldy, k);
    else fill_entries<double, double>(b, X, ldx, Y, ldy, k);
    b->bound = true;
    b->paramsStale = true;
}

void batch_run(Batch *b, void *stream) {
    if (!b->bound) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "batch has no bound vectors");
    const cudaStream_t s = pick(b, stream);
    if (!b->useGraph) {
        launch_direct(b, s);
        return;
    }
    const int32_t cls = b->maxK <= 1 ? 1 : 2;  // which kernel instance the graph holds
    if (!b->exec || b->execThreads != b->threads || b->execGrab != b->grab || b->execTile != b->rhsTile ||
        b->execClass != cls)
        build_graph(b);
    else if (b->paramsStale)
        refresh_graph_params(b);
    check_cuda(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch(batch)");
}

void batch_set_config(Batch *b, int32_t threads, int32_t grab, int32_t rhsTile, int32_t useGraph) {
    check_config(threads, grab, rhsTile);
    b->threads = threads;
    b->grab = grab;
    b->rhsTile = rhsTile;
    b->useGraph = useGraph ? 1 : 0;
}

void batch_get_config(const Batch *b, int32_t *threads, int32_t *grab, int32_t *rhsTile, int32_t *useGraph) {
    *threads = b->threads;
    *grab = b->grab;
    *rhsTile = b->rhsTile;
    *useGraph = b->useGraph;
}

void batch_autotune(Batch *b, void *stream, float *msOut, int32_t *candidates) {
    if (!b->bound) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bind the batch's vectors before tuning it");
    const cudaStream_t s = pick(b, stream);
    std::vector<int32_t> tiles = {8};
    if (b->maxK > 1) tiles = {4, 8, 16};
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 0.0f;
    int32_t bt = b->threads, bg = b->grab, bk = b->rhsTile, n = 0;
    try {
        for (int32_t th : {128, 256, 512})
            for (int32_t gr : {1, 2, 4, 8, 16})
                for (int32_t kt : tiles) {
                    b->threads = th;
                    b->grab = gr;
                    b->rhsTile = kt;
                    for (int w = 0; w < 2; ++w) launch_direct(b, s);
                    constexpr int kReps = 5;
                    check_cuda(cudaEventRecord(e0, s), "cudaEventRecord");
                    for (int r = 0; r < kReps; ++r) launch_direct(b, s);
                    check_cuda(cudaEventRecord(e1, s), "cudaEventRecord");
                    check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
                    float ms = 0.0f;
                    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                    ms /= kReps;
                    ++n;
                    if (n == 1 || ms < best) {
                        best = ms;
                        bt = th;
                        bg = gr;
                        bk = kt;
                    }
                }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->threads = bt;
        b->grab = bg;
        b->rhsTile = bk;
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->threads = bt;
    b->grab = bg;
    b->rhsTile = bk;
    if (msOut) *msOut = best;
    if (candidates) *candidates = n;
}

void batch_info(const Batch *b, int32_t *count, int32_t *totalTiles, int64_t *bytesPerRun) {
    *count = b->count;
    *totalTiles = static_cast<int32_t>(std::min<int64_t>(b->totalTiles, INT32_MAX));
    *bytesPerRun = b->bytesPerRun;
}

void *batch_stream(const Batch *b) { return b->own; }

}  // namespace hbdia
