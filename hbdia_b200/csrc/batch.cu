// Batches: many converted matrices computed as one unit of work.
//
// A batch fixes a list of device plans (same value type and storage, block
// width 32).  Binding gives every matrix its vectors (x/y, or k right-hand
// sides).  A run computes all of them, by one of two schedules:
//
//  * concurrent (default): every matrix's own single-matrix kernel (the one
//    hbdia_spmv_device / hbdia_spmm_device would launch, with the matrix's
//    kernel choice and tuning), issued on a ring of auxiliary streams forked
//    from and joined back into the run's stream.  On B200 the kernels of
//    different streams overlap, so there are no launch gaps and no per-matrix
//    tails, and every matrix keeps its kernel's full efficiency.
//  * queue: one persistent launch per segment of up to dev::kBatchSeg
//    matrices, warps taking tiles from an atomic counter
//    (batch_kernels.cuh): one launch for hundreds of matrices, for batches of
//    many tiny matrices where a launch per matrix would dominate.
//
// Either is replayed from a CUDA graph by default.  The concurrent graph is
// captured from the fork/join launches and re-captured (then updated in
// place) after a rebind; the queue graph is built by hand (a memset node,
// then one kernel node per segment) and gets new parameter blocks in place.
//
// Device memory of a batch: the queue schedule's work counters.
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
constexpr int kBatchUnroll = 9;     // offsets in flight per lane (the single-matrix default)
constexpr int kMaxAuxStreams = 64;  // concurrent schedule
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
    // binding (host copies, for the concurrent schedule)
    std::vector<const void *> X;
    std::vector<void *> Y;
    std::vector<int64_t> ldx, ldy;
    std::vector<int32_t> k;
    std::vector<int32_t> order;  // matrices by decreasing work (issue order)
    int64_t bytesPerRun = 0;
    bool bound = false;
    int32_t maxK = 0;
    // queue schedule
    std::vector<Seg> segs;
    std::vector<std::vector<unsigned char>> segBuf;  // parameter block of each segment
    int32_t *counters = nullptr;                     // one per segment
    int32_t sms = 0;
    // configuration
    int32_t schedule = HBDIA_BATCH_CONCURRENT;
    int32_t streams = 16;
    int32_t threads = 256, grab = 4, rhsTile = 8, useGraph = 1;
    // streams and events of the fork/join
    cudaStream_t own = nullptr;
    std::vector<cudaStream_t> aux;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    // graph of the current configuration and binding
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphNode_t> kernNodes;  // queue schedule
    int32_t execSchedule = -1, execStreams = 0, execThreads = 0, execGrab = 0, execTile = 0, execClass = -1;
    bool stale = false;  // binding changed since the graph was made
};

namespace {

void drop_graph(Batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->kernNodes.clear();
}

// ------------------------------------------------------------ binding
template <typename VT, typename XT>
void fill_segments(Batch *b) {
    using SegT = dev::BatchSeg<VT, XT>;
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
            e.k = b->k[i];
            e.X = static_cast<const XT *>(b->X[i]);
            e.Y = static_cast<XT *>(b->Y[i]);
            e.ldx = b->ldx[i];
            e.ldy = b->ldy[i];
        }
        S->next = b->counters + si;
        S->count = sg.count;
        S->totalTiles = sg.tiles;
        std::memcpy(b->segBuf[si].data(), S.get(), sizeof(SegT));
    }
}

size_t seg_bytes(int32_t dtype, int32_t storage) {
    if (dtype == HBDIA_F32) return sizeof(dev::BatchSeg<float, float>);
    if (storage == HBDIA_STORE_F32) return sizeof(dev::BatchSeg<float, double>);
    if (storage == HBDIA_STORE_BF16_SCALED) return sizeof(dev::BatchSeg<__nv_bfloat16, double>);
    return sizeof(dev::BatchSeg<double, double>);
}

// ------------------------------------------------------------ queue schedule
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

void queue_direct(Batch *b, cudaStream_t s) {
    const LaunchSpec L = spec(b);
    check_cuda(cudaMemsetAsync(b->counters, 0, sizeof(int32_t) * b->segs.size(), s), "cudaMemsetAsync(batch)");
    for (size_t si = 0; si < b->segs.size(); ++si) {
        void *args[1] = {b->segBuf[si].data()};
        check_cuda(cudaLaunchKernel(L.func, dim3(L.grid[si]), dim3(static_cast<unsigned>(b->threads)), args, 0, s),
                   "batch kernel launch");
    }
}

void queue_graph(Batch *b) {
    const LaunchSpec L = spec(b);
    check_cuda(cudaGraphCreate(&b->graph, 0), "cudaGraphCreate(batch)");
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
}

void queue_refresh(Batch *b) {
    const LaunchSpec L = spec(b);
    for (size_t si = 0; si < b->segs.size(); ++si) {
        void *slot = nullptr;
        const cudaKernelNodeParams p = node_params(b, L, si, &slot);
        check_cuda(cudaGraphExecKernelNodeSetParams(b->exec, b->kernNodes[si], &p),
                   "cudaGraphExecKernelNodeSetParams(batch)");
    }
}

// ------------------------------------------------------------ concurrent schedule
void ensure_aux(Batch *b) {
    while (static_cast<int32_t>(b->aux.size()) < b->streams) {
        cudaStream_t st = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate(batch aux)");
        b->aux.push_back(st);
        cudaEvent_t ev = nullptr;
        check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate(batch join)");
        b->join.push_back(ev);
    }
}

// Fork from s, one launch per bound matrix on the stream ring (largest
// first), join back into s.
void concurrent_issue(Batch *b, cudaStream_t s) {
    ensure_aux(b);
    const int32_t ns = b->streams;
    check_cuda(cudaEventRecord(b->fork, s), "cudaEventRecord(batch fork)");
    for (int32_t j = 0; j < ns; ++j) check_cuda(cudaStreamWaitEvent(b->aux[j], b->fork, 0), "cudaStreamWaitEvent");
    int32_t slot = 0;
    for (int32_t i : b->order) {
        const int32_t ki = b->k[i];
        if (ki == 0) continue;
        cudaStream_t st = b->aux[slot++ % ns];
        if (ki == 1) launch_spmv(*b->plans[i], b->X[i], b->Y[i], st);
        else launch_spmm(*b->plans[i], b->X[i], b->ldx[i], b->Y[i], b->ldy[i], ki, st);
    }
    for (int32_t j = 0; j < ns; ++j) {
        check_cuda(cudaEventRecord(b->join[j], b->aux[j]), "cudaEventRecord(batch join)");
        check_cuda(cudaStreamWaitEvent(s, b->join[j], 0), "cudaStreamWaitEvent");
    }
}

cudaGraph_t concurrent_capture(Batch *b) {
    cudaGraph_t g = nullptr;
    check_cuda(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture(batch)");
    try {
        concurrent_issue(b, b->own);
    } catch (...) {
        cudaStreamEndCapture(b->own, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(b->own, &g), "cudaStreamEndCapture(batch)");
    return g;
}

// ------------------------------------------------------------ common
int32_t kernel_class(const Batch *b) { return b->maxK <= 1 ? 1 : 2; }

bool graph_matches(const Batch *b) {
    if (!b->exec || b->execSchedule != b->schedule) return false;
    if (b->schedule == HBDIA_BATCH_CONCURRENT) return b->execStreams == b->streams;
    return b->execThreads == b->threads && b->execGrab == b->grab && b->execTile == b->rhsTile &&
           b->execClass == kernel_class(b);
}

void make_graph(Batch *b) {
    drop_graph(b);
    try {
        if (b->schedule == HBDIA_BATCH_CONCURRENT) {
            b->graph = concurrent_capture(b);
            check_cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate(batch)");
        } else {
            queue_graph(b);
        }
    } catch (...) {
        drop_graph(b);
        throw;
    }
    b->execSchedule = b->schedule;
    b->execStreams = b->streams;
    b->execThreads = b->threads;
    b->execGrab = b->grab;
    b->execTile = b->rhsTile;
    b->execClass = kernel_class(b);
    b->stale = false;
}

// New binding into the existing graph: parameter blocks in place (queue), or
// a fresh capture applied with cudaGraphExecUpdate (concurrent; rebuilt when
// the update is refused, e.g. after k changes the kernels).
void refresh_graph(Batch *b) {
    if (b->schedule == HBDIA_BATCH_QUEUE) {
        queue_refresh(b);
        b->stale = false;
        return;
    }
    cudaGraph_t g = concurrent_capture(b);
    cudaGraphExecUpdateResultInfo info;
    const cudaError_t rc = cudaGraphExecUpdate(b->exec, g, &info);
    if (rc == cudaSuccess) {
        if (b->graph) cudaGraphDestroy(b->graph);
        b->graph = g;
        b->stale = false;
        return;
    }
    (void)cudaGetLastError();
    cudaGraphDestroy(g);
    make_graph(b);
}

void run_direct(Batch *b, cudaStream_t s) {
    if (b->schedule == HBDIA_BATCH_QUEUE) queue_direct(b, s);
    else concurrent_issue(b, s);
}

cudaStream_t pick(const Batch *b, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : b->own;
}

void check_config(int32_t schedule, int32_t streams, int32_t threads, int32_t grab, int32_t tile) {
    if (schedule != HBDIA_BATCH_CONCURRENT && schedule != HBDIA_BATCH_QUEUE)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown batch schedule");
    if (streams < 1 || streams > kMaxAuxStreams)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "streams must be in [1, 64]");
    if (threads != 128 && threads != 256 && threads != 512)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "threads per block must be 128, 256 or 512");
    if (grab < 1 || grab > 64) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "tiles per grab must be in [1, 64]");
    if (tile != 4 && tile != 8 && tile != 16)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "right-hand-side tile must be 4, 8 or 16");
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
        if (P.quadLayout)
            throw Error(HBDIA_ERR_UNSUPPORTED, "quad-interleaved value storage supports SpMV only (matrix " +
                                                   std::to_string(i) + ")");
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
        b->segBuf.assign(segs.size(), std::vector<unsigned char>(seg_bytes(b->dtype, b->storage), 0));
        b->order.resize(plans.size());
        for (size_t i = 0; i < plans.size(); ++i) b->order[i] = static_cast<int32_t>(i);
        std::stable_sort(b->order.begin(), b->order.end(),
                         [&](int32_t a, int32_t c) { return plans[a]->numTiles > plans[c]->numTiles; });
        check_cuda(dev_alloc(reinterpret_cast<void **>(&b->counters), sizeof(int32_t) * segs.size()),
                   "cudaMalloc(batch counters)");
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        check_cuda(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "cudaStreamCreate(batch)");
        check_cuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate(batch fork)");
        b->streams = std::min<int32_t>(16, b->count);
    } catch (...) {
        batch_free(b);
        throw;
    }
    return b;
}

void batch_free(Batch *b) {
    if (!b) return;
    drop_graph(b);
    if (b->own) cudaStreamSynchronize(b->own);
    for (cudaStream_t st : b->aux) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own) cudaStreamDestroy(b->own);
    if (b->counters) cudaFree(b->counters);
    delete b;
}

void batch_bind(Batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                const int32_t *k) {
    // Launches already enqueued carry copies of their arguments, so the new
    // binding needs no synchronisation.  Everything is validated before
    // anything changes.
    const size_t n = static_cast<size_t>(b->count);
    std::vector<const void *> nX(n, nullptr);
    std::vector<void *> nY(n, nullptr);
    std::vector<int64_t> nldx(n, 1), nldy(n, 1);
    std::vector<int32_t> nk(n, 1);
    int64_t bytes = 0;
    int32_t maxK = 0;
    for (int32_t i = 0; i < b->count; ++i) {
        const DevicePlan &P = *b->plans[i];
        const int32_t ki = k ? k[i] : 1;
        if (ki < 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "negative right-hand-side count");
        nk[i] = ki;
        if (ki > 0) {
            if (!X || !Y || !X[i] || !Y[i])
                throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null vector for matrix " + std::to_string(i));
            nX[i] = X[i];
            nY[i] = Y[i];
            nldx[i] = ki > 1 ? (ldx ? ldx[i] : ki) : 1;
            nldy[i] = ki > 1 ? (ldy ? ldy[i] : ki) : 1;
            if (ki > 1 && (nldx[i] < ki || nldy[i] < ki))
                throw Error(HBDIA_ERR_INVALID_ARGUMENT, "leading dimension smaller than k for matrix " +
                                                            std::to_string(i));
            if (ki == 1 && ((ldx && ldx[i] != 1) || (ldy && ldy[i] != 1)))
                throw Error(HBDIA_ERR_INVALID_ARGUMENT,
                            "k == 1 takes contiguous vectors (leading dimension 1) for matrix " + std::to_string(i));
            const int64_t xs = P.dtype == HBDIA_F32 ? 4 : 8;
            bytes += P.bytesPerSpmv + static_cast<int64_t>(ki - 1) * (2 * xs * P.n + xs * P.nCoo);
        }
        maxK = std::max(maxK, ki);
    }
    b->X.swap(nX);
    b->Y.swap(nY);
    b->ldx.swap(nldx);
    b->ldy.swap(nldy);
    b->k.swap(nk);
    b->bytesPerRun = bytes;
    b->maxK = maxK;
    if (b->dtype == HBDIA_F32) fill_segments<float, float>(b);
    else if (b->storage == HBDIA_STORE_F32) fill_segments<float, double>(b);
    else if (b->storage == HBDIA_STORE_BF16_SCALED) fill_segments<__nv_bfloat16, double>(b);
    else fill_segments<double, double>(b);
    b->bound = true;
    b->stale = true;
}

void batch_run(Batch *b, void *stream) {
    if (!b->bound) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "batch has no bound vectors");
    const cudaStream_t s = pick(b, stream);
    if (!b->useGraph) {
        run_direct(b, s);
        return;
    }
    if (!graph_matches(b)) make_graph(b);
    else if (b->stale) refresh_graph(b);
    check_cuda(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch(batch)");
}

void batch_set_config(Batch *b, const hbdia_batch_config &c) {
    check_config(c.schedule, c.streams, c.threadsPerBlock, c.tilesPerGrab, c.rhsTile);
    b->schedule = c.schedule;
    b->streams = c.streams;
    b->threads = c.threadsPerBlock;
    b->grab = c.tilesPerGrab;
    b->rhsTile = c.rhsTile;
    b->useGraph = c.useGraph ? 1 : 0;
}

void batch_get_config(const Batch *b, hbdia_batch_config &c) {
    c.schedule = b->schedule;
    c.streams = b->streams;
    c.threadsPerBlock = b->threads;
    c.tilesPerGrab = b->grab;
    c.rhsTile = b->rhsTile;
    c.useGraph = b->useGraph;
}

void batch_autotune(Batch *b, void *stream, float *msOut, int32_t *candidates) {
    if (!b->bound) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bind the batch's vectors before tuning it");
    const cudaStream_t s = pick(b, stream);
    struct Cand {
        int32_t schedule, streams, threads, grab, tile;
    };
    const int32_t keepStreams = b->streams, keepThreads = b->threads, keepGrab = b->grab, keepTile = b->rhsTile,
                  keepSched = b->schedule;
    std::vector<Cand> cands;
    for (int32_t ns : {4, 16, 64}) cands.push_back({HBDIA_BATCH_CONCURRENT, ns, keepThreads, keepGrab, keepTile});
    std::vector<int32_t> tiles = {8};
    if (b->maxK > 1) tiles = {4, 8, 16};
    for (int32_t th : {128, 256, 512})
        for (int32_t gr : {1, 2, 4, 8, 16})
            for (int32_t kt : tiles) cands.push_back({HBDIA_BATCH_QUEUE, keepStreams, th, gr, kt});
    auto apply = [&](const Cand &c) {
        b->schedule = c.schedule;
        b->streams = c.streams;
        b->threads = c.threads;
        b->grab = c.grab;
        b->rhsTile = c.tile;
    };
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 0.0f;
    size_t bi = 0;
    try {
        for (size_t ci = 0; ci < cands.size(); ++ci) {
            apply(cands[ci]);
            for (int w = 0; w < 2; ++w) run_direct(b, s);
            constexpr int kReps = 5;
            check_cuda(cudaEventRecord(e0, s), "cudaEventRecord");
            for (int r = 0; r < kReps; ++r) run_direct(b, s);
            check_cuda(cudaEventRecord(e1, s), "cudaEventRecord");
            check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            ms /= kReps;
            if (ci == 0 || ms < best) {
                best = ms;
                bi = ci;
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        apply({keepSched, keepStreams, keepThreads, keepGrab, keepTile});
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(cands[bi]);
    if (msOut) *msOut = best;
    if (candidates) *candidates = static_cast<int32_t>(cands.size());
}

void batch_info(const Batch *b, int32_t *count, int32_t *totalTiles, int64_t *bytesPerRun) {
    *count = b->count;
    *totalTiles = static_cast<int32_t>(std::min<int64_t>(b->totalTiles, INT32_MAX));
    *bytesPerRun = b->bytesPerRun;
}

void *batch_stream(const Batch *b) { return b->own; }

}  // namespace hbdia
