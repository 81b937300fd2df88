// Conjugate-gradient solver on the HBDIA SpMV (SPD matrices), with the
// iterations on a reduced-storage copy of the matrix and reliable updates in
// FP64.
//
//   every iteration:  q = A_it p    (A_it: FP32 or BF16-with-scale values,
//                                     FP64 accumulation; or the FP64 values)
//                     alpha = r.r / p.q;  x += alpha p;  r -= alpha q
//                     beta = r.r_new / r.r;  p = r + beta p
//   reliable update:  r = b - A x   with the FP64 values, when the iterated
//                     residual has fallen below updateFactor times the
//                     largest iterated residual since the last update, and
//                     before the solve is declared converged
//   stop:             ||b - A x|| / ||b|| <= tol  (always an FP64 residual)
//
// x, r, p, q, the dot products, norms and scalars are FP64; only the matrix
// values of the iterated operator are narrower.  Unlike restarted iterative
// refinement (an inner CG from scratch on each correction), a reliable
// update keeps the search direction, so the Krylov space built so far is not
// thrown away: the iteration count stays close to FP64 CG's while every
// iteration reads the narrower values (the method of Sleijpen and van der
// Vorst, "Reliable updated residuals in hybrid Bi-CG methods", 1996, as used
// by mixed-precision Krylov solvers on GPUs).
//
// Reductions are deterministic: every block reduces a fixed slice in a fixed
// order and every consumer of the partial sums adds them in the same order,
// so a solve is bit-reproducible run to run.  Scalars (alpha, beta, r.r) live
// in device memory; the iterations are captured once per solve in a CUDA
// graph of `checkEvery` iterations that is replayed, so the host
// synchronises once per `checkEvery` iterations.
//
// L2 residency (option): the solver's vectors r, p, q live in one range that
// is marked persisting in L2 (a stream access-policy window) while the solve
// runs, so the value stream of the SpMV does not evict them; each iteration
// then draws mostly the matrix values from HBM.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>

#include "hbdia_internal.hpp"

namespace hbdia {
namespace {

constexpr int kThreads = 256;

// sum of a block's values in a fixed order (warp shuffles, then warp 0)
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) ws[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = l < kThreads / 32 ? ws[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    return s;  // valid in thread 0
}

// total of the partial sums, same order for every reader
__device__ __forceinline__ double sum_partials(const double *__restrict__ part, int nparts) {
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += kThreads) v += part[i];
    __shared__ double tot;
    const double s = block_sum(v);
    if (threadIdx.x == 0) tot = s;
    __syncthreads();
    return tot;
}

// partial sums of a . b
__global__ void __launch_bounds__(kThreads) dot_partial(const double *__restrict__ a, const double *__restrict__ b,
                                                        int64_t n, double *__restrict__ part) {
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        v = fma(a[i], b[i], v);
    const double s = block_sum(v);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// r = b - q; partial sums of r . r
__global__ void __launch_bounds__(kThreads) residual(const double *__restrict__ b, const double *__restrict__ q,
                                                     double *__restrict__ r, int64_t n, double *__restrict__ part) {
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads) {
        const double ri = b[i] - q[i];
        r[i] = ri;
        v = fma(ri, ri, v);
    }
    const double s = block_sum(v);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// scal[0] = r.r (from partials); with `start`, also p = r (first direction)
__global__ void __launch_bounds__(kThreads) cg_start(const double *__restrict__ r, double *__restrict__ p, int64_t n,
                                                     const double *__restrict__ part, int nparts,
                                                     double *__restrict__ scal, int start) {
    const double rr = sum_partials(part, nparts);
    if (blockIdx.x == 0 && threadIdx.x == 0) scal[0] = rr;
    if (!start) return;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        p[i] = r[i];
}

// alpha = r.r / p.q;  x += alpha p;  r -= alpha q;  partial sums of new r.r
__global__ void __launch_bounds__(kThreads) cg_update(double *__restrict__ x, double *__restrict__ r,
                                                      const double *__restrict__ p, const double *__restrict__ q,
                                                      int64_t n, const double *__restrict__ pqPart, int nparts,
                                                      const double *__restrict__ scal, double *__restrict__ rrPart) {
    const double pq = sum_partials(pqPart, nparts);
    const double alpha = pq != 0.0 ? scal[0] / pq : 0.0;
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        v = fma(ri, ri, v);
    }
    const double s = block_sum(v);
    if (threadIdx.x == 0) rrPart[blockIdx.x] = s;
}

// beta = r.r_new / r.r;  p = r + beta p.  Every block reads r.r from scalIn;
// block 0 writes r.r_new to the separate slot scalOut, which copy_scalar moves
// into scalIn before the next iteration, so no block sees a half-updated value.
__global__ void __launch_bounds__(kThreads) cg_direction(const double *__restrict__ r, double *__restrict__ p,
                                                         int64_t n, const double *__restrict__ rrPart, int nparts,
                                                         const double *__restrict__ scalIn,
                                                         double *__restrict__ scalOut) {
    const double rrNew = sum_partials(rrPart, nparts);
    const double rrOld = scalIn[0];
    const double beta = rrOld != 0.0 ? rrNew / rrOld : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) scalOut[0] = rrNew;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        p[i] = fma(beta, p[i], r[i]);
}

__global__ void copy_scalar(const double *__restrict__ src, double *__restrict__ dst) { dst[0] = src[0]; }

// The partials land in page-locked memory: a copy into pageable memory is
// synchronous inside the driver, and with several solvers on their own
// threads those waits starved every other thread's CUDA calls (measured on a
// served mix: SpMV requests beside 4 solvers held back for up to 0.4 s).
double host_sum(const double *dpart, int nparts, cudaStream_t s, double *pinned) {
    check_cuda(cudaMemcpyAsync(pinned, dpart, sizeof(double) * nparts, cudaMemcpyDeviceToHost, s), "copy partials");
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    double t = 0.0;
    for (int i = 0; i < nparts; ++i) t += pinned[i];
    return t;
}

// Bytes of L2 this process may keep persisting (set once per device, to the
// device's maximum; a per-context limit that ends with the process).
size_t persisting_l2_bytes(int dev) {
    static std::atomic<int64_t> cached[64];
    static std::atomic<uint64_t> done{0};
    if (dev < 0 || dev >= 64) return 0;
    if (done.load() & (1ull << dev)) return static_cast<size_t>(cached[dev].load());
    int maxPersist = 0;
    size_t granted = 0;
    if (cudaDeviceGetAttribute(&maxPersist, cudaDevAttrMaxPersistingL2CacheSize, dev) == cudaSuccess &&
        maxPersist > 0 && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, maxPersist) == cudaSuccess &&
        cudaDeviceGetLimit(&granted, cudaLimitPersistingL2CacheSize) != cudaSuccess)
        granted = 0;
    cudaGetLastError();
    cached[dev].store(static_cast<int64_t>(granted));
    done.fetch_or(1ull << dev);
    return granted;
}

}  // namespace

struct CgWork {
    int64_t n = 0;
    int nparts = 0;
    double *buf = nullptr;  // r, p, q (n each, contiguous: the L2 window) + 3 partial arrays + scalars
    double *r, *p, *q, *pqPart, *rrPart, *nPart, *scal;
    double *host = nullptr;  // page-locked: nparts partial sums, then r.r
};

void cg_free(CgWork *w) {
    if (!w) return;
    if (w->buf) cudaFree(w->buf);
    if (w->host) cudaFreeHost(w->host);
    delete w;
}

CgWork *cg_work(CgWork *w, int64_t n) {
    if (w && w->n >= n) return w;  // a larger workspace serves smaller systems
    cg_free(w);
    w = new CgWork();
    w->n = n;
    int dev = 0, sms = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    w->nparts = static_cast<int>(std::min<int64_t>(int64_t(sms) * 4, (n + kThreads - 1) / kThreads));
    if (w->nparts < 1) w->nparts = 1;
    const size_t words = 3 * static_cast<size_t>(n) + 3 * static_cast<size_t>(w->nparts) + 8;
    try {
        check_cuda(dev_alloc(&w->buf, words * sizeof(double)), "cudaMalloc(CG workspace)");
        check_cuda(pinned_alloc(&w->host, (static_cast<size_t>(w->nparts) + 1) * sizeof(double)),
                   "cudaMallocHost(CG partials)");
    } catch (...) {
        cg_free(w);
        throw;
    }
    double *b = w->buf;
    w->r = b; b += n;
    w->p = b; b += n;
    w->q = b; b += n;
    w->pqPart = b; b += w->nparts;
    w->rrPart = b; b += w->nparts;
    w->nPart = b; b += w->nparts;
    w->scal = b;  // scal[0], scal[1]: r.r of the current / next iteration
    return w;
}

int64_t cg_work_bytes(int64_t n, int sms) {
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * 4, (n + kThreads - 1) / kThreads));
    return 8 * (3 * n + 3 * parts + 8);
}

void cg_solve(const DevicePlan &A64, const DevicePlan &Ait, CgWork *w, const double *b, double *x,
              const CgParams &prm, void *stream, CgStats *st) {
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : A64.stream);
    const int64_t n = A64.n;
    if (n > w->n) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "CG workspace smaller than the system");
    // reduction partitions from n alone (what a workspace sized to n has), so
    // the result does not depend on the workspace's size
    const int G = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(w->nparts, (n + kThreads - 1) / kThreads)));
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    bool window = false;
    auto cleanup = [&] {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (window) {  // the stream goes back to normal caching
            cudaStreamAttrValue a;
            std::memset(&a, 0, sizeof(a));
            a.accessPolicyWindow.num_bytes = 0;
            cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &a);
            cudaGetLastError();
        }
    };
    int updates = 0, iters = 0;
    double rel = 0.0;
    try {
        if (prm.l2Persist) {
            int dev = 0;
            check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
            const size_t persist = persisting_l2_bytes(dev);
            const size_t bytes = 3 * sizeof(double) * static_cast<size_t>(n);
            int maxWindow = 0;
            cudaDeviceGetAttribute(&maxWindow, cudaDevAttrMaxAccessPolicyWindowSize, dev);
            cudaGetLastError();
            if (persist > 0 && maxWindow > 0) {
                cudaStreamAttrValue a;
                std::memset(&a, 0, sizeof(a));
                a.accessPolicyWindow.base_ptr = w->r;
                a.accessPolicyWindow.num_bytes = std::min(bytes, static_cast<size_t>(maxWindow));
                a.accessPolicyWindow.hitRatio =
                    static_cast<float>(std::min(1.0, double(persist) / double(a.accessPolicyWindow.num_bytes)));
                a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
                a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
                window = cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &a) == cudaSuccess;
                cudaGetLastError();
            }
        }
        // ||b||
        dot_partial<<<G, kThreads, 0, s>>>(b, b, n, w->nPart);
        const double bnorm = std::sqrt(host_sum(w->nPart, G, s, w->host));
        const double target = prm.tol * (bnorm > 0 ? bnorm : 1.0);
        // FP64 residual r = b - A x, its norm on the host and r.r in scal[0]
        auto true_residual = [&](int start) {
            launch_spmv(A64, x, w->q, s);
            residual<<<G, kThreads, 0, s>>>(b, w->q, w->r, n, w->nPart);
            cg_start<<<G, kThreads, 0, s>>>(w->r, w->p, n, w->nPart, G, w->scal, start);
            check_cuda(cudaGetLastError(), "CG residual");
            return std::sqrt(host_sum(w->nPart, G, s, w->host));
        };
        double rnorm = true_residual(1);
        rel = bnorm > 0 ? rnorm / bnorm : rnorm;
        double maxIterated = rnorm;  // largest iterated residual since the last update
        // one iteration = 5 launches; scal[0] holds r.r, scal[1] the next value
        auto iteration = [&](cudaStream_t stq) {
            launch_spmv(Ait, w->p, w->q, stq);
            dot_partial<<<G, kThreads, 0, stq>>>(w->p, w->q, n, w->pqPart);
            cg_update<<<G, kThreads, 0, stq>>>(x, w->r, w->p, w->q, n, w->pqPart, G, w->scal, w->rrPart);
            cg_direction<<<G, kThreads, 0, stq>>>(w->r, w->p, n, w->rrPart, G, w->scal, w->scal + 1);
            copy_scalar<<<1, 1, 0, stq>>>(w->scal + 1, w->scal);
        };
        bool fresh = true;  // rnorm is the FP64 residual of the current x
        while (rnorm > target && std::isfinite(rnorm) && iters < prm.maxIterations) {
            if (!exec) {
                check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                try {
                    for (int k = 0; k < prm.checkEvery; ++k) iteration(s);
                } catch (...) {
                    // end the failed capture: a stream left capturing would
                    // refuse this thread's later allocations and launches
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(s, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    throw;
                }
                check_cuda(cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture");
                check_cuda(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
            }
            check_cuda(cudaGraphLaunch(exec, s), "cudaGraphLaunch");
            iters += prm.checkEvery;
            fresh = false;
            double *rrHost = w->host + w->nparts;
            check_cuda(cudaMemcpyAsync(rrHost, w->scal, sizeof(double), cudaMemcpyDeviceToHost, s), "copy r.r");
            check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            const double iterated = std::sqrt(*rrHost);
            if (!std::isfinite(iterated)) break;
            maxIterated = std::max(maxIterated, iterated);
            const bool converging = iterated <= target;
            const bool drifted = iterated < prm.updateFactor * maxIterated;
            if (!(converging || drifted || iters >= prm.maxIterations)) continue;
            // reliable update: the FP64 residual replaces the iterated one
            // (p, the search direction, is kept)
            if (updates >= prm.maxUpdates) break;
            ++updates;
            rnorm = true_residual(0);
            fresh = true;
            maxIterated = rnorm;
        }
        if (!fresh) rnorm = true_residual(0);  // the reported residual is always b - A x in FP64
        rel = bnorm > 0 ? rnorm / bnorm : rnorm;
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    st->updates = updates;
    st->iterations = iters;
    st->relResidual = rel;
    st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace hbdia
