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
// Lockstep groups: several solves on the same matrix (each with its own b, x
// and workspace) advance together, their iterations' SpMVs forming ONE
// vector-list SpMM (each stored value read once for all of them; column j
// equals the SpMV of p_j bit for bit) and their vector kernels one launch
// each (blockIdx.y = solve, the same per-solve partition as a lone solve).
// Each solve keeps its own reliable-update and convergence schedule and
// leaves the group when done, so its result equals what it gives alone, bit
// for bit; a lone solve is a group of one.
//
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

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

// The iteration's vector kernels for a group: solve j = blockIdx.y uses its
// own vectors, partial sums and scalars, with blockIdx.x / gridDim.x exactly
// as a lone solve's launch has them.
constexpr int kCgGroupMax = 16;
struct GroupVecs {
    double *x[kCgGroupMax], *r[kCgGroupMax], *p[kCgGroupMax], *q[kCgGroupMax];
    double *pqPart[kCgGroupMax], *rrPart[kCgGroupMax], *scal[kCgGroupMax];
};

__global__ void __launch_bounds__(kThreads) g_dot_pq(const __grid_constant__ GroupVecs V, int64_t n) {
    const int j = blockIdx.y;
    const double *__restrict__ a = V.p[j];
    const double *__restrict__ b = V.q[j];
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        v = fma(a[i], b[i], v);
    const double s = block_sum(v);
    if (threadIdx.x == 0) V.pqPart[j][blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) g_update(const __grid_constant__ GroupVecs V, int64_t n, int nparts) {
    const int j = blockIdx.y;
    double *__restrict__ x = V.x[j];
    double *__restrict__ r = V.r[j];
    const double *__restrict__ p = V.p[j];
    const double *__restrict__ q = V.q[j];
    const double pq = sum_partials(V.pqPart[j], nparts);
    const double alpha = pq != 0.0 ? V.scal[j][0] / pq : 0.0;
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        v = fma(ri, ri, v);
    }
    const double s = block_sum(v);
    if (threadIdx.x == 0) V.rrPart[j][blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) g_direction(const __grid_constant__ GroupVecs V, int64_t n, int nparts) {
    const int j = blockIdx.y;
    const double *__restrict__ r = V.r[j];
    double *__restrict__ p = V.p[j];
    const double rrNew = sum_partials(V.rrPart[j], nparts);
    const double rrOld = V.scal[j][0];
    const double beta = rrOld != 0.0 ? rrNew / rrOld : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) V.scal[j][1] = rrNew;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        p[i] = fma(beta, p[i], r[i]);
}

__global__ void g_copy_scalar(const __grid_constant__ GroupVecs V, int k) {
    const int j = threadIdx.x;
    if (j < k) V.scal[j][0] = V.scal[j][1];
}

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

}  // namespace

struct CgWork {
    int64_t n = 0;
    int nparts = 0;
    double *buf = nullptr;  // r, p, q (n each) + 3 partial arrays + scalars
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

void cg_solve_group(const DevicePlan &A64, const DevicePlan &Ait, CgCall *calls, int k, const CgParams &prm,
                    void *stream) {
    if (k < 1 || k > kCgGroupMax) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "CG group of 1 to 16 solves");
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : A64.stream);
    const int64_t n = A64.n;
    for (int j = 0; j < k; ++j)
        if (!calls[j].w || n > calls[j].w->n) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "CG workspace smaller than the system");
    // reduction partitions from n alone (what a workspace sized to n has), so
    // the result does not depend on the workspace's size
    int G = 1;
    {
        int dev = 0, sms = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        G = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * 4, (n + kThreads - 1) / kThreads)));
    }
    for (int j = 0; j < k; ++j)  // a workspace for at least n rows holds at least G partial sums
        if (calls[j].w->nparts < G) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "CG workspace smaller than the system");
    struct State {
        double bnorm = 0, target = 0, rnorm = 0, maxIterated = 0;
        int iters = 0, updates = 0;
        bool fresh = true, done = false;
    };
    std::vector<State> S(static_cast<size_t>(k));
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    std::vector<int> graphSet;  // the active solves the captured graph iterates
    auto dropGraph = [&] {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graphSet.clear();
    };
    auto cleanup = [&] { dropGraph(); };
    // FP64 residual of solve j: r = b - A x, its norm on the host and r.r in
    // its scal[0]; with `start` also p = r
    auto true_residual = [&](int j, int start) {
        CgWork *w = calls[j].w;
        launch_spmv(A64, calls[j].x, w->q, s);
        residual<<<G, kThreads, 0, s>>>(calls[j].b, w->q, w->r, n, w->nPart);
        cg_start<<<G, kThreads, 0, s>>>(w->r, w->p, n, w->nPart, G, w->scal, start);
        check_cuda(cudaGetLastError(), "CG residual");
        return std::sqrt(host_sum(w->nPart, G, s, w->host));
    };
    auto alive = [&](const State &st) { return st.rnorm > st.target && std::isfinite(st.rnorm) && st.iters < prm.maxIterations; };
    try {
        for (int j = 0; j < k; ++j) {
            CgWork *w = calls[j].w;
            dot_partial<<<G, kThreads, 0, s>>>(calls[j].b, calls[j].b, n, w->nPart);
            S[j].bnorm = std::sqrt(host_sum(w->nPart, G, s, w->host));
            S[j].target = prm.tol * (S[j].bnorm > 0 ? S[j].bnorm : 1.0);
            S[j].rnorm = true_residual(j, 1);
            S[j].maxIterated = S[j].rnorm;
            S[j].done = !alive(S[j]);
        }
        for (;;) {
            std::vector<int> act;
            for (int j = 0; j < k; ++j)
                if (!S[j].done) act.push_back(j);
            if (act.empty()) break;
            if (act != graphSet) {
                // one iteration = the SpMM of the active solves + 4 launches
                dropGraph();
                GroupVecs V;
                std::memset(&V, 0, sizeof(V));
                std::vector<const void *> ps;
                std::vector<void *> qs;
                for (size_t a = 0; a < act.size(); ++a) {
                    CgWork *w = calls[act[a]].w;
                    V.x[a] = calls[act[a]].x;
                    V.r[a] = w->r;
                    V.p[a] = w->p;
                    V.q[a] = w->q;
                    V.pqPart[a] = w->pqPart;
                    V.rrPart[a] = w->rrPart;
                    V.scal[a] = w->scal;
                    ps.push_back(w->p);
                    qs.push_back(w->q);
                }
                const int ka = static_cast<int>(act.size());
                const dim3 grid(static_cast<unsigned>(G), static_cast<unsigned>(ka));
                check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                try {
                    for (int it = 0; it < prm.checkEvery; ++it) {
                        if (ka == 1 || Ait.quadLayout) {  // (quad-interleaved values: SpMV only)
                            for (int a = 0; a < ka; ++a) launch_spmv(Ait, ps[a], qs[a], s);
                        } else {
                            launch_spmv_list(Ait, ps.data(), qs.data(), ka, s);
                        }
                        g_dot_pq<<<grid, kThreads, 0, s>>>(V, n);
                        g_update<<<grid, kThreads, 0, s>>>(V, n, G);
                        g_direction<<<grid, kThreads, 0, s>>>(V, n, G);
                        g_copy_scalar<<<1, 32, 0, s>>>(V, ka);
                    }
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
                graphSet = act;
            }
            check_cuda(cudaGraphLaunch(exec, s), "cudaGraphLaunch");
            for (int j : act) {
                S[j].iters += prm.checkEvery;
                S[j].fresh = false;
                CgWork *w = calls[j].w;
                check_cuda(cudaMemcpyAsync(w->host + w->nparts, w->scal, sizeof(double), cudaMemcpyDeviceToHost, s),
                           "copy r.r");
            }
            check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            for (int j : act) {
                State &st = S[j];
                CgWork *w = calls[j].w;
                const double iterated = std::sqrt(w->host[w->nparts]);
                if (!std::isfinite(iterated)) {
                    st.done = true;
                    continue;
                }
                st.maxIterated = std::max(st.maxIterated, iterated);
                const bool converging = iterated <= st.target;
                const bool drifted = iterated < prm.updateFactor * st.maxIterated;
                if (!(converging || drifted || st.iters >= prm.maxIterations)) continue;
                // reliable update: the FP64 residual replaces the iterated one
                // (p, the search direction, is kept)
                if (st.updates >= prm.maxUpdates) {
                    st.done = true;
                    continue;
                }
                ++st.updates;
                st.rnorm = true_residual(j, 0);
                st.fresh = true;
                st.maxIterated = st.rnorm;
                if (!alive(st)) st.done = true;
            }
        }
        // the reported residual is always b - A x in FP64
        for (int j = 0; j < k; ++j)
            if (!S[j].fresh) S[j].rnorm = true_residual(j, 0);
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int j = 0; j < k; ++j) {
        CgStats *st = calls[j].stats;
        if (!st) continue;
        st->updates = S[j].updates;
        st->iterations = S[j].iters;
        st->relResidual = S[j].bnorm > 0 ? S[j].rnorm / S[j].bnorm : S[j].rnorm;
        st->seconds = secs;
    }
}

void cg_solve(const DevicePlan &A64, const DevicePlan &Ait, CgWork *w, const double *b, double *x,
              const CgParams &prm, void *stream, CgStats *st) {
    CgCall c{b, x, w, st};
    cg_solve_group(A64, Ait, &c, 1, prm, stream);
}

}  // namespace hbdia
