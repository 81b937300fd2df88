// Conjugate-gradient solver on the HBDIA SpMV with mixed-precision iterative
// refinement (SPD matrices).
//
//   outer (FP64):  r = b - A x   with the FP64 layout;  stop when
//                  ||r|| / ||b|| <= tol
//   inner:         CG on A d = r with the reduced-storage layout (FP32 values,
//                  FP64 accumulation; the reference values for the outer
//                  residual stay FP64) until ||r_in|| <= innerTol ||r||
//   update (FP64): x += d
//
// All vectors, dot products and norms are FP64.  Reductions are
// deterministic: every block reduces a fixed slice in a fixed order and every
// consumer of the partial sums adds them in the same order, so a solve is
// bit-reproducible run to run.  Scalars (alpha, beta, r.r) live in device
// memory; the inner iterations are captured once per solve in a CUDA graph of
// `checkEvery` iterations that is replayed until the inner tolerance is met,
// so the host synchronises once per `checkEvery` iterations.

#include <cuda_runtime.h>

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

// scal[0] = r.r (from partials); d = 0; p = r
__global__ void __launch_bounds__(kThreads) cg_start(const double *__restrict__ r, double *__restrict__ d,
                                                     double *__restrict__ p, int64_t n, const double *__restrict__ part,
                                                     int nparts, double *__restrict__ scal) {
    const double rr = sum_partials(part, nparts);
    if (blockIdx.x == 0 && threadIdx.x == 0) scal[0] = rr;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads) {
        d[i] = 0.0;
        p[i] = r[i];
    }
}

// alpha = r.r / p.q;  d += alpha p;  r -= alpha q;  partial sums of new r.r
__global__ void __launch_bounds__(kThreads) cg_update(double *__restrict__ d, double *__restrict__ r,
                                                      const double *__restrict__ p, const double *__restrict__ q,
                                                      int64_t n, const double *__restrict__ pqPart, int nparts,
                                                      const double *__restrict__ scal, double *__restrict__ rrPart) {
    const double pq = sum_partials(pqPart, nparts);
    const double alpha = pq != 0.0 ? scal[0] / pq : 0.0;
    double v = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads) {
        d[i] = fma(alpha, p[i], d[i]);
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

__global__ void __launch_bounds__(kThreads) add_into(double *__restrict__ x, const double *__restrict__ d,
                                                     int64_t n) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
        x[i] += d[i];
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

}  // namespace

struct CgWork {
    int64_t n = 0;
    int nparts = 0;
    double *buf = nullptr;  // r, p, q, d, tmp (n each) + 3 partial arrays + scalars
    double *r, *p, *q, *d, *tmp, *pqPart, *rrPart, *nPart, *scal;
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
    const size_t words = 5 * static_cast<size_t>(n) + 3 * static_cast<size_t>(w->nparts) + 8;
    try {
        check_cuda(cudaMalloc(&w->buf, words * sizeof(double)), "cudaMalloc(CG workspace)");
        check_cuda(cudaMallocHost(&w->host, (static_cast<size_t>(w->nparts) + 1) * sizeof(double)),
                   "cudaMallocHost(CG partials)");
    } catch (...) {
        cg_free(w);
        throw;
    }
    double *b = w->buf;
    w->r = b; b += n;
    w->p = b; b += n;
    w->q = b; b += n;
    w->d = b; b += n;
    w->tmp = b; b += n;
    w->pqPart = b; b += w->nparts;
    w->rrPart = b; b += w->nparts;
    w->nPart = b; b += w->nparts;
    w->scal = b;  // scal[0], scal[1]: r.r of the current / next iteration
    return w;
}

// Mixed-precision CG.  A64 computes the outer residual; Ainner (FP32 or FP64
// storage of the same matrix) runs the inner iterations.
void cg_solve(const DevicePlan &A64, const DevicePlan &Ainner, CgWork *w, const double *b, double *x, double tol,
              int maxOuter, int maxInner, double innerTol, int checkEvery, void *stream, int32_t *outerIt,
              int32_t *innerIt, double *relRes, double *seconds) {
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : A64.stream);
    const int64_t n = A64.n;
    if (n > w->n) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "CG workspace smaller than the system");
    // reduction partitions from n alone (what a workspace sized to n has), so
    // the result does not depend on the workspace's size
    const int G = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(w->nparts, (n + kThreads - 1) / kThreads)));
    // ||b||
    dot_partial<<<G, kThreads, 0, s>>>(b, b, n, w->nPart);
    const double bnorm = std::sqrt(host_sum(w->nPart, G, s, w->host));
    int outer = 0, inner = 0;
    double rel = 0.0;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    auto cleanup = [&] {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    };
    try {
        // one inner iteration = 4 launches; scal[0] holds r.r, scal[1] the next value
        auto iteration = [&](cudaStream_t st) {
            launch_spmv(Ainner, w->p, w->q, st);
            dot_partial<<<G, kThreads, 0, st>>>(w->p, w->q, n, w->pqPart);
            cg_update<<<G, kThreads, 0, st>>>(w->d, w->r, w->p, w->q, n, w->pqPart, G, w->scal, w->rrPart);
            cg_direction<<<G, kThreads, 0, st>>>(w->r, w->p, n, w->rrPart, G, w->scal, w->scal + 1);
            copy_scalar<<<1, 1, 0, st>>>(w->scal + 1, w->scal);
        };
        for (;;) {
            // outer residual in FP64
            launch_spmv(A64, x, w->tmp, s);
            residual<<<G, kThreads, 0, s>>>(b, w->tmp, w->r, n, w->nPart);
            const double rnorm = std::sqrt(host_sum(w->nPart, G, s, w->host));
            rel = bnorm > 0 ? rnorm / bnorm : rnorm;
            if (rel <= tol || outer >= maxOuter || !std::isfinite(rel)) break;
            ++outer;
            // inner CG on A d = r
            cg_start<<<G, kThreads, 0, s>>>(w->r, w->d, w->p, n, w->nPart, G, w->scal);
            check_cuda(cudaGetLastError(), "CG start");
            if (!exec) {
                check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                for (int k = 0; k < checkEvery; ++k) iteration(s);
                check_cuda(cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture");
                check_cuda(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
            }
            const double target = innerTol * rnorm;
            int it = 0;
            while (it < maxInner) {
                check_cuda(cudaGraphLaunch(exec, s), "cudaGraphLaunch");
                it += checkEvery;
                double *rrHost = w->host + w->nparts;
                check_cuda(cudaMemcpyAsync(rrHost, w->scal, sizeof(double), cudaMemcpyDeviceToHost, s), "copy r.r");
                check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
                const double rr = *rrHost;
                if (!(std::sqrt(rr) > target)) break;  // converged (or not finite)
            }
            inner += it;
            add_into<<<G, kThreads, 0, s>>>(x, w->d, n);
            check_cuda(cudaGetLastError(), "CG update");
        }
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    *outerIt = outer;
    *innerIt = inner;
    *relRes = rel;
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace hbdia
