// Serving engine: resident matrices, requests from host threads, continuous
// batching of SpMVs and a pool of CG solvers.
//
// Requests come from any host thread (hbdia_server_submit) and complete in
// the background (hbdia_server_wait).  Two kinds:
//  * SpMV: y = A x.  A scheduler thread serves them in steps.  With batching
//    on, a step takes every pending request (up to maxRhs per matrix, oldest
//    first; the rest wait for the next step): the requests of one matrix
//    become one column-major SpMM -- each x copied straight into its column
//    of the matrix's staging block, each y copied straight out of its column
//    -- so the matrix's values cross HBM once for all of them, and the
//    matrices of a step run concurrently on a ring of streams.  Requests
//    that arrive during a step join the next one.  With batching off, one
//    request per launch in arrival order (the plain form it is measured
//    against).
//  * CG: solve A y = x to a relative residual, by the mixed-precision CG of
//    cg.cu on one of cgWorkers worker threads (own stream, own workspace).
// x and y are host buffers (hbdia_server_submit: copied in and out on the
// server's streams) or device buffers (hbdia_server_submit_device: read and
// written in place).  A step's device SpMV requests on one matrix become one
// vector-list SpMM (each value read once for up to 32 requests, no staging
// copies); its host requests one column-major SpMM over the staging block.
// A request's result does not depend on what it was batched with: column j
// of the SpMM equals the SpMV of x_j bit for bit, and a CG solve depends only
// on its matrix and right-hand side.
//
// Admission: a matrix is accepted only while everything the server holds on
// the device -- its plans (FP64, and the reduced-storage copy SpMVs and the
// CG inner iterations use), its staging blocks, and the CG workspaces --
// stays within memoryBudget.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "handles.hpp"
#include "hbdia_internal.hpp"

namespace hbdia {

namespace {

constexpr int kSpmvStreams = 16;

struct ServedMatrix {
    DevicePlan p64;   // FP64 values: CG outer residual; SpMVs when spmvStorage is NATIVE
    DevicePlan pLow;  // reduced storage (when one is asked for)
    int32_t n = 0, rowsX = 0;
    double *X = nullptr, *Y = nullptr;  // column-major staging blocks, maxRhs columns
    int64_t bytes = 0;
    const DevicePlan &spmvPlan(int32_t storage) const { return storage == HBDIA_STORE_NATIVE ? p64 : pLow; }
    const DevicePlan &cgInner(int32_t storage) const { return storage == HBDIA_STORE_NATIVE ? p64 : pLow; }
};

struct Request {
    uint64_t ticket = 0;
    int32_t matrix = 0, kind = 0;
    const ServedMatrix *m = nullptr;  // taken under the server lock at submit
    const double *x = nullptr;
    double *y = nullptr;
    bool device = false;  // x, y in device memory
    hbdia_request_info info{};
    bool done = false;
};

double now_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct Server {
    hbdia_server_options opt{};
    int device = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable cvWork, cvDone, cvCg;
    std::vector<std::unique_ptr<ServedMatrix>> mats;
    int64_t used = 0;  // device bytes held
    int32_t maxN = 0;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request *> spmvQ, cgQ;
    uint64_t nextTicket = 1;
    bool stop = false;
    bool paused = false;  // requests queue up; no step or solve starts
    hbdia_server_stats stats{};
    std::vector<cudaStream_t> streams;
    std::thread sched;
    std::vector<std::thread> cgThreads;
};

namespace {

void complete(Server *S, const std::vector<Request *> &rs, int status, double finished) {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Request *r : rs) {
        r->info.status = status;
        r->info.finished = finished;
        r->done = true;
        S->stats.completed += 1;
    }
    S->cvDone.notify_all();
}

// One scheduler step: the requests in `step`, grouped by matrix in order of
// first arrival.
void serve_step(Server *S, std::vector<Request *> &step) {
    std::vector<int32_t> order;
    std::map<int32_t, std::vector<Request *>> groups;
    for (Request *r : step) {
        auto &g = groups[r->matrix];
        if (g.empty()) order.push_back(r->matrix);
        g.push_back(r);
    }
    const double started = now_since(S->t0);
    int status = HBDIA_OK;
    std::string err;
    size_t used = 0;
    try {
        for (size_t gi = 0; gi < order.size(); ++gi) {
            const int32_t mid = order[gi];
            auto &g = groups[mid];
            const ServedMatrix &M = *g[0]->m;
            cudaStream_t st = S->streams[gi % S->streams.size()];
            used = std::min(S->streams.size(), std::max(used, gi + 1));  // streams of the ring in use
            const DevicePlan &P = M.spmvPlan(S->opt.spmvStorage);
            std::vector<Request *> host;
            std::vector<const void *> dx;
            std::vector<void *> dy;
            for (Request *r : g) {
                r->info.started = started;
                if (r->device) {
                    dx.push_back(r->x);
                    dy.push_back(r->y);
                } else {
                    host.push_back(r);
                }
            }
            for (Request *r : g) r->info.batchRhs = static_cast<int32_t>(r->device ? dx.size() : host.size());
            // device requests: one vector-list SpMM, in place
            if (dx.size() == 1) launch_spmv(P, dx[0], dy[0], st);
            else if (!dx.empty()) launch_spmv_list(P, dx.data(), dy.data(), static_cast<int32_t>(dx.size()), st);
            // host requests: through the staging block
            const int32_t k = static_cast<int32_t>(host.size());
            const size_t xb = static_cast<size_t>(M.rowsX) * sizeof(double);
            const size_t yb = static_cast<size_t>(M.n) * sizeof(double);
            for (int32_t j = 0; j < k; ++j)
                check_cuda(cudaMemcpyAsync(M.X + static_cast<int64_t>(j) * M.rowsX, host[j]->x, xb,
                                           cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(request x)");
            if (k == 1) launch_spmv(P, M.X, M.Y, st);
            else if (k > 1) launch_spmm(P, M.X, M.rowsX, M.Y, M.n, k, st, true);
            for (int32_t j = 0; j < k; ++j)
                check_cuda(cudaMemcpyAsync(host[j]->y, M.Y + static_cast<int64_t>(j) * M.n, yb,
                                           cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(request y)");
        }
    } catch (const Error &e) {
        status = e.status;
        err = e.what();
    }
    for (size_t j = 0; j < used; ++j) {
        const cudaError_t rc = cudaStreamSynchronize(S->streams[j]);
        if (rc != cudaSuccess && status == HBDIA_OK) status = HBDIA_ERR_CUDA;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stats.spmvSteps += 1;
        S->stats.spmvLaunches += static_cast<int64_t>(order.size());
    }
    complete(S, step, status, now_since(S->t0));
}

void scheduler(Server *S) {
    cudaSetDevice(S->device);
    for (;;) {
        std::vector<Request *> step;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cvWork.wait(lk, [&] { return S->stop || (!S->paused && !S->spmvQ.empty()); });
            if (S->spmvQ.empty()) return;  // stopping and drained
            if (!S->opt.batching) {
                step.push_back(S->spmvQ.front());
                S->spmvQ.pop_front();
            } else {
                std::map<int32_t, int32_t> taken;
                std::deque<Request *> rest;
                for (Request *r : S->spmvQ) {
                    int32_t &c = taken[r->matrix];
                    if (c < S->opt.maxRhs) {
                        ++c;
                        step.push_back(r);
                    } else {
                        rest.push_back(r);
                    }
                }
                S->spmvQ.swap(rest);
            }
        }
        serve_step(S, step);
    }
}

void cg_worker(Server *S) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    CgWork *w = nullptr;
    double *bx = nullptr;  // b and x, maxN each
    int32_t cap = 0;
    const bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cvCg.wait(lk, [&] { return S->stop || (!S->paused && !S->cgQ.empty()); });
            if (S->cgQ.empty()) break;
            r = S->cgQ.front();
            S->cgQ.pop_front();
        }
        r->info.started = now_since(S->t0);
        r->info.batchRhs = 1;
        int status = HBDIA_OK;
        try {
            if (!ok) throw Error(HBDIA_ERR_CUDA, "CG worker stream");
            const ServedMatrix &M = *r->m;
            if (!r->device && M.n > cap) {
                if (bx) cudaFree(bx);
                bx = nullptr;
                check_cuda(cudaMalloc(&bx, 2 * sizeof(double) * static_cast<size_t>(M.n)), "cudaMalloc(CG b, x)");
                cap = M.n;
            }
            w = cg_work(w, M.n);
            // device requests solve in place: b = request x, solution into request y
            const double *b = r->device ? r->x : bx;
            double *x = r->device ? r->y : bx + cap;
            const size_t nb = sizeof(double) * static_cast<size_t>(M.n);
            if (!r->device)
                check_cuda(cudaMemcpyAsync(bx, r->x, nb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(CG b)");
            check_cuda(cudaMemsetAsync(x, 0, nb, st), "cudaMemsetAsync(CG x)");
            const hbdia_server_options &o = S->opt;
            double secs = 0.0;
            cg_solve(M.p64, M.cgInner(o.cgInnerStorage), w, b, x, o.cgTol, o.cgMaxOuter, o.cgMaxInner, o.cgInnerTol,
                     o.cgCheckEvery, st, &r->info.cgOuter, &r->info.cgInner, &r->info.cgRelResidual, &secs);
            if (!r->device)
                check_cuda(cudaMemcpyAsync(r->y, x, nb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(CG y)");
            check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize(CG)");
            if (r->info.cgRelResidual > o.cgTol) status = HBDIA_ERR_RUNTIME;  // not converged
        } catch (const Error &e) {
            status = e.status;
        } catch (const std::exception &) {
            status = HBDIA_ERR_RUNTIME;
        }
        complete(S, {r}, status, now_since(S->t0));
    }
    cg_free(w);
    if (bx) cudaFree(bx);
    if (st) cudaStreamDestroy(st);
}

void free_matrix(ServedMatrix &M) {
    free_plan(M.p64);
    free_plan(M.pLow);
    if (M.X) cudaFree(M.X);
    if (M.Y) cudaFree(M.Y);
    M.X = M.Y = nullptr;
}

}  // namespace

void server_default_options(hbdia_server_options *o) {
    std::memset(o, 0, sizeof(*o));
    o->memoryBudget = 150LL * 1000 * 1000 * 1000;
    o->batching = 1;
    o->maxRhs = 16;
    o->spmvStorage = HBDIA_STORE_F32;
    o->cgInnerStorage = HBDIA_STORE_F32;
    o->cgWorkers = 4;
    o->cgTol = 1e-10;
    o->cgInnerTol = 1e-6;
    o->cgMaxOuter = 50;
    o->cgMaxInner = 5000;
    o->cgCheckEvery = 10;
}

Server *server_create(const hbdia_server_options &o) {
    if (o.memoryBudget <= 0 || o.maxRhs < 1 || o.maxRhs > 64 || o.cgWorkers < 1 || o.cgWorkers > 64 ||
        o.cgTol <= 0 || o.cgInnerTol <= 0 || o.cgMaxOuter < 1 || o.cgMaxInner < 1 || o.cgCheckEvery < 1)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad server options");
    for (int32_t st : {o.spmvStorage, o.cgInnerStorage})
        if (st != HBDIA_STORE_NATIVE && st != HBDIA_STORE_F32 && st != HBDIA_STORE_BF16_SCALED)
            throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown value storage");
    if (o.spmvStorage != HBDIA_STORE_NATIVE && o.cgInnerStorage != HBDIA_STORE_NATIVE &&
        o.spmvStorage != o.cgInnerStorage)
        throw Error(HBDIA_ERR_UNSUPPORTED, "SpMV and CG inner storage must match when both are reduced");
    auto S = std::make_unique<Server>();
    S->opt = o;
    check_cuda(cudaGetDevice(&S->device), "cudaGetDevice");
    for (int i = 0; i < kSpmvStreams; ++i) {
        cudaStream_t st = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate(server)");
        S->streams.push_back(st);
    }
    Server *raw = S.get();
    S->sched = std::thread(scheduler, raw);
    for (int32_t i = 0; i < o.cgWorkers; ++i) S->cgThreads.emplace_back(cg_worker, raw);
    return S.release();
}

void server_destroy(Server *S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cvWork.notify_all();
    S->cvCg.notify_all();
    if (S->sched.joinable()) S->sched.join();
    for (auto &t : S->cgThreads)
        if (t.joinable()) t.join();
    for (cudaStream_t st : S->streams) cudaStreamDestroy(st);
    for (auto &m : S->mats) free_matrix(*m);
    delete S;
}

int32_t server_add_matrix(Server *S, const hbdia_matrix *m) {
    if (m->dtype != HBDIA_F64) throw Error(HBDIA_ERR_UNSUPPORTED, "the server serves double matrices");
    if (!m->hasHBDIA || !m->hostLayout) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix has no host HBDIA layout");
    const HostLayout<double> &L = m->L64;
    auto M = std::make_unique<ServedMatrix>();
    M->n = L.numRows;
    M->rowsX = std::max(L.numRows, L.numCols);
    const int32_t low = S->opt.spmvStorage != HBDIA_STORE_NATIVE ? S->opt.spmvStorage : S->opt.cgInnerStorage;
    try {
        build_plan(L, HBDIA_STORE_NATIVE, M->p64);
        if (low != HBDIA_STORE_NATIVE) build_plan(L, low, M->pLow);
        const int64_t staging =
            static_cast<int64_t>(S->opt.maxRhs) * (static_cast<int64_t>(M->rowsX) + M->n) * 8;
        // CG workspaces grow to the largest system: 5 vectors of the workspace + b, x per worker
        int64_t cgGrow = 0;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (M->n > S->maxN) cgGrow = static_cast<int64_t>(S->opt.cgWorkers) * 7 * 8 * (M->n - S->maxN);
        }
        M->bytes = static_cast<int64_t>(M->p64.bytes + M->pLow.bytes) + staging;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->used + M->bytes + cgGrow > S->opt.memoryBudget)
                throw Error(HBDIA_ERR_NO_MEMORY,
                            "admission refused: the matrix needs " + std::to_string(M->bytes + cgGrow) +
                                " device bytes and the server holds " + std::to_string(S->used) + " of its " +
                                std::to_string(S->opt.memoryBudget) + "-byte budget");
        }
        check_cuda(cudaMalloc(&M->X, sizeof(double) * static_cast<size_t>(S->opt.maxRhs) * M->rowsX),
                   "cudaMalloc(server staging x)");
        check_cuda(cudaMalloc(&M->Y, sizeof(double) * static_cast<size_t>(S->opt.maxRhs) * M->n),
                   "cudaMalloc(server staging y)");
        std::lock_guard<std::mutex> lk(S->mu);
        S->used += M->bytes + cgGrow;
        S->maxN = std::max(S->maxN, M->n);
        S->mats.push_back(std::move(M));
        S->stats.deviceBytes = S->used;
        return static_cast<int32_t>(S->mats.size() - 1);
    } catch (...) {
        free_matrix(*M);
        throw;
    }
}

uint64_t server_submit(Server *S, int32_t matrix, int32_t kind, const double *x, double *y, bool device) {
    if (!x || !y) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null request vector");
    if (kind != HBDIA_REQ_SPMV && kind != HBDIA_REQ_CG) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown request kind");
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) throw Error(HBDIA_ERR_RUNTIME, "server is stopping");
    if (matrix < 0 || matrix >= static_cast<int32_t>(S->mats.size()))
        throw Error(HBDIA_ERR_OUT_OF_RANGE, "unknown matrix id");
    auto r = std::make_unique<Request>();
    r->ticket = S->nextTicket++;
    r->matrix = matrix;
    r->m = S->mats[matrix].get();
    r->kind = kind;
    r->x = x;
    r->y = y;
    r->device = device;
    r->info.kind = kind;
    r->info.matrix = matrix;
    r->info.submitted = now_since(S->t0);
    r->info.status = HBDIA_OK;
    Request *raw = r.get();
    S->reqs.emplace(raw->ticket, std::move(r));
    if (kind == HBDIA_REQ_SPMV) {
        S->spmvQ.push_back(raw);
        S->stats.spmvRequests += 1;
        S->cvWork.notify_one();
    } else {
        S->cgQ.push_back(raw);
        S->stats.cgRequests += 1;
        S->cvCg.notify_one();
    }
    return raw->ticket;
}

void server_pause(Server *S, bool paused) {
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->paused = paused;
    }
    S->cvWork.notify_all();
    S->cvCg.notify_all();
}

void server_wait(Server *S, uint64_t ticket, hbdia_request_info *info) {
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown or already collected ticket");
    Request *r = it->second.get();
    if (S->paused && !r->done) throw Error(HBDIA_ERR_RUNTIME, "server is paused: the request cannot complete");
    S->cvDone.wait(lk, [&] { return r->done; });
    if (info) *info = r->info;
    S->reqs.erase(it);
}

void server_stats(Server *S, hbdia_server_stats *out) {
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->deviceBytes = S->used;
    out->matrices = static_cast<int32_t>(S->mats.size());
}

}  // namespace hbdia
