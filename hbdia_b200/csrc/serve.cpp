// Serving engine: resident matrices, requests from host threads, continuous
// batching of SpMVs and a pool of CG solvers.
//
// Requests come from any host thread (hbdia_server_submit) and complete in
// the background (hbdia_server_wait).  Two kinds:
//  * SpMV: y = A x.  Each resident matrix has its own queue and its own
//    stream.  Whenever a matrix has pending requests and fewer than
//    maxInFlight batches running, the scheduler thread takes up to maxRhs of
//    them (oldest first; with batching off, one) and issues them as one SpMM
//    -- device vectors as a vector-list SpMM read and written in place, host
//    vectors through the matrix's column-major staging block -- so the
//    matrix's values cross HBM once for all of them.  A host function queued
//    behind each batch wakes the same thread, which completes the batch and
//    issues the matrix's next one, so a request waits only for its own
//    matrix, never for a global step; requests that arrive while a batch runs
//    form the next one (continuous batching).  No thread polls the GPU.  With
//    batching off, one request per launch (the plain form it is measured
//    against).
//  * CG: solve A y = x to a relative residual, by the mixed-precision CG of
//    cg.cu on one of cgWorkers worker threads (own stream, own workspace).
// x and y are host buffers (hbdia_server_submit: copied in and out on the
// server's streams) or device buffers (hbdia_server_submit_device: read and
// written in place).  A batch's device SpMV requests on one matrix become one
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


struct Request;

// An SpMV batch on its matrix's stream: its requests and the event (from the
// matrix's pool) recorded behind its work.
struct SpmvBatch {
    std::vector<Request *> reqs;
    cudaEvent_t done = nullptr;
};

struct ServedMatrix {
    DevicePlan p64;   // FP64 values: CG outer residual; SpMVs when spmvStorage is NATIVE
    DevicePlan pLow;  // reduced storage of the SpMVs (when one is asked for)
    DevicePlan pCg;   // the CG iterations' storage when it differs from pLow's
    int32_t n = 0, rowsX = 0;
    double *X = nullptr, *Y = nullptr;  // column-major staging blocks, maxRhs columns
    int64_t bytes = 0;
    Server *server = nullptr;
    cudaStream_t stream = nullptr;         // this matrix's SpMV batches, in order
    std::vector<cudaEvent_t> freeEvents;   // maxInFlight events, reused (scheduler thread)
    std::deque<SpmvBatch> running;         // issued, in stream order (scheduler thread)
    std::deque<Request *> pending;         // SpMV requests not yet issued (server lock)
    const DevicePlan &spmvPlan(int32_t storage) const { return storage == HBDIA_STORE_NATIVE ? p64 : pLow; }
    const DevicePlan &cgIter(int32_t storage) const {
        return storage == HBDIA_STORE_NATIVE ? p64 : pCg.base ? pCg : pLow;
    }
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

// With batches in flight and no doorbell, the scheduler queries every running
// batch's event this often (a batch whose doorbell never runs -- a failed
// host-function launch, a context error -- still completes).
constexpr int kSweepMs = 50;

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
    std::deque<Request *> cgQ;
    int64_t spmvPending = 0;  // SpMV requests queued on the matrices
    std::vector<ServedMatrix *> rung;  // matrices whose doorbell rang since the scheduler last looked
    uint64_t nextTicket = 1;
    bool stop = false;
    bool paused = false;  // requests queue up; no batch or solve starts
    hbdia_server_stats stats{};
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

// Host function queued behind every batch: tells the scheduler that work on
// this matrix's stream has finished.  It makes no CUDA call (a host function
// must not), and no thread holds the server lock across a CUDA call, so it
// cannot deadlock against one.
void CUDART_CB doorbell(void *p) {
    ServedMatrix *M = static_cast<ServedMatrix *>(p);
    Server *S = M->server;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->rung.push_back(M);
    }
    S->cvWork.notify_one();
}

// Issues one matrix's batch on its stream (scheduler thread, no lock held).
// On a failure the requests complete with its status at once.
void issue_batch(Server *S, ServedMatrix *M, std::vector<Request *> &reqs) {
    const double started = now_since(S->t0);
    cudaStream_t st = M->stream;
    try {
        const DevicePlan &P = M->spmvPlan(S->opt.spmvStorage);
        std::vector<Request *> host;
        std::vector<const void *> dx;
        std::vector<void *> dy;
        for (Request *r : reqs) {
            r->info.started = started;
            r->info.status = HBDIA_OK;
            if (r->device) {
                dx.push_back(r->x);
                dy.push_back(r->y);
            } else {
                host.push_back(r);
            }
        }
        for (Request *r : reqs) r->info.batchRhs = static_cast<int32_t>(r->device ? dx.size() : host.size());
        // device requests: one vector-list SpMM, in place
        if (dx.size() == 1) launch_spmv(P, dx[0], dy[0], st);
        else if (!dx.empty()) launch_spmv_list(P, dx.data(), dy.data(), static_cast<int32_t>(dx.size()), st);
        // host requests: through the staging block
        const int32_t k = static_cast<int32_t>(host.size());
        const size_t xb = static_cast<size_t>(M->rowsX) * sizeof(double);
        const size_t yb = static_cast<size_t>(M->n) * sizeof(double);
        for (int32_t j = 0; j < k; ++j)
            check_cuda(cudaMemcpyAsync(M->X + static_cast<int64_t>(j) * M->rowsX, host[j]->x, xb,
                                       cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(request x)");
        if (k == 1) launch_spmv(P, M->X, M->Y, st);
        else if (k > 1) launch_spmm(P, M->X, M->rowsX, M->Y, M->n, k, st, true);
        for (int32_t j = 0; j < k; ++j)
            check_cuda(cudaMemcpyAsync(host[j]->y, M->Y + static_cast<int64_t>(j) * M->n, yb,
                                       cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(request y)");
        SpmvBatch b;
        b.reqs = reqs;
        b.done = M->freeEvents.back();
        check_cuda(cudaEventRecord(b.done, st), "cudaEventRecord(batch)");
        M->freeEvents.pop_back();
        M->running.push_back(std::move(b));
        // without the doorbell the periodic sweep still completes the batch
        if (cudaLaunchHostFunc(st, doorbell, M) != cudaSuccess) cudaGetLastError();
    } catch (const Error &e) {
        cudaStreamSynchronize(st);  // nothing issued may still touch the request buffers
        complete(S, reqs, e.status, now_since(S->t0));
    }
}

// The SpMV scheduler: one thread issues every batch and completes it.  It
// sleeps until a request arrives or a doorbell rings; then it completes the
// batches whose events have fired (front of each rung matrix's queue, which
// its stream runs in order), and issues a new batch on every matrix with
// pending requests and fewer than maxInFlight batches running -- up to maxRhs
// requests, oldest first (with batching off, one).  Requests that arrive
// while their matrix's batch runs form its next batch (continuous batching);
// a request waits only for its own matrix.  No thread polls the GPU.
void scheduler(Server *S) {
    cudaSetDevice(S->device);
    const int32_t perBatch = S->opt.batching ? S->opt.maxRhs : 1;
    int64_t running = 0;  // batches in flight over all matrices
    std::vector<ServedMatrix *> rung;
    std::vector<std::pair<std::vector<Request *>, int>> finished;  // requests, status
    std::vector<std::pair<ServedMatrix *, std::vector<Request *>>> batches;
    for (;;) {
        bool sweep = false;
        rung.clear();
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto drained = [&] { return S->stop && S->spmvPending == 0 && running == 0; };
            auto ready = [&] {
                if (!S->rung.empty()) return true;
                if (S->spmvPending == 0 || (S->paused && !S->stop)) return false;  // stopping drains
                for (auto &m : S->mats)
                    if (!m->pending.empty() && static_cast<int32_t>(m->running.size()) < S->opt.maxInFlight)
                        return true;
                return false;
            };
            auto pred = [&] { return drained() || ready(); };
            if (running > 0) {
                if (!S->cvWork.wait_for(lk, std::chrono::milliseconds(kSweepMs), pred)) sweep = true;
            } else {
                S->cvWork.wait(lk, pred);
            }
            if (drained()) return;
            rung.swap(S->rung);
            if (sweep)
                for (auto &m : S->mats)
                    if (!m->running.empty()) rung.push_back(m.get());
        }
        // completions (CUDA queries outside the lock)
        finished.clear();
        auto retire = [&](ServedMatrix *M) {
            while (!M->running.empty()) {
                SpmvBatch &b = M->running.front();
                const cudaError_t q = cudaEventQuery(b.done);
                if (q == cudaErrorNotReady) break;
                finished.emplace_back(std::move(b.reqs), q == cudaSuccess ? HBDIA_OK : HBDIA_ERR_CUDA);
                M->freeEvents.push_back(b.done);
                M->running.pop_front();
                running -= 1;
            }
        };
        for (ServedMatrix *M : rung) retire(M);
        batches.clear();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            const double t = now_since(S->t0);
            for (auto &f : finished)
                for (Request *r : f.first) {
                    r->info.status = f.second;
                    r->info.finished = t;
                    r->done = true;
                    S->stats.completed += 1;
                }
            if (!(S->paused && !S->stop) && S->spmvPending > 0) {
                for (auto &m : S->mats) {
                    if (m->pending.empty() || static_cast<int32_t>(m->running.size()) >= S->opt.maxInFlight)
                        continue;
                    std::vector<Request *> b;
                    while (!m->pending.empty() && static_cast<int32_t>(b.size()) < perBatch) {
                        b.push_back(m->pending.front());
                        m->pending.pop_front();
                    }
                    S->spmvPending -= static_cast<int64_t>(b.size());
                    batches.emplace_back(m.get(), std::move(b));
                }
                if (!batches.empty()) {
                    S->stats.spmvSteps += 1;
                    S->stats.spmvLaunches += static_cast<int64_t>(batches.size());
                }
            }
        }
        if (!finished.empty()) S->cvDone.notify_all();
        for (auto &b : batches) {
            const size_t before = b.first->running.size();
            issue_batch(S, b.first, b.second);
            running += static_cast<int64_t>(b.first->running.size() - before);
        }
    }
}

// A CG worker takes the oldest CG request and the other pending CG requests
// on the same matrix (up to cgMaxGroup) and solves them as one lockstep
// group: one SpMM per iteration over all of them, each with its own
// workspace, schedule and result (bit-identical to solving it alone).
void cg_worker(Server *S) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    std::vector<CgWork *> ws;   // one workspace per group slot
    std::vector<double *> bx;   // per slot: b and x of host requests, cap each
    std::vector<int32_t> caps;
    const bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    const size_t maxGroup = static_cast<size_t>(S->opt.cgMaxGroup);
    for (;;) {
        std::vector<Request *> grp;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cvCg.wait(lk, [&] { return S->stop || (!S->paused && !S->cgQ.empty()); });
            if (S->cgQ.empty()) break;
            grp.push_back(S->cgQ.front());
            S->cgQ.pop_front();
            for (auto it = S->cgQ.begin(); it != S->cgQ.end() && grp.size() < maxGroup;) {
                if ((*it)->m == grp[0]->m) {
                    grp.push_back(*it);
                    it = S->cgQ.erase(it);
                } else {
                    ++it;
                }
            }
            S->stats.cgGroups += 1;
        }
        const double started = now_since(S->t0);
        const int32_t k = static_cast<int32_t>(grp.size());
        std::vector<int> status(grp.size(), HBDIA_OK);
        for (Request *r : grp) {
            r->info.started = started;
            r->info.batchRhs = k;
        }
        try {
            if (!ok) throw Error(HBDIA_ERR_CUDA, "CG worker stream");
            const ServedMatrix &M = *grp[0]->m;
            const size_t nb = sizeof(double) * static_cast<size_t>(M.n);
            if (ws.size() < grp.size()) {
                ws.resize(grp.size(), nullptr);
                bx.resize(grp.size(), nullptr);
                caps.resize(grp.size(), 0);
            }
            std::vector<CgCall> calls(grp.size());
            std::vector<CgStats> stats(grp.size());
            for (size_t i = 0; i < grp.size(); ++i) {
                Request *r = grp[i];
                ws[i] = cg_work(ws[i], M.n);
                if (!r->device && M.n > caps[i]) {
                    if (bx[i]) cudaFree(bx[i]);
                    bx[i] = nullptr;
                    caps[i] = 0;
                    check_cuda(dev_alloc(&bx[i], 2 * nb), "cudaMalloc(CG b, x)");
                    caps[i] = M.n;
                }
                // device requests solve in place: b = request x, solution into request y
                const double *b = r->device ? r->x : bx[i];
                double *x = r->device ? r->y : bx[i] + caps[i];
                if (!r->device)
                    check_cuda(cudaMemcpyAsync(bx[i], r->x, nb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(CG b)");
                check_cuda(cudaMemsetAsync(x, 0, nb, st), "cudaMemsetAsync(CG x)");
                calls[i] = CgCall{b, x, ws[i], &stats[i]};
            }
            const hbdia_server_options &o = S->opt;
            CgParams prm;
            prm.tol = o.cgTol;
            prm.updateFactor = o.cgUpdateFactor;
            prm.maxUpdates = o.cgMaxUpdates;
            prm.maxIterations = o.cgMaxIterations;
            prm.checkEvery = o.cgCheckEvery;
            cg_solve_group(M.p64, M.cgIter(o.cgIterStorage), calls.data(), k, prm, st);
            for (size_t i = 0; i < grp.size(); ++i) {
                Request *r = grp[i];
                if (!r->device)
                    check_cuda(cudaMemcpyAsync(r->y, calls[i].x, nb, cudaMemcpyDeviceToHost, st),
                               "cudaMemcpyAsync(CG y)");
                r->info.cgUpdates = stats[i].updates;
                r->info.cgIterations = stats[i].iterations;
                r->info.cgRelResidual = stats[i].relResidual;
                if (stats[i].relResidual > o.cgTol) status[i] = HBDIA_ERR_RUNTIME;  // not converged
            }
            check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize(CG)");
        } catch (const Error &e) {
            cudaStreamSynchronize(st);  // nothing issued may still touch the request buffers
            std::fill(status.begin(), status.end(), e.status);
        } catch (const std::exception &) {
            cudaStreamSynchronize(st);
            std::fill(status.begin(), status.end(), static_cast<int>(HBDIA_ERR_RUNTIME));
        }
        const double finished = now_since(S->t0);
        for (size_t i = 0; i < grp.size(); ++i) complete(S, {grp[i]}, status[i], finished);
    }
    for (CgWork *w : ws) cg_free(w);
    for (double *p : bx)
        if (p) cudaFree(p);
    if (st) cudaStreamDestroy(st);
}

void free_matrix(ServedMatrix &M) {
    free_plan(M.p64);
    free_plan(M.pLow);
    free_plan(M.pCg);
    if (M.X) cudaFree(M.X);
    if (M.Y) cudaFree(M.Y);
    if (M.stream) cudaStreamDestroy(M.stream);
    for (cudaEvent_t e : M.freeEvents) cudaEventDestroy(e);
    M.freeEvents.clear();
    M.X = M.Y = nullptr;
    M.stream = nullptr;
}

}  // namespace

void server_default_options(hbdia_server_options *o) {
    std::memset(o, 0, sizeof(*o));
    o->memoryBudget = 150LL * 1000 * 1000 * 1000;
    o->batching = 1;
    o->maxRhs = 16;
    o->spmvStorage = HBDIA_STORE_F32;
    o->cgIterStorage = HBDIA_STORE_F32_QUAD;  // the fastest CG iterations measured on B200
    o->cgWorkers = 4;
    o->cgTol = 1e-10;
    o->cgUpdateFactor = 0.1;
    o->cgMaxUpdates = 100;
    o->cgMaxIterations = 20000;
    o->cgCheckEvery = 10;
    o->cgMaxGroup = 1;
    o->maxInFlight = 1;
}

Server *server_create(const hbdia_server_options &o) {
    if (o.memoryBudget <= 0 || o.maxRhs < 1 || o.maxRhs > 64 || o.cgWorkers < 1 || o.cgWorkers > 64 ||
        o.cgTol <= 0 || o.cgUpdateFactor <= 0 || o.cgUpdateFactor >= 1 || o.cgMaxUpdates < 1 ||
        o.cgMaxIterations < 1 || o.cgCheckEvery < 1 || o.cgMaxGroup < 1 || o.cgMaxGroup > 16 ||
        o.maxInFlight < 1 || o.maxInFlight > 8)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad server options");
    if (o.spmvStorage != HBDIA_STORE_NATIVE && o.spmvStorage != HBDIA_STORE_F32 &&
        o.spmvStorage != HBDIA_STORE_BF16_SCALED)  // SpMV batches are SpMMs: no quad-interleaved storage
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown or unsupported SpMV value storage");
    if (o.cgIterStorage < HBDIA_STORE_NATIVE || o.cgIterStorage > HBDIA_STORE_BF16_QUAD)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown CG iteration value storage");
    auto S = std::make_unique<Server>();
    S->opt = o;
    check_cuda(cudaGetDevice(&S->device), "cudaGetDevice");
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
    // a doorbell may still be queued behind the last batch's event: let it run
    // before its matrix goes
    for (auto &m : S->mats)
        if (m->stream) cudaStreamSynchronize(m->stream);
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
    const int32_t sp = S->opt.spmvStorage, cgs = iteration_storage(L, S->opt.cgIterStorage);
    try {
        build_plan(L, HBDIA_STORE_NATIVE, M->p64);
        if (sp != HBDIA_STORE_NATIVE) build_plan(L, sp, M->pLow);
        if (cgs != HBDIA_STORE_NATIVE && cgs != sp) build_plan(L, cgs, M->pCg);
        const int64_t staging =
            static_cast<int64_t>(S->opt.maxRhs) * (static_cast<int64_t>(M->rowsX) + M->n) * 8;
        // CG workspaces grow to the largest system: 3 vectors of the workspace + b, x per
        // group slot of every worker
        int64_t cgGrow = 0;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (M->n > S->maxN)
                cgGrow = static_cast<int64_t>(S->opt.cgWorkers) * S->opt.cgMaxGroup * 5 * 8 * (M->n - S->maxN);
        }
        M->bytes = static_cast<int64_t>(M->p64.bytes + M->pLow.bytes + M->pCg.bytes) + staging;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->used + M->bytes + cgGrow > S->opt.memoryBudget)
                throw Error(HBDIA_ERR_NO_MEMORY,
                            "admission refused: the matrix needs " + std::to_string(M->bytes + cgGrow) +
                                " device bytes and the server holds " + std::to_string(S->used) + " of its " +
                                std::to_string(S->opt.memoryBudget) + "-byte budget");
        }
        check_cuda(dev_alloc(&M->X, sizeof(double) * static_cast<size_t>(S->opt.maxRhs) * M->rowsX),
                   "cudaMalloc(server staging x)");
        check_cuda(dev_alloc(&M->Y, sizeof(double) * static_cast<size_t>(S->opt.maxRhs) * M->n),
                   "cudaMalloc(server staging y)");
        check_cuda(cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking), "cudaStreamCreate(server)");
        for (int32_t i = 0; i < S->opt.maxInFlight; ++i) {
            cudaEvent_t e = nullptr;
            check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(server)");
            M->freeEvents.push_back(e);
        }
        M->server = S;
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
        S->mats[matrix]->pending.push_back(raw);
        S->spmvPending += 1;
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
