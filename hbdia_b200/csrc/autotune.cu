// Autotuner for a matrix's SpMV (k == 1) and SpMM (k > 1) launches.
//
// Every candidate configuration computes bit-identical results, so the tuner
// only compares speed: it times each candidate with CUDA events on the
// caller's own buffers and stream and keeps the fastest in the matrix's plan.
// A process-wide table keyed on the matrix's shape class -- block width,
// stored offsets per block, COO fraction, number of right-hand sides, value
// type and storage -- lets later matrices of the same class take the choice
// without timing.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "hbdia_internal.hpp"

namespace hbdia {
namespace {

using Key = std::tuple<int32_t, int32_t, int32_t, int32_t, int32_t, int32_t>;

struct Choice {
    int32_t kernel = HBDIA_KERNEL_AUTO;
    int32_t unroll = 0;
    int32_t tile = 0;
    float ms = 0.f;
};

std::mutex g_mu;
std::map<Key, Choice> g_table;

int32_t k_bucket(int32_t k) {
    int32_t b = 1;
    while (b < k) b <<= 1;
    return b;
}

Key key_of(const DevicePlan &P, int32_t k) {
    const int32_t offsPerBlock =
        P.numBlocks > 0 ? static_cast<int32_t>(std::lround(double(P.totalOffsets) / P.numBlocks)) : 0;
    const double cooFrac = P.slots + P.nCoo > 0 ? double(P.nCoo) / double(P.slots + P.nCoo) : 0.0;
    // COO fraction bucket: 0, (0, 0.1%], (0.1%, 1%], (1%, 10%], > 10%
    const int32_t cooBucket = cooFrac == 0 ? 0 : cooFrac <= 1e-3 ? 1 : cooFrac <= 1e-2 ? 2 : cooFrac <= 0.1 ? 3 : 4;
    return Key(P.bw, offsPerBlock, cooBucket, k_bucket(k), P.dtype, P.storage);
}

void apply(DevicePlan &P, int32_t k, const Choice &c) {
    if (k == 1) {
        P.kernel = c.kernel;
        P.unroll = c.unroll;
    } else {
        P.spmmTile[k] = c.tile;
    }
}

float time_launch(DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k, const Choice &c,
                  cudaStream_t s) {
    apply(P, k, c);
    auto run = [&] {
        if (k == 1) launch_spmv(P, X, Y, s);
        else launch_spmm_tile(P, X, ldx, Y, ldy, k, c.tile, s);
    };
    run();
    run();
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    const int reps = 5;
    check_cuda(cudaEventRecord(e0, s), "cudaEventRecord");
    for (int r = 0; r < reps; ++r) run();
    check_cuda(cudaEventRecord(e1, s), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.f;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

}  // namespace

// Returns the chosen configuration; fromCache = 1 when taken from the table.
void autotune(DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k, void *stream, bool force,
              int32_t *kernel, int32_t *unroll, int32_t *tile, int32_t *fromCache, float *ms) {
    if (!P.base) throw Error(HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
    if (k <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "k must be positive");
    const Key key = key_of(P, k);
    Choice best;
    bool cached = false;
    if (!force) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_table.find(key);
        if (it != g_table.end()) {
            best = it->second;
            cached = true;
        }
    }
    if (!cached) {
        cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : P.stream);
        std::vector<Choice> cand;
        if (k == 1) {
            if (P.bw == 32) {
                for (int32_t kern : {HBDIA_KERNEL_PIPE, HBDIA_KERNEL_QUAD, HBDIA_KERNEL_WARP, HBDIA_KERNEL_STAGED})
                    for (int32_t u : {0, 27}) {
                        if (kern != HBDIA_KERNEL_PIPE && u) continue;  // unroll is the pipelined kernel's knob
                        Choice c;
                        c.kernel = kern;
                        c.unroll = u;
                        cand.push_back(c);
                    }
            } else {
                Choice c;
                c.kernel = HBDIA_KERNEL_ROWWISE;
                cand.push_back(c);
            }
        } else {
            for (int32_t t : {2, 4, 8, 16, 32}) {
                if (t > 4 && t / 2 >= k) break;  // a tile twice as wide as k only adds idle work
                Choice c;
                c.tile = t;
                cand.push_back(c);
            }
        }
        const int32_t keepKernel = P.kernel, keepUnroll = P.unroll;
        float bestMs = INFINITY;
        try {
            for (const Choice &c : cand) {
                if (k == 1 && select_kernel([&] {
                        DevicePlan Q = P;  // would this candidate actually run as itself?
                        Q.kernel = c.kernel;
                        return Q;
                    }(), X) != c.kernel)
                    continue;
                const float t = time_launch(P, X, ldx, Y, ldy, k, c, s);
                if (t < bestMs) {
                    bestMs = t;
                    best = c;
                    best.ms = t;
                }
            }
        } catch (...) {
            P.kernel = keepKernel;
            P.unroll = keepUnroll;
            throw;
        }
        if (!std::isfinite(bestMs)) {  // nothing eligible: keep the defaults
            best.kernel = keepKernel;
            best.unroll = keepUnroll;
            best.tile = default_spmm_tile(k);
        }
        std::lock_guard<std::mutex> lk(g_mu);
        g_table[key] = best;
    }
    apply(P, k, best);
    if (kernel) *kernel = best.kernel;
    if (unroll) *unroll = best.unroll;
    if (tile) *tile = best.tile;
    if (fromCache) *fromCache = cached ? 1 : 0;
    if (ms) *ms = best.ms;
}

void autotune_clear_cache() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
}

}  // namespace hbdia
