// COO -> device HBDIA layout on the GPU (row-sorted COO), the same layout as
// convertToHBDIAFormat (src/Format/HBDIA.cpp:507-718) followed by
// prepareForGPU, without materialising the host layout.
//
//   1. rowStart[r] = first entry of row r (binary search in the sorted rows);
//      block b's entries are rowStart[b*bw] .. rowStart[(b+1)*bw].
//   2. per block (one CTA): its offsets sorted in shared memory (bitonic),
//      run-length encoded into the ascending distinct (offset, count) list --
//      what the reference's std::map<int,int> per block holds; blocks with
//      more entries than the shared array holds extract the distinct offsets
//      one by one with block-wide minima.
//   3. the keep/drop filter (HBDIA.cpp:567-586): an offset is kept when its
//      count reaches the threshold, or once the running count of dropped
//      entries has reached max_coo_entries.  The running count is a prefix
//      sum over the dropped candidates in block / offset order, so a
//      candidate is dropped exactly when the candidates before it sum to
//      less than max_coo_entries -- a scan, not a sequential loop.
//   4. kept counts -> blockStart (scan), kept offsets compacted per block.
//   5. fill, one thread per row walking its entries in input order: a kept
//      entry is ASSIGNED to its slot (so duplicates are last-wins, as in the
//      reference), the others are counted, then (second pass) written to the
//      COO remainder at the row's scanned position -- input order, since the
//      input is row-sorted.  The scanned per-row counts are the COO remainder's
//      CSR row pointer.
//   6. histograms (HBDIA.cpp:619-631) and numberDiagonals (distinct offsets
//      over all blocks) with atomics.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>
#include <vector>

#include "hbdia_internal.hpp"

namespace hbdia {

namespace {

constexpr int kSortCap = 4096;  // block entries sorted in shared memory
constexpr int kCtaThreads = 256;

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Device scratch owned by one conversion.
struct Scratch {
    std::vector<void *> ptrs;
    template <typename T>
    T *get(size_t count) {
        void *p = nullptr;
        check_cuda(dev_alloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc(converter scratch)");
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Scratch() {
        for (void *p : ptrs) cudaFree(p);
    }
};

template <typename In, typename Out>
void exclusive_scan(const In *in, Out *out, int64_t n, Scratch &S) {
    size_t bytes = 0;
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n), "cub scan (size)");
    void *tmp = S.get<char>(bytes);
    check_cuda(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n), "cub scan");
}

template <typename T>
T device_sum(const T *in, int64_t n, Scratch &S) {
    T *d = S.get<T>(1);
    size_t bytes = 0;
    check_cuda(cub::DeviceReduce::Sum(nullptr, bytes, in, d, n), "cub reduce (size)");
    void *tmp = S.get<char>(bytes);
    check_cuda(cub::DeviceReduce::Sum(tmp, bytes, in, d, n), "cub reduce");
    T h{};
    check_cuda(cudaMemcpy(&h, d, sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy(sum)");
    return h;
}

// ---------------------------------------------------------------- kernels
// Bit 0: rows not sorted; bit 1: an index outside the matrix.
__global__ void validate_coo(const int32_t *__restrict__ R, const int32_t *__restrict__ C, int64_t nnz, int32_t nR,
                             int32_t nC, int32_t *__restrict__ flags) {
    int32_t f = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t r = R[i], c = C[i];
        if (r < 0 || r >= nR || c < 0 || c >= nC) f |= 2;
        if (i > 0 && R[i - 1] > r) f |= 1;
    }
    if (f) atomicOr(flags, f);
}

__global__ void row_starts(const int32_t *__restrict__ R, int64_t nnz, int32_t nR, int64_t *__restrict__ rs) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r > nR) return;
    int64_t lo = 0, hi = nnz;  // first entry with row >= r
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(R + mid) < r) lo = mid + 1;
        else hi = mid;
    }
    rs[r] = lo;
}

__device__ __forceinline__ int64_t block_begin(const int64_t *rs, int32_t b, int32_t bw, int32_t nR) {
    return rs[min(static_cast<int64_t>(b) * bw, static_cast<int64_t>(nR))];
}

// Block-wide sum / min of one value per thread (kCtaThreads threads).
template <typename T, typename Op>
__device__ __forceinline__ T cta_reduce(T v, T *red, Op op) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    T t = red[0];
    for (int i = 1; i < kCtaThreads / 32; ++i) t = op(t, red[i]);
    return t;
}

// Step 2: distinct (offset, count) per block, written at the block's own
// entry range (uoff/ucnt[begin ..]); also the block's dropped-candidate sum.
__global__ void __launch_bounds__(kCtaThreads)
block_distinct(const int32_t *__restrict__ R, const int32_t *__restrict__ C, const int64_t *__restrict__ rs,
               int32_t bw, int32_t nR, int32_t thr, int32_t *__restrict__ uoff, int32_t *__restrict__ ucnt,
               int32_t *__restrict__ ndist, int64_t *__restrict__ candSum) {
    __shared__ int32_t s[kSortCap];
    __shared__ int32_t pos[kSortCap + 1];
    __shared__ int64_t red64[kCtaThreads / 32];
    __shared__ int32_t red32[kCtaThreads / 32];
    __shared__ int32_t nd;
    const int32_t b = blockIdx.x;
    const int64_t e0 = block_begin(rs, b, bw, nR), e1 = block_begin(rs, b + 1, bw, nR);
    const int64_t m = e1 - e0;
    int64_t cand = 0;
    if (m <= kSortCap) {
        int p2 = 1;
        while (p2 < m) p2 <<= 1;
        for (int i = threadIdx.x; i < p2; i += kCtaThreads)
            s[i] = i < m ? __ldg(C + e0 + i) - __ldg(R + e0 + i) : INT_MAX;
        __syncthreads();
        for (int k = 2; k <= p2; k <<= 1)  // bitonic sort, ascending
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < p2; i += kCtaThreads) {
                    const int l = i ^ j;
                    if (l > i) {
                        const bool up = (i & k) == 0;
                        const int32_t a = s[i], c = s[l];
                        if ((a > c) == up) {
                            s[i] = c;
                            s[l] = a;
                        }
                    }
                }
                __syncthreads();
            }
        // starts of runs, in order (thread 0 walks: m is at most kSortCap)
        if (threadIdx.x == 0) {
            int32_t n = 0;
            for (int i = 0; i < m; ++i)
                if (i == 0 || s[i] != s[i - 1]) pos[n++] = i;
            pos[n] = static_cast<int32_t>(m);
            nd = n;
        }
        __syncthreads();
        for (int u = threadIdx.x; u < nd; u += kCtaThreads) {
            const int32_t c = pos[u + 1] - pos[u];
            uoff[e0 + u] = s[pos[u]];
            ucnt[e0 + u] = c;
            if (c < thr) cand += c;
        }
    } else {
        // many entries: extract the distinct offsets in ascending order
        int64_t prev = static_cast<int64_t>(INT_MIN) - 1;
        int32_t n = 0;
        for (;;) {
            int32_t mine = INT_MAX;
            bool any = false;
            for (int64_t i = e0 + threadIdx.x; i < e1; i += kCtaThreads) {
                const int32_t o = __ldg(C + i) - __ldg(R + i);
                if (o > prev && o <= mine) {
                    mine = o;
                    any = true;
                }
            }
            const int32_t anyAll = cta_reduce<int32_t>(any ? 1 : 0, red32, [](int32_t a, int32_t c) { return a + c; });
            if (!anyAll) break;
            const int32_t lo = cta_reduce<int32_t>(mine, red32, [](int32_t a, int32_t c) { return min(a, c); });
            int32_t cnt = 0;
            for (int64_t i = e0 + threadIdx.x; i < e1; i += kCtaThreads)
                cnt += (__ldg(C + i) - __ldg(R + i)) == lo;
            cnt = cta_reduce<int32_t>(cnt, red32, [](int32_t a, int32_t c) { return a + c; });
            if (threadIdx.x == 0) {
                uoff[e0 + n] = lo;
                ucnt[e0 + n] = cnt;
                if (cnt < thr) cand += cnt;
            }
            ++n;
            prev = lo;
        }
        if (threadIdx.x == 0) nd = n;
        __syncthreads();
    }
    const int64_t total = cta_reduce<int64_t>(cand, red64, [](int64_t a, int64_t c) { return a + c; });
    if (threadIdx.x == 0) {
        ndist[b] = nd;
        candSum[b] = total;
    }
}

// Steps 3-4: keep flags (written over ucnt's sign: kept counts stay
// positive, dropped ones are negated), kept count and kept-entry count per
// block.  candBase: exclusive scan of candSum (binding max_coo only).
__global__ void __launch_bounds__(kCtaThreads)
block_keep(const int64_t *__restrict__ rs, int32_t bw, int32_t nR, int32_t thr, int64_t maxCoo, bool binding,
           const int64_t *__restrict__ candBase, const int32_t *__restrict__ ndist, int32_t *__restrict__ ucnt,
           const int32_t *__restrict__ uoff, uint64_t *__restrict__ diagBits, int32_t nRm1,
           int64_t *__restrict__ keptOffs, int64_t *__restrict__ keptEntries) {
    const int32_t b = blockIdx.x;
    if (threadIdx.x != 0) return;
    const int64_t e0 = block_begin(rs, b, bw, nR);
    const int32_t nd = ndist[b];
    int64_t run = binding ? candBase[b] : 0;
    int64_t ko = 0, ke = 0;
    for (int32_t u = 0; u < nd; ++u) {
        const int32_t c = ucnt[e0 + u];
        const int64_t k = static_cast<int64_t>(uoff[e0 + u]) + nRm1;
        atomicOr(reinterpret_cast<unsigned long long *>(diagBits + (k >> 6)), 1ull << (k & 63));
        bool keep = c >= thr;
        if (!keep) {
            if (binding && run >= maxCoo) keep = true;
            else run += c;
        }
        if (keep) {
            ++ko;
            ke += c;
        } else {
            ucnt[e0 + u] = -c;
        }
    }
    keptOffs[b] = ko;
    keptEntries[b] = ke;
}

__global__ void __launch_bounds__(kCtaThreads)
block_offsets(const int64_t *__restrict__ rs, int32_t bw, int32_t nR, const int32_t *__restrict__ ndist,
              const int32_t *__restrict__ uoff, const int32_t *__restrict__ ucnt, const int64_t *__restrict__ kstart,
              const int64_t *__restrict__ keptOffs, const int64_t *__restrict__ keptEntries, int32_t *__restrict__ offs,
              int32_t *__restrict__ blkOff, int32_t *__restrict__ histBlocks, int32_t *__restrict__ histNnz) {
    const int32_t b = blockIdx.x;
    if (threadIdx.x != 0) return;
    const int64_t e0 = block_begin(rs, b, bw, nR);
    int64_t p = kstart[b];
    blkOff[b] = static_cast<int32_t>(p);
    for (int32_t u = 0; u < ndist[b]; ++u)
        if (ucnt[e0 + u] > 0) offs[p++] = uoff[e0 + u];
    atomicAdd(histBlocks + keptOffs[b], 1);
    atomicAdd(histNnz + keptOffs[b], static_cast<int32_t>(keptEntries[b]));
}

// Step 5: one thread per row.  pass 0: assign kept entries (in order:
// last-wins) and count the row's COO entries; pass 1: write them.
template <typename T>
__global__ void row_fill(const int32_t *__restrict__ R, const int32_t *__restrict__ C, const T *__restrict__ V,
                         const int64_t *__restrict__ rs, int32_t nR, int32_t bw, int32_t nb,
                         const int32_t *__restrict__ offs, const int32_t *__restrict__ blkOff, T *__restrict__ D,
                         int pass, int32_t *__restrict__ rowCoo, const int32_t *__restrict__ cooRowPtr,
                         int32_t *__restrict__ cr, int32_t *__restrict__ cc, T *__restrict__ cv) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= nR) return;
    const int32_t b = static_cast<int32_t>(r / bw);
    const int32_t lane = static_cast<int32_t>(r - static_cast<int64_t>(b) * bw);
    int32_t k0 = 0, nk = 0;
    if (b < nb) {
        k0 = __ldg(blkOff + b);
        nk = __ldg(blkOff + b + 1) - k0;
    }
    int64_t out = pass ? __ldg(cooRowPtr + r) : 0;
    int32_t ncoo = 0;
    for (int64_t i = rs[r]; i < rs[r + 1]; ++i) {
        const int32_t off = __ldg(C + i) - __ldg(R + i);
        int32_t lo = 0, hi = nk;  // kept offsets of the block are ascending
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (__ldg(offs + k0 + mid) < off) lo = mid + 1;
            else hi = mid;
        }
        if (lo < nk && __ldg(offs + k0 + lo) == off) {
            if (pass == 0) D[(static_cast<int64_t>(k0) + lo) * bw + lane] = V[i];
        } else if (pass == 0) {
            ++ncoo;
        } else {
            cr[out] = static_cast<int32_t>(r);
            cc[out] = __ldg(C + i);
            cv[out] = V[i];
            ++out;
        }
    }
    if (pass == 0) rowCoo[r] = ncoo;
}

__global__ void tiles_from_rows(const int32_t *__restrict__ crp, int32_t n, int32_t numTiles, int32_t *__restrict__ tile) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > numTiles) return;
    tile[t] = crp[min(t * 32, static_cast<int64_t>(n))];
}

__global__ void popcount_words(const uint64_t *__restrict__ w, int64_t n, int64_t *__restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __popcll(w[i]);
}

// Reduced value storage from the FP64 slots (the host builder's rounding).
__global__ void to_f32(const double *__restrict__ in, float *__restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __double2float_rn(in[i]);
}

__global__ void __launch_bounds__(kCtaThreads)
to_bf16_scaled(const double *__restrict__ in, const int32_t *__restrict__ blkOff, int32_t bw,
               __nv_bfloat16 *__restrict__ out, float *__restrict__ scale) {
    __shared__ double red[kCtaThreads / 32];
    const int32_t b = blockIdx.x;
    const int64_t s0 = static_cast<int64_t>(blkOff[b]) * bw, s1 = static_cast<int64_t>(blkOff[b + 1]) * bw;
    double mx = 0.0;
    for (int64_t i = s0 + threadIdx.x; i < s1; i += kCtaThreads) mx = fmax(mx, fabs(in[i]));
    mx = cta_reduce<double>(mx, red, [](double a, double c) { return fmax(a, c); });
    const float sc = mx > 0.0 ? __double2float_rn(mx) : 1.0f;
    if (threadIdx.x == 0) scale[b] = sc;
    for (int64_t i = s0 + threadIdx.x; i < s1; i += kCtaThreads)
        out[i] = __float2bfloat16_rn(__double2float_rn(__ddiv_rn(in[i], static_cast<double>(sc))));
}

unsigned blocks_for(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

template <typename T>
void convert_on_device(const Coo<T> &coo, int32_t bw, int32_t thr, int64_t maxCoo, int storage, DevicePlan &P,
                       DeviceLayoutMeta &meta) {
    if (bw <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "blockWidth must be positive");
    const int64_t nnz = static_cast<int64_t>(coo.vals.size());
    const int32_t nR = coo.numRows, nC = coo.numCols;
    if (nR <= 0 || nC <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "empty matrix");
    if (nnz > INT32_MAX) throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^31-1 entries");
    const int dtype = std::is_same<T, float>::value ? HBDIA_F32 : HBDIA_F64;
    if (storage != HBDIA_STORE_NATIVE && dtype != HBDIA_F64)
        throw Error(HBDIA_ERR_UNSUPPORTED, "reduced value storage needs a double matrix");
    if (storage < HBDIA_STORE_NATIVE || storage > HBDIA_STORE_BF16_SCALED)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown value storage");
    const int32_t nb = static_cast<int32_t>((static_cast<int64_t>(std::min(nR, nC)) + bw - 1) / bw);

    Scratch S;
    int32_t *R = S.get<int32_t>(nnz), *C = S.get<int32_t>(nnz);
    T *V = S.get<T>(nnz);
    check_cuda(cudaMemcpy(R, coo.rows.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice), "cudaMemcpy(rows)");
    check_cuda(cudaMemcpy(C, coo.cols.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice), "cudaMemcpy(cols)");
    check_cuda(cudaMemcpy(V, coo.vals.data(), sizeof(T) * nnz, cudaMemcpyHostToDevice), "cudaMemcpy(vals)");
    {
        int32_t *flags = S.get<int32_t>(1);
        check_cuda(cudaMemset(flags, 0, sizeof(int32_t)), "cudaMemset(flags)");
        validate_coo<<<1184, 256>>>(R, C, nnz, nR, nC, flags);
        int32_t f = 0;
        check_cuda(cudaMemcpy(&f, flags, sizeof(int32_t), cudaMemcpyDeviceToHost), "cudaMemcpy(flags)");
        if (f & 2) throw Error(HBDIA_ERR_OUT_OF_RANGE, "entry outside the matrix");
        if (f & 1) throw Error(HBDIA_ERR_UNSUPPORTED, "the device converter needs row-sorted COO input");
    }

    // 1. row starts
    int64_t *rs = S.get<int64_t>(static_cast<size_t>(nR) + 1);
    row_starts<<<blocks_for(static_cast<int64_t>(nR) + 1), 256>>>(R, nnz, nR, rs);
    check_cuda(cudaGetLastError(), "row_starts");
    int64_t inBlocks = 0;
    check_cuda(cudaMemcpy(&inBlocks, rs + std::min<int64_t>(static_cast<int64_t>(nb) * bw, nR), sizeof(int64_t),
                          cudaMemcpyDeviceToHost), "cudaMemcpy(inBlocks)");

    // 2. distinct offsets per block
    int32_t *uoff = S.get<int32_t>(inBlocks), *ucnt = S.get<int32_t>(inBlocks);
    int32_t *ndist = S.get<int32_t>(nb);
    int64_t *candSum = S.get<int64_t>(nb), *candBase = S.get<int64_t>(nb);
    if (nb > 0) {
        block_distinct<<<nb, kCtaThreads>>>(R, C, rs, bw, nR, thr, uoff, ucnt, ndist, candSum);
        check_cuda(cudaGetLastError(), "block_distinct");
    }
    // 3. filter
    const int64_t candidates = nb > 0 ? device_sum(candSum, nb, S) : 0;
    const bool binding = candidates > maxCoo;
    if (binding) exclusive_scan(candSum, candBase, nb, S);
    const int64_t span = static_cast<int64_t>(nR) + nC;
    const int64_t words = (span + 63) / 64;
    uint64_t *diagBits = S.get<uint64_t>(words);
    check_cuda(cudaMemset(diagBits, 0, sizeof(uint64_t) * words), "cudaMemset(diagonal bits)");
    int64_t *keptOffs = S.get<int64_t>(nb), *keptEntries = S.get<int64_t>(nb);
    int64_t *kstart = S.get<int64_t>(static_cast<size_t>(nb) + 1);
    if (nb > 0) {
        block_keep<<<nb, 32>>>(rs, bw, nR, thr, maxCoo, binding, candBase, ndist, ucnt, uoff, diagBits, nR - 1,
                               keptOffs, keptEntries);
        check_cuda(cudaGetLastError(), "block_keep");
    }
    {
        int64_t *pc = S.get<int64_t>(words);
        popcount_words<<<blocks_for(words), 256>>>(diagBits, words, pc);
        meta.numberDiagonals = static_cast<int32_t>(device_sum(pc, words, S));
    }
    // 4. kept offsets, flattened
    int64_t totalOffsets = 0, kept = 0;
    if (nb > 0) {
        exclusive_scan(keptOffs, kstart, nb, S);
        int64_t last = 0, lastStart = 0;
        check_cuda(cudaMemcpy(&last, keptOffs + nb - 1, sizeof(int64_t), cudaMemcpyDeviceToHost), "cudaMemcpy");
        check_cuda(cudaMemcpy(&lastStart, kstart + nb - 1, sizeof(int64_t), cudaMemcpyDeviceToHost), "cudaMemcpy");
        totalOffsets = lastStart + last;
        kept = device_sum(keptEntries, nb, S);
    }
    const int64_t slots = totalOffsets * bw;
    if (static_cast<double>(slots) > 1e11)
        throw Error(HBDIA_ERR_RUNTIME, "Excessive memory requirement for HBDIA format");
    if (totalOffsets > INT32_MAX) throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^31-1 stored offsets");
    const int64_t nCoo = nnz - kept;
    int32_t maxd = 0;
    {
        // the largest kept count per block bounds the histograms
        std::vector<int64_t> ko(static_cast<size_t>(nb));
        if (nb > 0)
            check_cuda(cudaMemcpy(ko.data(), keptOffs, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
        for (int64_t v : ko) maxd = std::max<int32_t>(maxd, static_cast<int32_t>(v));
    }

    // the plan's one allocation (build_plan's layout, no staged schedule)
    DevicePlan Q;
    Q.kernel = P.kernel;
    Q.waitTimeoutNs = P.waitTimeoutNs;
    Q.skipTile = P.skipTile;
    Q.xsConfig = P.xsConfig;
    Q.quadGroup = P.quadGroup;
    Q.unroll = P.unroll;
    free_plan(P);
    Q.dtype = dtype;
    Q.storage = storage;
    Q.n = nR;
    Q.xn = nR;
    Q.numCols = nC;
    Q.bw = bw;
    Q.numBlocks = nb;
    Q.numTiles = static_cast<int32_t>((static_cast<int64_t>(nR) + 31) / 32);
    Q.totalOffsets = totalOffsets;
    Q.slots = slots;
    Q.nCoo = nCoo;
    const size_t vsz = storage == HBDIA_STORE_F32 ? 4 : storage == HBDIA_STORE_BF16_SCALED ? 2 : sizeof(T);
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += align256(bytes);
        return o;
    };
    const size_t oVals = carve(slots * vsz);
    const size_t oScale = carve(storage == HBDIA_STORE_BF16_SCALED ? nb * sizeof(float) : 0);
    const size_t oOffs = carve(totalOffsets * sizeof(int32_t));
    const size_t oBlk = carve((static_cast<size_t>(nb) + 1) * sizeof(int32_t));
    const size_t oCR = carve(nCoo * sizeof(int32_t));
    const size_t oCC = carve(nCoo * sizeof(int32_t));
    const size_t oCV = carve(nCoo * sizeof(T));
    const size_t oRP = carve((static_cast<size_t>(nR) + 1) * sizeof(int32_t));
    const size_t oTile = carve((static_cast<size_t>(Q.numTiles) + 1) * sizeof(int32_t));
    const size_t oStatus = carve(sizeof(int32_t));
    Q.bytes = off;
    check_cuda(dev_alloc(&Q.base, Q.bytes), "cudaMalloc(matrix layout)");
    try {
        char *base = static_cast<char *>(Q.base);
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

        // offsets, block starts, histograms
        int32_t *histB = S.get<int32_t>(static_cast<size_t>(maxd) + 1);
        int32_t *histN = S.get<int32_t>(static_cast<size_t>(maxd) + 1);
        check_cuda(cudaMemset(histB, 0, sizeof(int32_t) * (maxd + 1)), "cudaMemset");
        check_cuda(cudaMemset(histN, 0, sizeof(int32_t) * (maxd + 1)), "cudaMemset");
        if (nb > 0) {
            block_offsets<<<nb, 32>>>(rs, bw, nR, ndist, uoff, ucnt, kstart, keptOffs, keptEntries, Q.offs,
                                      Q.blkOff, histB, histN);
            check_cuda(cudaGetLastError(), "block_offsets");
        }
        const int32_t tot32 = static_cast<int32_t>(totalOffsets);
        check_cuda(cudaMemcpy(Q.blkOff + nb, &tot32, sizeof(int32_t), cudaMemcpyHostToDevice), "cudaMemcpy");
        meta.histBlocks.assign(static_cast<size_t>(maxd) + 1, 0);
        meta.histNnz.assign(static_cast<size_t>(maxd) + 1, 0);
        check_cuda(cudaMemcpy(meta.histBlocks.data(), histB, sizeof(int32_t) * (maxd + 1), cudaMemcpyDeviceToHost),
                   "cudaMemcpy(histogram)");
        check_cuda(cudaMemcpy(meta.histNnz.data(), histN, sizeof(int32_t) * (maxd + 1), cudaMemcpyDeviceToHost),
                   "cudaMemcpy(histogram)");

        // 5. fill: FP64 (native) slots, zero-padded
        T *D = storage == HBDIA_STORE_NATIVE ? static_cast<T *>(Q.vals) : S.get<T>(slots);
        check_cuda(cudaMemset(D, 0, sizeof(T) * slots), "cudaMemset(values)");
        int32_t *rowCoo = S.get<int32_t>(static_cast<size_t>(nR) + 1);
        row_fill<T><<<blocks_for(nR), 256>>>(R, C, V, rs, nR, bw, nb, Q.offs, Q.blkOff, D, 0, rowCoo, nullptr,
                                             nullptr, nullptr, nullptr);
        check_cuda(cudaGetLastError(), "row_fill");
        check_cuda(cudaMemset(rowCoo + nR, 0, sizeof(int32_t)), "cudaMemset");
        exclusive_scan(rowCoo, Q.cooRowPtr, static_cast<int64_t>(nR) + 1, S);
        row_fill<T><<<blocks_for(nR), 256>>>(R, C, V, rs, nR, bw, nb, Q.offs, Q.blkOff, D, 1, nullptr, Q.cooRowPtr,
                                             Q.cooRow, Q.cooCol, static_cast<T *>(Q.cooVal));
        check_cuda(cudaGetLastError(), "row_fill");
        tiles_from_rows<<<blocks_for(static_cast<int64_t>(Q.numTiles) + 1), 256>>>(Q.cooRowPtr, nR, Q.numTiles,
                                                                                  Q.cooTile);
        check_cuda(cudaGetLastError(), "tiles_from_rows");
        if (storage == HBDIA_STORE_F32) {
            to_f32<<<blocks_for(slots), 256>>>(reinterpret_cast<const double *>(D), static_cast<float *>(Q.vals), slots);
        } else if (storage == HBDIA_STORE_BF16_SCALED && nb > 0) {
            to_bf16_scaled<<<nb, kCtaThreads>>>(reinterpret_cast<const double *>(D), Q.blkOff, bw,
                                                static_cast<__nv_bfloat16 *>(Q.vals), Q.scale);
        }
        check_cuda(cudaGetLastError(), "value storage");
        int32_t nCooCheck = 0;
        check_cuda(cudaMemcpy(&nCooCheck, Q.cooRowPtr + nR, sizeof(int32_t), cudaMemcpyDeviceToHost), "cudaMemcpy");
        if (nCooCheck != nCoo) throw Error(HBDIA_ERR_RUNTIME, "device converter: COO count mismatch");
        cudaStream_t s;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        Q.stream = s;
        check_cuda(cudaGetDevice(&Q.device), "cudaGetDevice");
    } catch (...) {
        free_plan(Q);
        throw;
    }
    const int64_t xs = static_cast<int64_t>(sizeof(T));
    int64_t bytes = Q.slots * static_cast<int64_t>(vsz) + 4 * Q.totalOffsets + 4 * (static_cast<int64_t>(nb) + 1) +
                    2 * xs * Q.n + (8 + xs) * Q.nCoo + xs * Q.nCoo;
    if (Q.scale) bytes += 4 * static_cast<int64_t>(nb);
    if (Q.nCoo > 0) bytes += bw == 32 ? 4 * (static_cast<int64_t>(Q.numTiles) + 1) : 4 * (static_cast<int64_t>(nR) + 1);
    Q.bytesPerSpmv = bytes;
    Q.tailHeavy = tail_heavy(meta.histBlocks);
    P = Q;
}

template void convert_on_device<double>(const Coo<double> &, int32_t, int32_t, int64_t, int, DevicePlan &,
                                        DeviceLayoutMeta &);
template void convert_on_device<float>(const Coo<float> &, int32_t, int32_t, int64_t, int, DevicePlan &,
                                       DeviceLayoutMeta &);

}  // namespace hbdia
