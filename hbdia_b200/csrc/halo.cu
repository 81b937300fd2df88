// Halo copies of row-partitioned SpMV: a fixed list of element segments
// copied between two device buffers by one kernel launch (packing the x
// ranges other ranks asked for into a send buffer, and unpacking received
// ranges into the x window).  The segment table is validated on the host
// against both buffer lengths and uploaded once; a copy is then one launch
// that allocates nothing and can be captured in a CUDA graph.
//
// Thread mapping: element e of the concatenated segments belongs to the
// segment s with start[s] <= e < start[s + 1] (binary search over the
// prefix table, which stays in L1/L2: a few KB for thousands of segments).
// Reads and writes are contiguous runs within a segment; the kernel is a
// plain copy, bound by HBM (or by the NVLink transfer it feeds).

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "hbdia_internal.hpp"

namespace hbdia {

struct Halo {
    int32_t elemBytes = 8;
    int32_t numSegments = 0;
    int64_t total = 0;
    int64_t *table = nullptr;  // device: start[nseg + 1] | src[nseg] | dst[nseg]
};

namespace {

template <typename E>
__global__ void __launch_bounds__(256) copy_segments(const int64_t *__restrict__ table, int32_t nseg, int64_t total,
                                                     const E *__restrict__ src, E *__restrict__ dst) {
    const int64_t *start = table;
    const int64_t *so = table + nseg + 1;
    const int64_t *d0 = so + nseg;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int32_t lo = 0, hi = nseg - 1;  // last segment with start <= e
        while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(start + mid) <= e) lo = mid;
            else hi = mid - 1;
        }
        const int64_t k = e - __ldg(start + lo);
        dst[__ldg(d0 + lo) + k] = src[__ldg(so + lo) + k];
    }
}

}  // namespace

Halo *halo_create(int32_t elemBytes, const int64_t *srcOff, const int64_t *dstOff, const int64_t *len,
                  int32_t numSegments, int64_t srcLen, int64_t dstLen) {
    if (elemBytes != 4 && elemBytes != 8) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "element size must be 4 or 8");
    if (numSegments < 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "negative segment count");
    if (numSegments > 0 && (!srcOff || !dstOff || !len))
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null segment array");
    std::vector<int64_t> t(static_cast<size_t>(3) * numSegments + 1, 0);
    int64_t total = 0;
    for (int32_t s = 0; s < numSegments; ++s) {
        if (len[s] < 0 || srcOff[s] < 0 || dstOff[s] < 0 || srcOff[s] + len[s] > srcLen ||
            dstOff[s] + len[s] > dstLen)
            throw Error(HBDIA_ERR_OUT_OF_RANGE, "halo segment " + std::to_string(s) + " outside its buffers");
        t[s] = total;
        t[numSegments + 1 + s] = srcOff[s];
        t[2 * static_cast<size_t>(numSegments) + 1 + s] = dstOff[s];
        total += len[s];
    }
    t[numSegments] = total;
    auto *h = new Halo();
    h->elemBytes = elemBytes;
    h->numSegments = numSegments;
    h->total = total;
    if (total > 0) {
        const int err = dev_alloc(&h->table, t.size() * sizeof(int64_t));
        if (err != cudaSuccess) {
            delete h;
            throw Error(HBDIA_ERR_NO_MEMORY, "cudaMalloc(halo table)");
        }
        const int e2 = cudaMemcpy(h->table, t.data(), t.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
        if (e2 != cudaSuccess) {
            cudaFree(h->table);
            delete h;
            check_cuda(e2, "cudaMemcpy(halo table)");
        }
    }
    return h;
}

void halo_copy(const Halo *h, const void *src, void *dst, void *stream) {
    if (h->total == 0) return;
    if (!src || !dst) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "null halo buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t blocks = std::min<int64_t>((h->total + 255) / 256, 148 * 8);
    if (h->elemBytes == 8)
        copy_segments<unsigned long long><<<static_cast<unsigned>(blocks), 256, 0, s>>>(
            h->table, h->numSegments, h->total, static_cast<const unsigned long long *>(src),
            static_cast<unsigned long long *>(dst));
    else
        copy_segments<unsigned int><<<static_cast<unsigned>(blocks), 256, 0, s>>>(
            h->table, h->numSegments, h->total, static_cast<const unsigned int *>(src),
            static_cast<unsigned int *>(dst));
    check_cuda(cudaGetLastError(), "copy_segments");
}

void halo_free(Halo *h) {
    if (!h) return;
    if (h->table) cudaFree(h->table);
    delete h;
}

int64_t halo_elements(const Halo *h) { return h->total; }

}  // namespace hbdia
