// hbdia_spmv_host_noalloc: the host-buffer SpMV with its device-side x and y
// kept in one fixed array of this module instead of device allocations.
//
// hbdia_spmv_host allocates its two device buffers with cudaMalloc on the
// first call for a matrix.  Some callers cannot let that happen:
//  - a process whose device memory is already handed out to another
//    allocator (a caching allocator such as PyTorch's, or a fixed per-service
//    memory budget), where a late cudaMalloc can fail for lack of memory that
//    is free only inside the other allocator's pool;
//  - a latency-bound service loop that must not pay for an allocation (and
//    the device-wide synchronisation an allocation may imply) inside a
//    request.
// This entry point needs only the array below, so after its set-up it issues
// copies and one SpMV launch and nothing else.
//
// Limits and sharing:
//  - max(numRows, numCols) <= kMaxElems (2^21, a 128^3 grid); larger
//    matrices are rejected with HBDIA_ERR_INVALID_ARGUMENT.
//  - The array is one per device and shared by every call and every matrix,
//    so two calls that overlap in time (from different host threads) race on
//    it and both results are undefined; callers serialise them.
//  - Nothing in the array has to start at zero: each call first copies all of
//    x in, and the SpMV writes every one of the numRows elements of y before
//    they are copied out.
//  - The first call on a device does the set-up: it looks up the array's
//    device address with the device current.  Under CUDA's lazy module
//    loading (the default) that lookup is also what loads this file's module
//    and so commits the array's 32 MiB on the device, so the first call can
//    fail for lack of device memory; make it at start-up, before other
//    allocators claim the device, and before any stream capture on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "hbdia_b200.h"
#include "hbdia_internal.hpp"

namespace {
constexpr int64_t kMaxElems = int64_t(1) << 21;
constexpr int kMaxDevices = 64;
}  // namespace

// x occupies the first kMaxElems doubles, y the next kMaxElems (a float
// matrix uses the first half of each region): 32 MiB per device.
static __device__ __align__(256) double g_hostSpmvScratch[2 * kMaxElems];

namespace {

std::mutex g_setupMu;
void *g_scratch[kMaxDevices] = {};

// Device address of g_hostSpmvScratch on the current device, looked up once
// per device.
char *scratch_for(int device) {
    if (device < 0 || device >= kMaxDevices)
        throw hbdia::Error(HBDIA_ERR_UNSUPPORTED, "device index beyond the no-allocation table");
    std::lock_guard<std::mutex> lk(g_setupMu);
    if (!g_scratch[device]) {
        void *p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_hostSpmvScratch);
        if (rc != cudaSuccess || p == nullptr) {
            (void)cudaGetLastError();
            throw hbdia::Error(HBDIA_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                                                   cudaGetErrorString(rc));
        }
        g_scratch[device] = p;
    }
    return static_cast<char *>(g_scratch[device]);
}

}  // namespace

extern "C" int hbdia_spmv_host_noalloc(hbdia_matrix *m, const void *xHost, void *yHost) {
    try {
        if (!m || !xHost || !yHost) return hbdia::record_error(HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia_matrix_info info;
        int st = hbdia_matrix_get_info(m, &info);
        if (st != HBDIA_OK) return st;
        if (!info.hasHBDIA) return hbdia::record_error(HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
        hbdia_partial_info pinfo;
        st = hbdia_matrix_partial_info(m, &pinfo);
        if (st != HBDIA_OK) return st;
        if (pinfo.isPartial)
            return hbdia::record_error(HBDIA_ERR_UNSUPPORTED, "partial matrices use hbdia_spmv_host or _device");
        if (!info.onDevice)
            return hbdia::record_error(HBDIA_ERR_NOT_CONVERTED,
                                       "matrix has no device layout: call hbdia_matrix_prepare_gpu first "
                                       "(an upload here would allocate)");
        const int64_t elems = std::max<int64_t>(info.numRows, info.numCols);
        if (elems > kMaxElems)
            return hbdia::record_error(HBDIA_ERR_INVALID_ARGUMENT,
                                       "matrix needs " + std::to_string(elems) +
                                           " elements per vector; hbdia_spmv_host_noalloc holds at most " +
                                           std::to_string(kMaxElems) + " (use hbdia_spmv_host)");
        void *stream = nullptr;
        st = hbdia_matrix_stream(m, &stream);
        if (st != HBDIA_OK) return st;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int cur = -1, dev = -1;
        hbdia::check_cuda(cudaGetDevice(&cur), "cudaGetDevice");
        hbdia::check_cuda(cudaStreamGetDevice(s, &dev), "cudaStreamGetDevice");
        if (cur != dev)
            return hbdia::record_error(HBDIA_ERR_INVALID_ARGUMENT,
                                       "the matrix lives on device " + std::to_string(dev) + " but device " +
                                           std::to_string(cur) + " is current (hbdia_set_device)");
        char *base = scratch_for(dev);
        char *xs = base;
        char *ys = base + kMaxElems * static_cast<int64_t>(sizeof(double));
        const size_t es = info.dtype == HBDIA_F32 ? sizeof(float) : sizeof(double);
        hbdia::check_cuda(cudaMemcpyAsync(xs, xHost, static_cast<size_t>(elems) * es, cudaMemcpyHostToDevice, s),
                          "cudaMemcpyAsync(x)");
        st = hbdia_spmv_device(m, xs, ys, stream);
        if (st != HBDIA_OK) return st;
        hbdia::check_cuda(
            cudaMemcpyAsync(yHost, ys, static_cast<size_t>(info.numRows) * es, cudaMemcpyDeviceToHost, s),
            "cudaMemcpyAsync(y)");
        return hbdia_matrix_synchronize(m);
    } catch (const hbdia::Error &e) {
        return hbdia::record_error(e.status, e.what());
    } catch (const std::exception &e) {
        return hbdia::record_error(HBDIA_ERR_RUNTIME, e.what());
    }
}
