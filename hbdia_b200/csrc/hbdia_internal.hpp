// Internal data structures of libhbdia_b200.so (not part of the ABI).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "hbdia_b200.h"

namespace hbdia {

// Error carrying an hbdia_status, thrown inside the library and turned into
// a status code at the C ABI.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &msg) : std::runtime_error(msg), status(s) {}
};

// COO input of one matrix (the reference's values/rowIndices/colIndices).
template <typename T>
struct Coo {
    std::vector<int32_t> rows, cols;
    std::vector<T> vals;
    int32_t numRows = 0, numCols = 0;
    std::vector<int32_t> nnzPerRow;  // filled by the stencil generator only
    // Partial matrix (one rank's rows): global row of local row 0.  Offsets
    // are col - (row + rowBase), as the reference computes them from its
    // global row mapping (src/Format/HBDIA.cpp:546-552).
    int32_t rowBase = 0;
};

// Host HBDIA layout: exactly the reference's host-side members after
// convertToHBDIAFormat (include/Format/HBDIA.hpp:232-253), with
// offsetsPerBlock stored flattened.
template <typename T>
struct HostLayout {
    int32_t numRows = 0, numCols = 0, blockWidth = 0, threshold = 0;
    int64_t maxCoo = 0;
    int32_t rowBase = 0;                   // partial matrices: global row of local row 0
    int32_t numBlocks = 0;                 // maxNumBlocks
    std::vector<int32_t> offsets;          // kept offsets, ascending per block
    std::vector<int32_t> blockStart;       // numBlocks + 1, offset units
    std::vector<T> data;                   // [block][offsetIdx][lane]
    std::vector<int32_t> cooRow, cooCol;   // COO remainder, input order
    std::vector<T> cooVal;
    std::vector<int32_t> cooRowPtr;        // numRows + 1 (reference's cpuRowPtr)
    int32_t numberDiagonals = 0;
    std::vector<int32_t> histBlocks, histNnz;
    bool cooRowSorted = true;              // COO rows non-decreasing
};

// Partial matrix (one rank's rows, partition.cpp): the reference's
// PartialMatrixMetadata plus this library's x window.
struct PartialMeta {
    bool partial = false, hasMetadata = false;
    int32_t numGlobalRows = 0, numGlobalCols = 0, rank = 0, size = 1;
    int64_t numGlobalNonZeros = 0;
    std::vector<int32_t> dataRanges;      // pairs [start, end), ascending
    std::vector<int32_t> processRanges;   // triples (process, start, end)
    int64_t totalBufferSize = 0, leftBufferSize = 0, rightBufferSize = 0;
    int32_t windowLo = 0, windowLen = 0;
};
template <typename T>
void partition_rows(const Coo<T> &g, int32_t numProcesses, int32_t part, Coo<T> &local);
template <typename T>
void partial_metadata(const Coo<T> &c, const HostLayout<T> &L, PartialMeta &m);

// Halo copies (halo.cu): a fixed list of (src, dst, len) element segments
// between two device buffers, copied by one kernel.
struct Halo;
Halo *halo_create(int32_t elemBytes, const int64_t *srcOff, const int64_t *dstOff, const int64_t *len,
                  int32_t numSegments, int64_t srcLen, int64_t dstLen);
void halo_copy(const Halo *h, const void *src, void *dst, void *stream);
void halo_free(Halo *h);
int64_t halo_elements(const Halo *h);

// Converter: convertToHBDIAFormat restated for speed (OpenMP), bit-exact.
template <typename T>
void convert_to_hbdia(const Coo<T> &coo, int32_t blockWidth, int32_t threshold, int64_t maxCoo,
                      HostLayout<T> &out);

// DIA format and storage costs (dia.cpp)
template <typename T>
void remove_coo_duplicates(Coo<T> &c);
template <typename T>
void convert_to_dia(Coo<T> &c, bool cooIsUnique, std::vector<int32_t> &offsets, std::vector<T> &diagonals,
                    int32_t &diagLength);
void storage_costs(int64_t valueBytes, int32_t numRows, int32_t numCols, int64_t numNonZeros,
                   int32_t numberDiagonals, int32_t numBlocks, int32_t blockWidth, int64_t hbdiaSlots,
                   int64_t cooEntries, const std::vector<int32_t> &histBlocks, const std::vector<int32_t> &nnzPerRow,
                   hbdia_storage_costs &out);

// Generators (generate.cpp)
template <typename T>
void reference_stencil27(int nx, int ny, int nz, double noise, int iteration, Coo<T> &out);
template <typename T>
bool load_mtx(const std::string &path, int numRows, int numCols, Coo<T> &out);

// Simple sequential stable sort of COO (rows) used when the COO remainder is
// not row-sorted; returns the permutation.
std::vector<int64_t> stable_row_order(const std::vector<int32_t> &rows, int32_t numRows);

}  // namespace hbdia

namespace hbdia {

// Device layout of one converted matrix (prepareForGPU's arrays,
// src/Format/HBDIA.cpp:720-816, in this library's form).  All arrays live in
// one device allocation, each 256-byte aligned.
struct DevicePlan {
    int32_t dtype = HBDIA_F64;          // T of x, y and the COO values
    int32_t storage = HBDIA_STORE_NATIVE;  // value type: NATIVE, F32 or BF16_SCALED
    bool quadLayout = false;             // F32 / BF16 values of uniform quads interleaved
                                         // (HBDIA_STORE_F32_QUAD / _BF16_QUAD: QUAD kernel only)
    int32_t n = 0, numCols = 0, bw = 0, numBlocks = 0, numTiles = 0;
    int32_t xn = 0;  // DIA column bound: n, or a partial matrix's x-window length
    int64_t totalOffsets = 0, slots = 0, nCoo = 0;
    void *base = nullptr;
    size_t bytes = 0;
    void *vals = nullptr;                // storage type
    float *scale = nullptr;              // per-block scale (bf16 storage)
    int32_t *offs = nullptr, *blkOff = nullptr;
    int32_t *cooRow = nullptr, *cooCol = nullptr;
    void *cooVal = nullptr;              // T
    int32_t *cooRowPtr = nullptr, *cooTile = nullptr;
    void *stream = nullptr;              // cudaStream_t owned by the plan
    int32_t device = -1;                 // the device the layout lives on (current when it was built)
    void *xScratch = nullptr, *yScratch = nullptr;  // hbdia_spmv_host buffers
    int64_t bytesPerSpmv = 0;            // algorithmic HBM bytes of one SpMV
    int32_t *status = nullptr;           // device error bits of bounded waits (staged kernel)
    int32_t kernel = HBDIA_KERNEL_AUTO;  // hbdia_kernel choice
    uint64_t waitTimeoutNs = 2000000000ull;
    int32_t skipTile = -1;               // test hook of the staged kernel
    int32_t xsConfig = 0;                // HBDIA_TUNE_STAGES: staged kernel's shape (0: default)
    int32_t quadGroup = 0;               // HBDIA_TUNE_QUAD_GROUP: quad kernel's offsets in flight (0: default)
    int32_t unroll = 0;                  // offsets in flight per lane (0: default)
    std::map<int32_t, int32_t> spmmTile; // autotuned RHS tile per k
    int32_t spmmTileForced = 0;          // HBDIA_TUNE_SPMM_TILE (0: autotuned / default)
    int32_t prefetchL2 = -1;             // HBDIA_TUNE_PREFETCH: pipe kernel L2 prefetch of the next
                                         // tile (-1: when x exceeds L2, 0: off, 1: on)
    int32_t maskedTail = -1;             // HBDIA_TUNE_TAIL: the pipe kernel's offsets past its last full
                                         // group in masked groups (-1: when tailHeavy, 0: off, 1: on)
    bool tailHeavy = false;              // at least half the stored offsets lie past full groups
};

// Host-side facts of a layout built on the device (convert_gpu.cu).
struct DeviceLayoutMeta {
    int32_t numberDiagonals = 0;
    std::vector<int32_t> histBlocks, histNnz;
};
// COO -> device plan on the GPU; row-sorted COO only (HBDIA_ERR_UNSUPPORTED
// otherwise); the same layout as convert_to_hbdia + build_plan, without the
// staged kernel's schedule.
template <typename T>
void convert_on_device(const Coo<T> &coo, int32_t blockWidth, int32_t threshold, int64_t maxCoo, int storage,
                       DevicePlan &P, DeviceLayoutMeta &meta);

// kernel that launch_spmv would use for x (HBDIA_KERNEL_*)
int32_t select_kernel(const DevicePlan &P, const void *x);

// The x window of a partial matrix's plan: global column c is read at
// x[c - lo], lo <= c < lo + len; the rank's rows start at global row rowBase.
struct ColumnWindow {
    int32_t lo = 0, len = 0, rowBase = 0;
};

template <typename T>
void build_plan(const HostLayout<T> &L, int storage, DevicePlan &P, const ColumnWindow *W = nullptr);
// The storage an iteration operator (CG) is built with: a quad-interleaved
// storage the layout cannot take (blockWidth other than 32, more than 2^30
// rows) becomes its per-block counterpart, which gives the same y.
int32_t iteration_storage(const HostLayout<double> &L, int32_t storage);
// A plan over a caller-owned device layout (layout_plan.cu).
void borrow_plan(const hbdia_layout_desc &d, DevicePlan &P);
void free_plan(DevicePlan &P);
// True when at least half of the stored offsets fall past the last full group
// of the pipe kernel (histBlocks[d] = blocks with d offsets).
bool tail_heavy(const std::vector<int32_t> &histBlocks);
// y = A x on `stream` (a cudaStream_t; nullptr -> the plan's stream)
void launch_spmv(const DevicePlan &P, const void *x, void *y, void *stream);
// Y = A X for k right-hand sides: row-major blocks (element (i, j) at
// X[i * ldx + j]) or, with colMajor, column-major ones (X[j * ldx + i]).
void launch_spmm(const DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                 void *stream, bool colMajor = false);
void launch_spmm_tile(const DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                      int32_t tile, void *stream, bool colMajor = false);
int32_t default_spmm_tile(int32_t k, bool colMajor = false);
// k SpMVs of one matrix on separate device vectors (x[j] -> y[j]) as
// vector-list SpMMs of up to 32 vectors per launch, bit-identical to k SpMVs.
void launch_spmv_list(const DevicePlan &P, const void *const *x, void *const *y, int32_t k, void *stream);
void autotune(DevicePlan &P, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k, void *stream, bool force,
              int32_t *kernel, int32_t *unroll, int32_t *tile, int32_t *fromCache, float *ms);
void autotune_clear_cache();

// CG with reliable updates (cg.cu): iterations on Ait (reduced or FP64
// storage), FP64 residual recomputations with A64.
struct CgWork;
CgWork *cg_work(CgWork *w, int64_t n);
void cg_free(CgWork *w);
int64_t cg_work_bytes(int64_t n, int sms);  // device bytes of a workspace for n rows
struct CgParams {
    double tol = 1e-10;          // target ||b - A x|| / ||b||
    double updateFactor = 0.1;   // reliable update when the iterated residual falls below this
                                 // times the largest one since the last update
    int32_t maxUpdates = 100;    // FP64 residual recomputations
    int32_t maxIterations = 20000;
    int32_t checkEvery = 10;     // iterations per CUDA-graph replay / host check
};
struct CgStats {
    int32_t updates = 0, iterations = 0;
    double relResidual = 0.0, seconds = 0.0;
};
void cg_solve(const DevicePlan &A64, const DevicePlan &Ait, CgWork *w, const double *b, double *x,
              const CgParams &prm, void *stream, CgStats *stats);
// Up to 16 solves on one matrix in lockstep (one SpMM per iteration), each
// with its own workspace; every result equals its lone cg_solve bit for bit.
struct CgCall {
    const double *b;
    double *x;
    CgWork *w;
    CgStats *stats;
};
void cg_solve_group(const DevicePlan &A64, const DevicePlan &Ait, CgCall *calls, int k, const CgParams &prm,
                    void *stream);
// Many matrices in one persistent launch (batch.cu)
struct Batch;
Batch *batch_create(const std::vector<const DevicePlan *> &plans);
void batch_free(Batch *b);
void batch_bind(Batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                const int32_t *k);
void batch_run(Batch *b, void *stream);
void batch_set_config(Batch *b, const hbdia_batch_config &c);
void batch_get_config(const Batch *b, hbdia_batch_config &c);
void batch_autotune(Batch *b, void *stream, float *ms, int32_t *candidates);
void batch_info(const Batch *b, int32_t *count, int32_t *totalTiles, int64_t *bytesPerRun);
void *batch_stream(const Batch *b);

// Serving engine (serve.cpp)
struct Server;
void server_default_options(hbdia_server_options *o);
Server *server_create(const hbdia_server_options &o);
void server_destroy(Server *S);
int32_t server_add_matrix(Server *S, const hbdia_matrix *m);
uint64_t server_submit(Server *S, int32_t matrix, int32_t kind, const double *x, double *y, bool device);
void server_wait(Server *S, uint64_t ticket, hbdia_request_info *info);
void server_pause(Server *S, bool paused);
void server_stats(Server *S, hbdia_server_stats *out);

// throws Error(HBDIA_ERR_CUDA) with the CUDA error string
void check_cuda(int err, const char *what);
// Every device allocation (cudaMalloc) and page-locked host allocation
// (cudaMallocHost) of the library goes through these, which count the
// successful ones (hbdia_allocation_count).  They return the cudaError_t.
int dev_alloc_bytes(void **p, size_t bytes);
int pinned_alloc_bytes(void **p, size_t bytes);
template <typename T>
int dev_alloc(T **p, size_t bytes) {
    return dev_alloc_bytes(reinterpret_cast<void **>(p), bytes);
}
template <typename T>
int pinned_alloc(T **p, size_t bytes) {
    return pinned_alloc_bytes(reinterpret_cast<void **>(p), bytes);
}
void allocation_counts(int64_t *device, int64_t *pinned);
// Sets the message hbdia_last_error() reports on this thread; returns status.
int record_error(int status, const std::string &msg);

int generate_stencil(int stencilPoints, int32_t nx, int32_t ny, int32_t nz, double center,
                     double neighbor, double frac, double lo, double hi, uint64_t seed,
                     int64_t *nnzOut, int32_t *rows, int32_t *cols, double *vals);
int generate_banded(int32_t n, const int32_t *offs, int32_t noffs, double lo, double hi, double drop,
                    double scatter, uint64_t seed, int64_t *nnzOut, int32_t *rows, int32_t *cols,
                    double *vals);
void fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed);
int generate_stencil27_spd(int32_t nx, int32_t ny, int32_t nz, double shift, double extraFraction, uint64_t seed,
                           int64_t *nnzOut, int32_t *rows, int32_t *cols, double *vals);

}  // namespace hbdia
