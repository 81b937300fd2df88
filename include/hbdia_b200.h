/*
 * hbdia_b200 -- C ABI of the B200-native HBDIA SpMV library (libhbdia_b200.so).
 *
 * This is the drop-in boundary under the C++ API of include/hbdia/Format/HBDIA.hpp,
 * HBDIAVector.hpp and HBDIASpMV.hpp (HBDIA<T>, HBDIAVector<T>, hbdiaSpMV), which mirror the reference's
 * classes.  Every entry point names the reference interface it replaces
 * (paths relative to the reference project root).  The signatures use plain
 * pointers and sizes only; CUDA streams are passed as `void*`
 * (a cudaStream_t), NULL meaning the matrix's own stream.
 *
 * Conventions
 *  - Every function returns an hbdia_status (0 = success).  No function exits
 *    the process: the reference's CHECK_CUDA calls exit(1)
 *    (include/types.hpp:37-44); here CUDA errors become HBDIA_ERR_CUDA and the
 *    C++ layer throws.  hbdia_last_error() returns the calling thread's
 *    message for the last failing call.
 *  - Value type T is chosen per object with hbdia_dtype (double or float, the
 *    two instantiations of hbdiaSpMV, src/Operations/HBDIASpMV.cpp:254-255).
 *  - All SpMV entry points are asynchronous on their stream, as the
 *    reference's hbdiaSpMV is (it returns without synchronizing,
 *    src/Operations/HBDIASpMV.cpp:251); hbdia_spmv_host is the exception.
 *  - A converted matrix is immutable until destroyed, so concurrent SpMVs on
 *    different streams over the same matrix are allowed.
 */
#ifndef HBDIA_B200_H
#define HBDIA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hbdia_status {
    HBDIA_OK = 0,
    HBDIA_ERR_INVALID_ARGUMENT = -1, /* reference: std::invalid_argument      */
    HBDIA_ERR_OUT_OF_RANGE = -2,     /* reference: std::out_of_range (indices) */
    HBDIA_ERR_RUNTIME = -3,          /* reference: std::runtime_error          */
    HBDIA_ERR_CUDA = -4,             /* a CUDA runtime call failed             */
    HBDIA_ERR_NO_MEMORY = -5,        /* host or device allocation failed       */
    HBDIA_ERR_NOT_CONVERTED = -6,    /* matrix has no HBDIA layout yet         */
    HBDIA_ERR_UNSUPPORTED = -7,      /* combination not implemented            */
    HBDIA_ERR_DEVICE_TIMEOUT = -8    /* a bounded device-side wait ran out     */
} hbdia_status;

typedef enum hbdia_dtype { HBDIA_F64 = 0, HBDIA_F32 = 1 } hbdia_dtype;

/* ExecutionMode (include/types.hpp:7-10).  Kept for source compatibility:
 * the COO remainder always runs on the GPU, fused into the SpMV launch. */
typedef enum hbdia_exec_mode { HBDIA_CPU_COO = 0, HBDIA_GPU_COO = 1 } hbdia_exec_mode;

/* Device storage of the blocked-DIA values.  NATIVE stores T.  F32 and
 * BF16_SCALED store float / bfloat16 (with one float scale per block) for a
 * double matrix; the SpMV then still accumulates in double.  F32_QUAD and
 * BF16_QUAD store the same values with those of every uniform quad (four
 * consecutive blocks with one list of at most 32 offsets) interleaved
 * [offset][lane][block], so that the quad kernel reads a lane's four values of
 * an offset with one 16- / 8-byte load; they need blockWidth 32, run the SpMV
 * through the quad kernel only (whatever kernel is set) and give the same y
 * as F32 / BF16_SCALED bit for bit; SpMM, vector lists and batches refuse
 * them (HBDIA_ERR_UNSUPPORTED). */
typedef enum hbdia_value_storage {
    HBDIA_STORE_NATIVE = 0,
    HBDIA_STORE_F32 = 1,
    HBDIA_STORE_BF16_SCALED = 2,
    HBDIA_STORE_F32_QUAD = 3,
    HBDIA_STORE_BF16_QUAD = 4
} hbdia_value_storage;

/* SpMV kernel choice (all give bit-identical y).  AUTO picks the kernel
 * measured fastest on B200: for blockWidth 32 QUAD with 4- and 2-byte value
 * storage, PIPE with 8-byte values; ROWWISE for other block widths.  STAGED
 * needs a 16-byte aligned x and value array (else WARP runs); PIPE and STAGED
 * need numRows <= 2^30. */
typedef enum hbdia_kernel {
    HBDIA_KERNEL_AUTO = 0,
    HBDIA_KERNEL_ROWWISE = 1, /* one thread per row, any blockWidth             */
    HBDIA_KERNEL_WARP = 2,    /* one warp per 32-row block, blockWidth 32       */
    HBDIA_KERNEL_STAGED = 3,  /* persistent; each warp bulk-copies its next tiles' values and
                                 x runs into shared memory, blockWidth 32 */
    HBDIA_KERNEL_PIPE = 4,    /* persistent warp per block, pipelined across blocks, blockWidth 32 */
    HBDIA_KERNEL_QUAD = 5     /* persistent warp per 4 blocks sharing one offset list, blockWidth 32 */
} hbdia_kernel;

typedef struct hbdia_matrix hbdia_matrix; /* HBDIA<T>       (include/Format/HBDIA.hpp:24-291)      */
typedef struct hbdia_vector hbdia_vector; /* HBDIAVector<T> (include/Format/HBDIAVector.hpp:23-109) */

const char *hbdia_last_error(void);
const char *hbdia_version(void);

/* The library carries its own (static) CUDA runtime, which shares the
 * device's primary context with any other CUDA user in the process.  Its
 * current device is per host thread and starts at 0: a process driving
 * another GPU calls hbdia_set_device first (the reference relies on the
 * caller's cudaSetDevice, src/DataExchange/MPICommunicator.cpp).  No
 * counterpart is needed on one GPU. */
int hbdia_set_device(int32_t device);
int hbdia_get_device(int32_t *device);
/* Status name, e.g. "HBDIA_ERR_RUNTIME". */
const char *hbdia_status_string(int status);
/* Allocations the library has made since it was loaded: device memory
 * (cudaMalloc) and page-locked host memory (cudaMallocHost), successful calls
 * only.  No counterpart in the reference.  Read it around a call to check
 * that the call allocated nothing. */
int hbdia_allocation_count(int64_t *device, int64_t *pinnedHost);

/* ---------------------------------------------------------------- matrices */

/* HBDIA() (src/Format/HBDIA.cpp:20-21): empty matrix, to be filled by
 * hbdia_matrix_stencil27 or hbdia_matrix_load_mtx. */
int hbdia_matrix_create_empty(hbdia_dtype dtype, hbdia_matrix **out);

/* HBDIA(rowIndices, colIndices, values, numRows, numCols)
 * (src/Format/HBDIA.cpp:51-80): copies the COO triplets, validates sizes
 * (HBDIA_ERR_INVALID_ARGUMENT) and index bounds (HBDIA_ERR_OUT_OF_RANGE).
 * numRows <= 0 and numCols <= 0 together select the dimension-inferring
 * constructor HBDIA(rowIndices, colIndices, values) (src/Format/HBDIA.cpp:23-49). */
int hbdia_matrix_create(hbdia_dtype dtype, const int32_t *rowIndices, const int32_t *colIndices,
                        const void *values, int64_t nnz, int32_t numRows, int32_t numCols,
                        hbdia_matrix **out);

void hbdia_matrix_destroy(hbdia_matrix *m); /* ~HBDIA (src/Format/HBDIA.cpp:156-159) */

/* create3DStencil27Point(nx, ny, nz, noise, iteration)
 * (src/Format/HBDIA.cpp:1416-1607): replaces the matrix's COO data with the
 * reference's 27-point stencil; identical entries and order. */
int hbdia_matrix_stencil27(hbdia_matrix *m, int32_t nx, int32_t ny, int32_t nz, double noise,
                           int32_t iteration);

/* loadMTX(filename) / loadMTX(filename, numRows, numCols)
 * (src/Format/HBDIA.cpp:161-263 and :265-370).  numRows, numCols <= 0 select
 * the first overload.  *ok receives the reference's boolean result. */
int hbdia_matrix_load_mtx(hbdia_matrix *m, const char *path, int32_t numRows, int32_t numCols,
                          int32_t *ok);

/* convertToHBDIAFormat(blockWidth, threshold, max_coo_entries, COOisUnique,
 * execMode) (src/Format/HBDIA.cpp:507-718).  The host layout is bit-exact with
 * the reference's.  With upload != 0 it then builds the device layout
 * (prepareForGPU, src/Format/HBDIA.cpp:720-816), as the reference does for
 * every non-partial matrix; upload == 0 converts on the host only (no GPU
 * needed).  Like the reference, it is a no-op on an already converted or
 * empty matrix. */
int hbdia_matrix_convert(hbdia_matrix *m, int32_t blockWidth, int32_t threshold,
                         int64_t maxCooEntries, int32_t cooIsUnique, int32_t execMode,
                         int32_t upload);

/* prepareForGPU (src/Format/HBDIA.cpp:720-816): upload the layout, creating
 * the matrix's stream.  storage selects the device value format. */
int hbdia_matrix_prepare_gpu(hbdia_matrix *m, int32_t storage);

/* removeCOODuplicates (src/Format/HBDIA.cpp:372-412): entries with the same
 * (row, col) are summed (0 + v1 + v2 + ... in input order) and the COO is
 * left sorted by (row, col). */
int hbdia_matrix_remove_duplicates(hbdia_matrix *m);

/* convertToDIAFormat(COOisUnique) (src/Format/HBDIA.cpp:414-505): unless
 * cooIsUnique, removes duplicates first (changing the COO, as the reference
 * does); then one diagonal of min(numRows, numCols) values per distinct
 * offset col - row, ascending.  Host data only (the reference uploads DIA
 * data to no device).  No-op when converted already or without COO. */
int hbdia_matrix_convert_dia(hbdia_matrix *m, int32_t cooIsUnique);
/* isDIAFormat, getOffsets().size(), diagonal length */
int hbdia_matrix_dia_info(const hbdia_matrix *m, int32_t *hasDIA, int32_t *numDiagonals, int32_t *diagLength);
/* getOffsets (numDiagonals int32) and getDiagonals flattened [diagonal][position]
 * (include/Format/HBDIA.hpp:89-90). */
int hbdia_matrix_export_dia(const hbdia_matrix *m, int32_t *offsets, void *diagonals);

/* Storage costs in bytes of the matrix held as HBDIA (its values, block
 * pointers, stored offsets and COO remainder), COO, DIA, SELL-C (C =
 * blockWidth, from the per-row counts the 27-point stencil generator
 * records; meaningful for threshold 1) and CSR -- the figures the
 * reference's benchmark prints and saves (benchmarking/benchmark.cpp:171-215).
 * Needs the HBDIA conversion. */
typedef struct hbdia_storage_costs {
    int64_t hbdia, coo, dia, sell, csr;
} hbdia_storage_costs;
int hbdia_matrix_storage_costs(const hbdia_matrix *m, hbdia_storage_costs *costs);

/* convertToHBDIAFormat (src/Format/HBDIA.cpp:507-718) + prepareForGPU done
 * on the GPU: the same device layout (and the same offsets, values, COO
 * remainder, histograms and numberDiagonals) as hbdia_matrix_convert +
 * hbdia_matrix_prepare_gpu(storage), without the host pass over the
 * entries; the host layout is not materialised (hbdia_matrix_export_layout
 * reads the device copy back, for NATIVE storage).  Requires row-sorted COO
 * (HBDIA_ERR_UNSUPPORTED otherwise).  The staged kernel's schedule is not
 * built, so HBDIA_KERNEL_STAGED runs the warp kernel on such a matrix.  A
 * no-op on an already converted or empty matrix, like the reference. */
int hbdia_matrix_convert_on_device(hbdia_matrix *m, int32_t blockWidth, int32_t threshold,
                                   int64_t maxCooEntries, int32_t storage);

typedef struct hbdia_matrix_info {
    int32_t dtype;            /* hbdia_dtype                                    */
    int32_t numRows;          /* getNumRows   (include/Format/HBDIA.hpp:74)     */
    int32_t numCols;          /* getNumCols                                     */
    int32_t hasCOO;           /* getHasCOO                                      */
    int64_t numNonZeros;      /* getNumNonZeros                                 */
    int32_t hasHBDIA;         /* getHasHBDIA                                    */
    int32_t onDevice;         /* device layout present                          */
    int32_t blockWidth;       /* getBlockWidth                                  */
    int32_t threshold;        /* getThreshold                                   */
    int64_t maxCooEntries;    /* getMaxCooEntries                               */
    int32_t numBlocks;        /* getNumBlocks                                   */
    int32_t numberDiagonals;  /* getNumberDiagonals                             */
    int64_t totalOffsets;     /* sum of |getOffsetsPerBlock()[b]|               */
    int64_t numSlots;         /* getHBDIAData().size()                          */
    int64_t numCoo;           /* getCpuValues().size()                          */
    int32_t histogramLength;  /* getHistogramBlocks().size()                    */
    int32_t storage;          /* hbdia_value_storage on the device              */
    int64_t deviceBytes;      /* bytes held on the device by the layout         */
    int64_t bytesPerSpmv;     /* algorithmic HBM bytes of one SpMV              */
} hbdia_matrix_info;

int hbdia_matrix_get_info(const hbdia_matrix *m, hbdia_matrix_info *info);

/* Copy out the host layout (getters, include/Format/HBDIA.hpp:88-114).
 * offsetsPerBlock is returned flattened: offsets[blockStart[b] ..
 * blockStart[b+1]) are block b's ascending offsets (the form of
 * prepareForGPU, src/Format/HBDIA.cpp:733-760).  Any NULL pointer is skipped.
 * Sizes come from hbdia_matrix_get_info (cooRowPtr has numRows+1 entries). */
int hbdia_matrix_export_layout(const hbdia_matrix *m, int32_t *offsets, int32_t *blockStart,
                               void *data, int32_t *cooRow, int32_t *cooCol, void *cooVal,
                               int32_t *cooRowPtr, int32_t *histogramBlocks,
                               int32_t *histogramNnz);

/* getRowIndices / getColIndices / getValues (include/Format/HBDIA.hpp:82-84)
 * and getNnzPerRow (numRows entries, filled by stencil27 only). */
int hbdia_matrix_export_coo(const hbdia_matrix *m, int32_t *rowIndices, int32_t *colIndices,
                            void *values);
int hbdia_matrix_export_nnz_per_row(const hbdia_matrix *m, int32_t *nnzPerRow);

/* getBDIAStream (include/Format/HBDIA.hpp:168): the stream the matrix's
 * SpMVs run on (created by prepare_gpu). */
int hbdia_matrix_stream(const hbdia_matrix *m, void **stream);

/* The device arrays prepareForGPU leaves (src/Format/HBDIA.cpp:720-816),
 * returned by the GPU getters of include/Format/HBDIA.hpp:155-165
 * (getHBDIADataDevice, getFlattenedOffsetsDevice,
 * getBlockStartIndicesDevice, getBlockSizesDevice,
 * getFlattenedVectorOffsetsDevice, getCpuRowIndicesDevice,
 * getCpuColIndicesDevice, getCpuValuesDevice, getCpuRowPtrDevice).  They are
 * the arrays the fused SpMV reads, owned by the matrix and valid until it is
 * destroyed or prepared again:
 *  - hbdiaData: [block][offsetIdx][lane] values of T, blockWidth per offset;
 *    NULL when the values are stored in a reduced format (prepare_gpu with
 *    HBDIA_STORE_F32 / HBDIA_STORE_BF16_SCALED);
 *  - flattenedOffsets, blockStartIndices (numBlocks + 1, offset units) and
 *    blockSizes (numBlocks; built on the first request);
 *  - flattenedVectorOffsets: NULL for a whole matrix, as in the reference; for
 *    a partial matrix the offsets into its x window (column - windowLo - local
 *    row), which is what the fused kernel reads, with flattenedOffsets NULL;
 *  - the COO remainder cpuRowIndices / cpuColIndices / cpuValues (numCoo) in
 *    row order (the reference's list order for its row-sorted input) and
 *    cpuRowPtr (numRows + 1).  NULL when the matrix has no COO remainder. */
typedef struct hbdia_device_arrays {
    const void *hbdiaData;
    const int32_t *flattenedOffsets;
    const int32_t *blockStartIndices;
    const int32_t *blockSizes;
    const int32_t *flattenedVectorOffsets;
    const int32_t *cpuRowIndices;
    const int32_t *cpuColIndices;
    const void *cpuValues;
    const int32_t *cpuRowPtr;
} hbdia_device_arrays;
int hbdia_matrix_device_arrays(hbdia_matrix *m, hbdia_device_arrays *arrays);

/* ---------------------------------------------------------------- vectors */

/* HBDIAVector(localData) (src/Format/HBDIAVector.cpp:17-23): device buffer
 * holding n elements copied from host (hostData may be NULL: zeros).  On one
 * GPU the halo parts are empty, so the data and local pointers coincide. */
int hbdia_vector_create(hbdia_dtype dtype, const void *hostData, int64_t n, hbdia_vector **out);
void hbdia_vector_destroy(hbdia_vector *v);
/* getDeviceDataPtr / getDeviceLocalPtr (include/Format/HBDIAVector.hpp:48-50) */
int hbdia_vector_device_ptr(const hbdia_vector *v, void **devicePtr);
/* getDeviceCOOResultsPtr (include/Format/HBDIAVector.hpp:53): the
 * reference's separate buffer for the COO remainder's partial result, which
 * its callers clear before each SpMV (benchmarking/benchHBDIA.cpp:33).  The
 * fused SpMV never reads or writes it; it exists (n zeroed elements,
 * allocated on the first request, owned by the vector) so such callers run
 * unchanged. */
int hbdia_vector_coo_results_ptr(hbdia_vector *v, void **devicePtr);
int hbdia_vector_size(const hbdia_vector *v, int64_t *n);
/* blocking host<->device copies of the whole vector */
int hbdia_vector_upload(hbdia_vector *v, const void *hostData);
int hbdia_vector_download(const hbdia_vector *v, void *hostData);

/* ---------------------------------------------------------------- SpMV */

/* hbdiaSpMV(matrix, inputVector, outputVector, execCOOCPU, execCOOGPU)
 * (src/Operations/HBDIASpMV.cpp:186-251; declared include/Operations/HBDIASpMV.hpp:8-10).
 * y = A x in ONE fused launch (blocked-DIA part and COO remainder) on the
 * matrix's stream; returns without synchronizing.  If the matrix has COO
 * entries and both flags are 0 it fails with HBDIA_ERR_RUNTIME, as the
 * reference throws std::runtime_error("Invalid COO execution flags")
 * (src/Operations/HBDIASpMV.cpp:229-232).  Either flag selects the same fused
 * GPU path.  Every row of y is written. */
int hbdia_spmv(hbdia_matrix *m, const hbdia_vector *x, hbdia_vector *y, int32_t execCOOCPU,
               int32_t execCOOGPU);

/* Same product on caller-owned device buffers (numRows elements of T each)
 * and the caller's stream (NULL: the matrix's stream).  No allocation, so it
 * can be captured in a CUDA graph. */
int hbdia_spmv_device(const hbdia_matrix *m, const void *x, void *y, void *stream);

/* Multi-RHS product Y = A X for k right-hand sides.  X and Y are device
 * buffers in row-major layout with leading dimensions ldx, ldy >= k
 * (element (i, j) at i*ld + j).  Each value load is reused across all k. */
int hbdia_spmm_device(const hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy,
                      int32_t k, void *stream);

/* The same product on column-major blocks: right-hand side j is the
 * contiguous vector X + j * ldx (ldx >= max(numRows, numCols)), result j is
 * Y + j * ldy (ldy >= numRows).  For callers whose right-hand sides arrive
 * as separate vectors (a server's requests).  Column j equals
 * hbdia_spmv_device of that vector bit for bit.  No counterpart in the
 * reference. */
int hbdia_spmm_device_colmajor(const hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy,
                               int32_t k, void *stream);

/* k SpMVs of one matrix over separate device vectors: y[j] = A x[j] for
 * j < k (x[j] holding max(numRows, numCols) elements, y[j] numRows), with
 * each stored value read once for up to 32 vectors (vector-list SpMMs; the
 * pointer arrays are host arrays, passed to the kernel by value).  Each y[j]
 * equals hbdia_spmv_device(m, x[j], y[j]) bit for bit.  Allocation-free and
 * graph-capturable.  No counterpart in the reference. */
int hbdia_spmv_list_device(const hbdia_matrix *m, const void *const *x, void *const *y, int32_t k, void *stream);

/* End-to-end form on HOST buffers: copies x to the device, runs the SpMV,
 * copies y back and synchronizes.  Page-locked host buffers are fastest. */
int hbdia_spmv_host(hbdia_matrix *m, const void *xHost, void *yHost);

/* count SpMVs on host buffers, y[j] = A x[j], pipelined three deep: step j's
 * copy in, SpMV and copy out run in order on one of three streams (with its
 * own device staging pair, allocated on the first call and kept until the
 * matrix is destroyed or reconverted), so step j+1's upload overlaps step
 * j's kernel and download on the two directions of the host link.  Each
 * y[j] equals hbdia_spmv_host(m, x[j], y[j]) bit for bit; returns when all
 * are done.  The overlap needs page-locked host buffers.  A y buffer may
 * appear more than once only at least three steps apart.  No counterpart in
 * the reference. */
int hbdia_spmv_host_many(hbdia_matrix *m, const void *const *xHost, void *const *yHost, int32_t count);

/* ---- Plans over a device layout the caller owns ------------------------
 *
 * The arrays prepareForGPU leaves on the device (src/Format/HBDIA.cpp:720-816),
 * read through the reference's getters (include/Format/HBDIA.hpp:155-165):
 *   values      getHBDIADataDevice()          totalOffsets * blockWidth, [block][offsetIdx][lane]
 *   offsets     getFlattenedOffsetsDevice()   totalOffsets, ascending within each block
 *   blockStart  getBlockStartIndicesDevice()  numBlocks + 1, offset units
 *   cooRow, cooCol, cooVal, cooRowPtr         getCpuRowIndicesDevice() ... getCpuRowPtrDevice():
 *                                             numCoo entries, row-sorted; numRows + 1 row pointer
 * numBlocks = ceil(min(numRows, numCols) / blockWidth) as convertToHBDIAFormat
 * makes it.  storage F32 / BF16_SCALED describe float / bfloat16 values of a
 * double layout (with one float scale per block for BF16: value = stored *
 * scale). */
typedef struct hbdia_layout_desc {
    int32_t dtype;          /* hbdia_dtype of x, y and the COO values            */
    int32_t storage;        /* hbdia_value_storage of `values`                   */
    int32_t numRows, numCols, blockWidth, numBlocks;
    int64_t totalOffsets;   /* = blockStart[numBlocks]                           */
    int64_t numCoo;         /* COO remainder entries (0: the COO arrays unused)  */
    const void *values;
    const float *scales;    /* numBlocks, BF16_SCALED only                       */
    const int32_t *offsets;
    const int32_t *blockStart;
    const int32_t *cooRow, *cooCol;
    const void *cooVal;
    const int32_t *cooRowPtr;
} hbdia_layout_desc;
typedef struct hbdia_plan hbdia_plan;

/* A plan over the described device arrays, which it BORROWS: they must stay
 * valid and unchanged until hbdia_plan_destroy.  The arrays are checked on
 * the device first (block starts, row pointer, COO rows and columns);
 * HBDIA_ERR_INVALID_ARGUMENT / _OUT_OF_RANGE name what is malformed.  The
 * plan allocates only its per-tile COO ranges and a status word. */
int hbdia_plan_create(const hbdia_layout_desc *desc, hbdia_plan **out);
/* hbdiaSpMV on the plan (the same fused kernels and bit-identical y as
 * hbdia_spmv_device on the matrix the layout came from); x holds
 * max(numRows, numCols) elements. */
int hbdia_plan_spmv(const hbdia_plan *p, const void *x, void *y, void *stream);
/* Y = A X, row-major blocks (as hbdia_spmm_device). */
int hbdia_plan_spmm(const hbdia_plan *p, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                    void *stream);
void hbdia_plan_destroy(hbdia_plan *p);

/* hbdia_spmv_host without any device allocation.  No counterpart in the
 * reference.  For callers whose device memory belongs to another allocator
 * or budget, where the cudaMalloc that hbdia_spmv_host makes on its first
 * call could fail or stall a request.  x and y pass through one fixed
 * per-device array of the library (32 MiB), so:
 *  - max(numRows, numCols) must be <= 2^21 (HBDIA_ERR_INVALID_ARGUMENT
 *    otherwise), and the matrix must already be on the device
 *    (hbdia_matrix_prepare_gpu; HBDIA_ERR_NOT_CONVERTED otherwise);
 *  - every call shares that array: calls that overlap in time race and give
 *    undefined y, so callers serialise them;
 *  - the first call on a device does the set-up (a symbol-address lookup).
 *    With CUDA's lazy module loading (the default) that lookup loads the
 *    array's module and commits its 32 MiB on the device, so the first call
 *    can fail with HBDIA_ERR_CUDA when the device is full: make it at
 *    start-up, before other allocators take the device, and before any
 *    stream capture on that device.  Later calls commit nothing.
 * Same kernels and results as hbdia_spmv_host; synchronous. */
int hbdia_spmv_host_noalloc(hbdia_matrix *m, const void *xHost, void *yHost);

/* Blocks until the matrix's stream is idle, then reports (and clears) the
 * device status: HBDIA_ERR_DEVICE_TIMEOUT when a bounded wait inside a
 * kernel ran out since the last check (the affected y is invalid). */
int hbdia_matrix_synchronize(const hbdia_matrix *m);

/* Device status bits of the matrix's kernels (0: fine) without clearing. */
int hbdia_matrix_device_status(const hbdia_matrix *m, int32_t *bits);

/* Kernel choice for this matrix's SpMVs (hbdia_kernel). */
int hbdia_matrix_set_kernel(hbdia_matrix *m, int32_t kernel);
/* The kernel hbdia_spmv_device would launch for this x pointer. */
int hbdia_matrix_selected_kernel(const hbdia_matrix *m, const void *x, int32_t *kernel);

/* Kernel tuning knobs (used by the autotuner; results stay bit-identical).
 * HBDIA_TUNE_UNROLL: offsets in flight per lane in the staged and pipelined
 * kernels (0 = default 9, or 27).
 * HBDIA_TUNE_SPMM_TILE: right-hand sides per pass of the SpMM kernels for
 * every k (0 = autotuned / default, or 2, 4, 8, 16, 32).
 * HBDIA_TUNE_PREFETCH: 1 = the pipelined kernel asks L2 for the next
 * tile's value rows while computing the current one (bulk L2 prefetch),
 * 0 = off, -1 (default) = on when the x vector is larger than the GPU's L2;
 * for the quad kernel (which prefetches the next quad's values) always with
 * BF16 values and never with FP32 ones.
 * Measured on B200: with a 134 MB x, FP64 +1.5 % and FP32 storage +8 %; with
 * x in L2 (57 MB and below) -2 to -10 %, as the prefetched rows evict x.
 * HBDIA_TUNE_TAIL: the pipelined kernel takes a block's offsets in groups of
 * 9 (all loads of a group in flight); 1 = the offsets past the last full
 * group go in masked groups of 4 instead of one at a time, 0 = one at a time,
 * -1 (default) = masked when at least half of the stored offsets lie past
 * full groups (e.g. 7-point stencils: 7 offsets per block).  Measured on
 * B200: 7-point stencil +13-20 % (FP64), +40-49 % (FP32 storage); the masked
 * form costs 80 registers in FP64 and 14-26 % where there is no tail.
 * HBDIA_TUNE_STAGES: the staged kernel's shape, warps per CTA x stages per
 * warp: 1 = 8 x 2, 2 = 12 x 2, 3 = 16 x 2, 4 = 12 x 3, 5 = 16 x 4; 0
 * (default) = 12 x 2 for 8-byte values, 16 x 2 for 4-byte, 16 x 3 for
 * 2-byte.  A shape whose stages do not fit shared memory for the value type
 * runs the default.  Tiles with more than 32 offsets read global memory.
 * HBDIA_TUNE_QUAD_GROUP: offsets of the four blocks in flight per lane in the
 * quad kernel (0 = default: 4; or 1, 2, 4, 8). */
typedef enum hbdia_tuning_key {
    HBDIA_TUNE_UNROLL = 1,
    HBDIA_TUNE_SPMM_TILE = 2,
    HBDIA_TUNE_PREFETCH = 3,
    HBDIA_TUNE_TAIL = 4,
    HBDIA_TUNE_STAGES = 5,
    HBDIA_TUNE_QUAD_GROUP = 6
} hbdia_tuning_key;
int hbdia_matrix_set_tuning(hbdia_matrix *m, int32_t key, int32_t value);

/* Autotuner.  Times the candidate configurations of this matrix's SpMV
 * (k == 1: kernel x unroll; X, Y are x, y and ldx, ldy are ignored) or SpMM
 * (k > 1: RHS tile 4/8/16/32) on the given device buffers and stream, keeps
 * the fastest for the matrix, and records it in a process-wide table keyed on
 * (blockWidth, stored offsets per block, COO fraction, k, value type,
 * storage) so later matrices of the same class skip the timing (force != 0
 * times again).  All candidates give bit-identical results.  Overwrites Y. */
typedef struct hbdia_tune_result {
    int32_t kernel;     /* hbdia_kernel chosen for k == 1   */
    int32_t unroll;     /* HBDIA_TUNE_UNROLL value (k == 1) */
    int32_t spmmTile;   /* RHS tile (k > 1)                 */
    int32_t fromCache;  /* 1: taken from the table          */
    float msPerCall;    /* measured time of the choice      */
} hbdia_tune_result;
int hbdia_matrix_autotune(hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                          void *stream, int32_t force, hbdia_tune_result *out);
int hbdia_autotune_clear(void);

/* Time limit of every device-side wait of the staged kernel (default 2 s). */
int hbdia_matrix_set_wait_timeout(hbdia_matrix *m, uint64_t nanoseconds);

/* Test hook of the staged kernel: the warp that owns 32-row tile `tile` never
 * issues that tile's copies, so its wait runs into the time limit and the
 * kernel reports HBDIA_ERR_DEVICE_TIMEOUT at the next synchronize.  -1 turns
 * it off. */
int hbdia_matrix_test_skip_tile(hbdia_matrix *m, int32_t tile);

/* ---------------------------------------------------------------- solver */

/* Conjugate gradients for a symmetric positive definite double matrix.  No
 * counterpart in the reference (its SpMV has no solver); it runs on the same
 * SpMV kernels.  The iterations' SpMVs use the `iterStorage` copy of the
 * values (HBDIA_STORE_F32_QUAD, the fastest on B200, or HBDIA_STORE_F32: mixed
 * precision, the same iterates; a quad storage the matrix's layout cannot take
 * runs as its per-block form; HBDIA_STORE_NATIVE: plain FP64 CG); x, the residual r, the search direction, the dot products, norms and
 * the solution update are FP64.  Reliable updates: whenever the iterated
 * residual has fallen below updateFactor times the largest one since the last
 * update, and before convergence is declared, r is recomputed as b - A x with
 * the FP64 values while the search direction is kept, so the iterations do
 * not restart.  Convergence is judged on that FP64 residual.  x holds the
 * initial guess on entry and the solution on return
 * (device buffers of numRows doubles).  Synchronous. */
typedef struct hbdia_cg_options {
    double tol;            /* target ||b - A x|| / ||b|| (FP64), e.g. 1e-10              */
    double updateFactor;   /* reliable-update trigger, 0 < f < 1 (e.g. 0.1)              */
    int32_t maxUpdates;    /* FP64 residual recomputations                               */
    int32_t maxIterations; /* iterations in all                                          */
    int32_t iterStorage;   /* hbdia_value_storage of the iterations' operator            */
    int32_t checkEvery;    /* iterations per CUDA-graph replay / host check              */
} hbdia_cg_options;

typedef struct hbdia_cg_result {
    int32_t updates;           /* FP64 residual recomputations (reliable updates) */
    int32_t iterations;        /* SpMVs with the iteration operator */
    int32_t converged;
    double relResidual;        /* final ||b - A x|| / ||b|| in FP64 */
    double seconds;
} hbdia_cg_result;

int hbdia_cg_solve(hbdia_matrix *m, const double *b, double *x, const hbdia_cg_options *options, void *stream,
                   hbdia_cg_result *result);

/* ---------------------------------------------------------------- batches */

/* Many matrices computed as one unit of work.  No counterpart in the
 * reference (its hbdiaSpMV, src/Operations/HBDIASpMV.cpp:186-251, takes one
 * matrix per call); every y equals what hbdia_spmv_device / hbdia_spmm_device
 * give for that matrix alone, bit for bit.  The matrices must be on the
 * device, have blockWidth 32 and share value type and storage; they must
 * outlive the batch and keep their device layout (no further
 * hbdia_matrix_prepare_gpu) while it exists.  Two schedules:
 *  - CONCURRENT (default): each matrix's own single-matrix kernel, on a ring
 *    of auxiliary streams forked from and joined into the run's stream, so
 *    the kernels overlap on the GPU;
 *  - QUEUE: one persistent launch per segment of up to 160 matrices, warps
 *    taking 32-row tiles from an atomic counter (for many tiny matrices).
 * Runs of one batch must not overlap (they share streams and counters):
 * issue them on one stream.  Streams: NULL = the batch's own stream. */
typedef struct hbdia_batch hbdia_batch;
typedef enum hbdia_batch_schedule { HBDIA_BATCH_CONCURRENT = 0, HBDIA_BATCH_QUEUE = 1 } hbdia_batch_schedule;

int hbdia_batch_create(hbdia_matrix *const *matrices, int32_t count, hbdia_batch **out);
/* Waits only for the batch's own stream: synchronize the others first. */
void hbdia_batch_destroy(hbdia_batch *b);

/* Vectors of every matrix (device pointers): k[i] right-hand sides, X[i] an
 * x of max(numRows, numCols) elements (k[i] == 1) or a row-major
 * max(numRows, numCols) x k[i] block with leading dimension ldx[i]; Y[i] the
 * same for y.  k == NULL means 1 for all; k[i] == 0 leaves matrix i out of
 * the runs.  ldx / ldy == NULL mean k[i]; a k[i] == 1 vector is contiguous
 * (ldx[i] = ldy[i] = 1 when given).  Binding only writes host-side
 * parameter blocks: runs already enqueued keep the binding they were issued
 * with, later runs use the new one.  On an error the previous binding
 * stays. */
int hbdia_batch_bind(hbdia_batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                     const int32_t *k);

/* One run over all bound matrices, asynchronous on `stream`.  With useGraph
 * (the default) the run is a CUDA graph, made on the first run of a
 * configuration and replayed afterwards; a rebind updates it in place. */
int hbdia_batch_run(hbdia_batch *b, void *stream);

typedef struct hbdia_batch_config {
    int32_t schedule;        /* hbdia_batch_schedule (default CONCURRENT)             */
    int32_t streams;         /* CONCURRENT: auxiliary streams, 1-64 (min(16, count))  */
    int32_t threadsPerBlock; /* QUEUE: 128, 256 or 512 (default 256)                  */
    int32_t tilesPerGrab;    /* QUEUE: 32-row tiles a warp takes per atomic, 1-64 (4) */
    int32_t rhsTile;         /* QUEUE: right-hand sides per pass when k > 1: 4/8/16   */
    int32_t useGraph;        /* replay a CUDA graph (default 1)                       */
} hbdia_batch_config;

int hbdia_batch_set_config(hbdia_batch *b, const hbdia_batch_config *config);
int hbdia_batch_get_config(const hbdia_batch *b, hbdia_batch_config *config);

/* Times the configurations (CONCURRENT with 4, 16, 64 streams; QUEUE with
 * threads x tiles per grab x, when some k > 1, RHS tile) on the bound
 * vectors, on `stream`, and keeps the fastest.  The bound Y are
 * overwritten. */
int hbdia_batch_autotune(hbdia_batch *b, void *stream, float *msPerRun, int32_t *candidates);

/* count, total 32-row tiles, and the algorithmic HBM bytes of one run with
 * the current binding (per matrix: the SpMV's bytes, plus x, y and COO
 * gathers for every further right-hand side). */
int hbdia_batch_info(const hbdia_batch *b, int32_t *count, int32_t *totalTiles, int64_t *bytesPerRun);
int hbdia_batch_stream(const hbdia_batch *b, void **stream);

/* ---------------------------------------------------------------- serving */

/* A server holds resident matrices and serves requests submitted from any
 * host thread.  No counterpart in the reference.
 *  - SpMV requests (y = A x) are served by continuous batching per matrix:
 *    each matrix has its own queue and stream; whenever it has pending
 *    requests and fewer than maxInFlight batches running, up to maxRhs of
 *    them (oldest first) become one SpMM over the matrix's spmvStorage
 *    values (host vectors copied into and out of its staging columns, device
 *    vectors read and written in place); the matrices run concurrently, and
 *    requests arriving while their matrix is busy join its next batch.
 *    batching = 0 serves one request per launch in arrival order.
 *  - CG requests (solve A y = x, A symmetric positive definite) run on
 *    cgWorkers worker threads: CG with reliable updates (hbdia_cg_solve)
 *    iterating on the cgIterStorage values, converged to cgTol on the FP64
 *    residual.  With cgMaxGroup > 1 a worker takes the oldest CG request
 *    together with the other pending CG requests on the same matrix (up to
 *    cgMaxGroup) and solves them in lockstep: one SpMM per iteration reads
 *    each stored value once for all of them, and each solve keeps its own
 *    schedule, so its result is the one it gives alone, bit for bit.
 * A request's result does not depend on the requests it is served with.
 * Admission: hbdia_server_add_matrix returns HBDIA_ERR_NO_MEMORY when the
 * matrix's plans, staging blocks and CG workspace growth would take the
 * server's device memory past memoryBudget.  Host vectors must stay valid
 * until the request is collected; page-locked memory is fastest. */
typedef struct hbdia_server hbdia_server;
typedef enum hbdia_request_kind { HBDIA_REQ_SPMV = 0, HBDIA_REQ_CG = 1 } hbdia_request_kind;

typedef struct hbdia_server_options {
    int64_t memoryBudget;   /* device bytes the server may hold (default 150e9)             */
    int32_t batching;       /* continuous batching of SpMVs (default 1)                     */
    int32_t maxRhs;         /* SpMV requests of one matrix per batch, 1-64 (default 16)    */
    int32_t spmvStorage;    /* hbdia_value_storage of SpMVs (default HBDIA_STORE_F32;       */
                            /* not the quad-interleaved ones: batches are SpMMs)            */
    int32_t cgIterStorage;  /* storage of the CG iterations' SpMVs (default                 */
                            /* HBDIA_STORE_F32_QUAD; one other than spmvStorage is kept as  */
                            /* a second reduced copy)                                       */
    int32_t cgWorkers;      /* concurrent CG solves, 1-64 (default 4)                       */
    int32_t cgMaxUpdates;   /* FP64 residual recomputations per solve (default 100)         */
    int32_t cgMaxIterations;/* iterations per solve (default 20000)                         */
    int32_t cgCheckEvery;   /* iterations per graph replay (default 10)                     */
    double cgTol;           /* target ||b - A y|| / ||b|| (default 1e-10)                   */
    double cgUpdateFactor;  /* reliable-update trigger (default 0.1)                        */
    int32_t maxInFlight;    /* SpMV batches of one matrix issued and not yet completed,     */
                            /* 1-8 (default 1: the next batch forms while one runs)         */
    int32_t cgMaxGroup;     /* pending CG requests on one matrix solved as one lockstep     */
                            /* group, 1-16 (default 1: every solve on its own)              */
} hbdia_server_options;

typedef struct hbdia_request_info {
    int32_t status;         /* hbdia_status of the request (CG: RUNTIME if not converged) */
    int32_t kind, matrix;
    int32_t batchRhs;       /* SpMV: requests in its batch                               */
    double submitted, started, finished; /* seconds since the server was created         */
    int32_t cgUpdates, cgIterations;
    double cgRelResidual;
} hbdia_request_info;

typedef struct hbdia_server_stats {
    int64_t completed, spmvRequests, cgRequests;
    int64_t spmvSteps, spmvLaunches; /* scheduler passes that issued batches; batches */
    int64_t deviceBytes;    /* held under the budget */
    int32_t matrices;
    int64_t cgGroups;       /* lockstep CG groups solved (cgRequests / cgGroups: mean group) */
} hbdia_server_stats;

void hbdia_server_default_options(hbdia_server_options *options);
int hbdia_server_create(const hbdia_server_options *options, hbdia_server **out);
/* Serves everything pending, then stops. */
void hbdia_server_destroy(hbdia_server *s);
/* Makes a converted double matrix (host layout present) resident; the
 * server builds its own device copies, so the matrix may be destroyed
 * afterwards. */
int hbdia_server_add_matrix(hbdia_server *s, const hbdia_matrix *m, int32_t *id);
/* x: numCols doubles (the right-hand side b for CG); y: numRows doubles. */
int hbdia_server_submit(hbdia_server *s, int32_t matrix, int32_t kind, const double *xHost, double *yHost,
                        uint64_t *ticket);
/* The same request on device buffers (this process's current device):
 * read and written in place, no host copies.  A step's device SpMV requests
 * on one matrix run as one vector-list SpMM (hbdia_spmv_list_device); a
 * device CG request solves with b = xDevice into yDevice.  Both buffers must
 * stay valid and untouched until hbdia_server_wait returns. */
int hbdia_server_submit_device(hbdia_server *s, int32_t matrix, int32_t kind, const double *xDevice,
                               double *yDevice, uint64_t *ticket);
/* paused != 0: requests queue up but no SpMV step or CG solve starts (work
 * already running finishes); 0 resumes, and everything queued is served --
 * the SpMVs of the backlog batched together.  Waiting on an unfinished
 * request while paused fails with HBDIA_ERR_RUNTIME. */
int hbdia_server_pause(hbdia_server *s, int32_t paused);
/* Blocks until the request is done and collects it (once per ticket). */
int hbdia_server_wait(hbdia_server *s, uint64_t ticket, hbdia_request_info *info);
int hbdia_server_get_stats(hbdia_server *s, hbdia_server_stats *stats);

/* ---------------------------------------------------------------- workloads */

/* Seeded synthetic 27-point stencil on an nx*ny*nz grid (Dirichlet boundary,
 * index k*nx*ny + j*nx + i), centre value `center`, the 26 neighbours
 * `neighbor`, plus floor(extraFraction * stencil_nnz) extra entries at
 * uniformly drawn (row, col) positions outside the row's stencil pattern,
 * without repeats, values uniform in [extraLo, extraHi).  Output is row-sorted;
 * within a row the stencil entries come in ascending column order, then the
 * row's extras in draw order.  Call once with rows == NULL to get *nnz, then
 * again with arrays of that size. */
int hbdia_generate_stencil27(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor,
                             double extraFraction, double extraLo, double extraHi, uint64_t seed,
                             int64_t *nnz, int32_t *rows, int32_t *cols, double *values);

/* Same for the 7-point stencil (faces only). */
int hbdia_generate_stencil7(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor,
                            int64_t *nnz, int32_t *rows, int32_t *cols, double *values);

/* Banded matrix of order n with the given diagonal offsets: off-diagonal
 * values uniform in [lo, hi), each entry dropped with probability dropProb,
 * centre = |row sum| + 1 when offset 0 is listed, plus floor(scatterFraction
 * * band_nnz) scattered entries.  Row-sorted.  Two-call protocol as above. */
int hbdia_generate_banded(int32_t n, const int32_t *offsets, int32_t numOffsets, double lo,
                          double hi, double dropProb, double scatterFraction, uint64_t seed,
                          int64_t *nnz, int32_t *rows, int32_t *cols, double *values);

/* Symmetric positive definite 27-point stencil: off-diagonal a_ij = a_ji =
 * -(0.5 + u), u in [0, 1) drawn from a hash of the unordered pair (i, j) and
 * the seed, plus floor(extraFraction * stencil_nnz / 2) symmetric pairs
 * outside the 27-point pattern (distinct, seeded), diagonal
 * (1 + shift) * sum_j |a_ij| (shift >= 0): diagonally dominant, so SPD.
 * Row-sorted, ascending columns.  Two-call protocol as above. */
int hbdia_generate_stencil27_spd(int32_t nx, int32_t ny, int32_t nz, double shift, double extraFraction,
                                 uint64_t seed, int64_t *nnz, int32_t *rows, int32_t *cols, double *values);

/* n doubles uniform in [lo, hi) from the library's seeded generator. */
int hbdia_fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed);

/* ---- Row-partitioned distribution (one rank per GPU) -------------------
 *
 * A partial matrix holds one rank's contiguous rows of a square matrix: local
 * row indices, GLOBAL column indices, offsets col - globalRow.  After
 * hbdia_matrix_convert it also holds the reference's partial-matrix metadata
 * (the x ranges it reads and which rank owns each), and its device plan reads
 * x through a dense window of global columns [windowStart, windowStart +
 * windowLength): x_window[c - windowStart] = x[c].  The window holds the
 * rank's own x entries at [globalRowStart - windowStart, ... + numRows) and
 * the other ranks' entries at their data ranges; hbdia_spmv_device(m, x_window,
 * y_local, stream) then computes the rank's rows of y. */

/* HBDIA<T>(rows, cols, vals, numRows, numCols, globalRowMapping, partialMatrix=true,
 * numGlobalRows, numGlobalCols, numGlobalNonZeros, rank, size)
 * (src/Format/HBDIA.cpp:118-154) with the contiguous mapping global row =
 * globalRowStart + local row (the mapping BasicExtractor builds).  rows are
 * local (< numLocalRows), cols global (< numGlobalCols); the matrix must be
 * square (numGlobalRows == numGlobalCols) and globalRowStart + numLocalRows
 * <= numGlobalRows. */
int hbdia_matrix_create_partial(hbdia_dtype dtype, const int32_t *rows, const int32_t *cols,
                                const void *values, int64_t nnz, int32_t numLocalRows,
                                int32_t numGlobalRows, int32_t numGlobalCols, int64_t numGlobalNonZeros,
                                int32_t globalRowStart, int32_t rank, int32_t size, hbdia_matrix **out);

/* BasicExtractor::createMatrixPartitions + partitionRowWise
 * (src/DataExchange/BasicExtractor.cpp:16-45, 124-234) for one partition:
 * rows [part * (n / numProcesses), ...), the last partition taking n %
 * numProcesses more, entries in input order.  The result is a partial matrix
 * (rank = part, size = numProcesses).  Needs a square matrix with entries and
 * numProcesses <= numRows. */
int hbdia_matrix_partition(const hbdia_matrix *global, int32_t numProcesses, int32_t part, hbdia_matrix **out);

typedef struct hbdia_partial_info {
    int32_t isPartial;          /* isPartialMatrix (include/Format/HBDIA.hpp:126)        */
    int32_t hasMetadata;        /* metadata computed (after conversion)                  */
    int32_t globalRowStart;     /* getGlobalRowIndex(0)                                  */
    int32_t numGlobalRows;      /* getNumGlobalRows                                      */
    int32_t numGlobalCols;      /* getNumGlobalCols                                      */
    int32_t rank, size;
    int64_t numGlobalNonZeros;  /* getNumGlobalNonZeros                                  */
    int64_t numDataRanges;      /* getDataRanges().size() (analyzeDataRanges)           */
    int64_t numProcessRanges;   /* segments of processDataRanges, all processes          */
    int64_t totalBufferSize;    /* PartialMatrixMetadata::totalBufferSize                */
    int64_t leftBufferSize;     /* HBDIAVector(localData, matrix, rank, size) receive    */
    int64_t rightBufferSize;    /*   buffers (src/Format/HBDIAVector.cpp:39-66)          */
    int32_t windowStart;        /* this library's x window                              */
    int32_t windowLength;
} hbdia_partial_info;
int hbdia_matrix_partial_info(const hbdia_matrix *m, hbdia_partial_info *info);

/* dataRanges: numDataRanges pairs [start, end) -- HBDIA::analyzeDataRanges
 * (src/Format/HBDIA.cpp:1333-1414); processRanges: numProcessRanges triples
 * (process, start, end) -- BasicExtractor::extractPartialMatrixMetadataRowWise
 * (src/DataExchange/BasicExtractor.cpp:269-333), grouped by process in the
 * reference's order.  Either pointer may be NULL. */
int hbdia_matrix_export_ranges(const hbdia_matrix *m, int32_t *dataRanges, int32_t *processRanges);

/* Halo copy plan: numSegments element segments (src[srcOffset .. +length) ->
 * dst[dstOffset .. +length)) between a source buffer of srcLength and a
 * destination of dstLength elements of elemBytes (4 or 8), validated and
 * uploaded once.  hbdia_halo_copy runs them as one kernel on the stream:
 * allocation-free, graph-capturable.  It replaces the per-range packing of
 * MPICommunicator::exchangeData (src/DataExchange/MPICommunicator.cpp:253-412):
 * the ranges a peer requested are packed into one send buffer, and the
 * received buffer is unpacked into the x window. */
typedef struct hbdia_halo hbdia_halo;
int hbdia_halo_create(int32_t elemBytes, const int64_t *srcOffset, const int64_t *dstOffset,
                      const int64_t *length, int32_t numSegments, int64_t srcLength, int64_t dstLength,
                      hbdia_halo **out);
int hbdia_halo_copy(const hbdia_halo *h, const void *src, void *dst, void *stream);
int64_t hbdia_halo_elements(const hbdia_halo *h);
void hbdia_halo_destroy(hbdia_halo *h);

#ifdef __cplusplus
}
#endif

#endif /* HBDIA_B200_H */
