// Test infrastructure only: C entry points around the reference's OWN code.
//
// This translation unit is compiled by oracle/Makefile together with the
// reference's unmodified sources (src/Format/HBDIA.cpp, HBDIAPrinter.cpp,
// HBDIAVector.cpp, src/Operations/HBDIASpMV.cu) into oracle/_ref/libhbdia_ref.so.
// It includes src/Operations/HBDIASpMV.cpp so that the file-local template
// cpu_coo_spmv_kernel (src/Operations/HBDIASpMV.cpp:36-99) is reachable, and
// links src/DataExchange/BasicExtractor.cpp for the row partitioning.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
// arm load this library, and only as the checker or the timed CPU baseline.
// The product path (hbdia_b200) never links or calls it.
//
// GPU-free conversion: the reference's convertToHBDIAFormat ends in
// prepareForGPU() (cudaMalloc) for non-partial matrices
// (src/Format/HBDIA.cpp:715-717).  Constructing with the partial-matrix
// constructor and an EMPTY global row mapping (src/Format/HBDIA.cpp:118-154)
// skips that call while the offset arithmetic stays identical
// (src/Format/HBDIA.cpp:546-552: globalRow == localRow when the mapping is
// empty), so the layout can be produced on a host without a GPU.

#include "src/Operations/HBDIASpMV.cpp"
#include "include/DataExchange/BasicExtractor.hpp"

#include <cstring>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

extern "C" void *numa_alloc_onnode(size_t, int) {
    std::fprintf(stderr, "oracle: numa_alloc_onnode is not available in the oracle build\n");
    return nullptr;
}

namespace {

template <typename T>
HBDIA<T> *make_matrix(const int *rows, const int *cols, const T *vals, int64_t nnz,
                      int numRows, int numCols, int partial) {
    std::vector<int> r(rows, rows + nnz), c(cols, cols + nnz);
    std::vector<T> v(vals, vals + nnz);
    if (numRows <= 0 || numCols <= 0) {
        // dims-inferring constructor, src/Format/HBDIA.cpp:23-49
        return new HBDIA<T>(r, c, v);
    }
    if (partial) {
        return new HBDIA<T>(r, c, v, numRows, numCols, std::vector<int>{}, true,
                            numRows, numCols, static_cast<int>(nnz));
    }
    return new HBDIA<T>(r, c, v, numRows, numCols);
}

template <typename T>
void sizes(const HBDIA<T> *m, int64_t *out) {
    const auto &opb = m->getOffsetsPerBlock();
    int64_t total = 0;
    for (const auto &b : opb) total += static_cast<int64_t>(b.size());
    out[0] = static_cast<int64_t>(opb.size());
    out[1] = total;
    out[2] = static_cast<int64_t>(m->getHBDIAData().size());
    out[3] = static_cast<int64_t>(m->getCpuValues().size());
    out[4] = m->getHasHBDIA() ? m->getNumberDiagonals() : 0;
    out[5] = static_cast<int64_t>(m->getHistogramBlocks().size());
    out[6] = m->getHasHBDIA() ? 1 : 0;
    out[7] = m->getNumRows();
    out[8] = m->getNumCols();
    out[9] = static_cast<int64_t>(m->getCpuRowPtr().size());
}

template <typename T>
void export_layout(const HBDIA<T> *m, int *offsets, int *blockStart, T *data, int *cooRow,
                   int *cooCol, T *cooVal, int *cooRowPtr, int *histBlocks, int *histNnz) {
    const auto &opb = m->getOffsetsPerBlock();
    int64_t pos = 0;
    for (size_t b = 0; b < opb.size(); ++b) {
        blockStart[b] = static_cast<int>(pos);
        for (int o : opb[b]) offsets[pos++] = o;
    }
    blockStart[opb.size()] = static_cast<int>(pos);
    const auto &d = m->getHBDIAData();
    if (!d.empty()) std::memcpy(data, d.data(), d.size() * sizeof(T));
    const auto &cr = m->getCpuRowIndices();
    const auto &cc = m->getCpuColIndices();
    const auto &cv = m->getCpuValues();
    if (!cr.empty()) {
        std::memcpy(cooRow, cr.data(), cr.size() * sizeof(int));
        std::memcpy(cooCol, cc.data(), cc.size() * sizeof(int));
        std::memcpy(cooVal, cv.data(), cv.size() * sizeof(T));
    }
    const auto &rp = m->getCpuRowPtr();
    if (!rp.empty()) std::memcpy(cooRowPtr, rp.data(), rp.size() * sizeof(int));
    const auto &hb = m->getHistogramBlocks();
    const auto &hn = m->getHistogramNnz();
    if (!hb.empty()) std::memcpy(histBlocks, hb.data(), hb.size() * sizeof(int));
    if (!hn.empty()) std::memcpy(histNnz, hn.data(), hn.size() * sizeof(int));
}

template <typename T>
struct CooHolder {
    std::vector<int> rows, cols;
    std::vector<T> vals;
};

}  // namespace

extern "C" {

// ---- HBDIA<T> construction + convertToHBDIAFormat (src/Format/HBDIA.cpp:507-718)
void *ref_matrix_create_f64(const int *rows, const int *cols, const double *vals, int64_t nnz,
                            int numRows, int numCols, int partial) {
    try {
        return make_matrix<double>(rows, cols, vals, nnz, numRows, numCols, partial);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference ctor threw: %s\n", e.what());
        return nullptr;
    }
}
void *ref_matrix_create_f32(const int *rows, const int *cols, const float *vals, int64_t nnz,
                            int numRows, int numCols, int partial) {
    try {
        return make_matrix<float>(rows, cols, vals, nnz, numRows, numCols, partial);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference ctor threw: %s\n", e.what());
        return nullptr;
    }
}
int ref_matrix_convert_f64(void *h, int bw, int thr, int maxCoo, int cooUnique) {
    auto *m = static_cast<HBDIA<double> *>(h);
    m->convertToHBDIAFormat(bw, thr, maxCoo, cooUnique != 0, ExecutionMode::GPU_COO);
    return m->getHasHBDIA() ? 1 : 0;
}
int ref_matrix_convert_f32(void *h, int bw, int thr, int maxCoo, int cooUnique) {
    auto *m = static_cast<HBDIA<float> *>(h);
    m->convertToHBDIAFormat(bw, thr, maxCoo, cooUnique != 0, ExecutionMode::GPU_COO);
    return m->getHasHBDIA() ? 1 : 0;
}
void ref_matrix_sizes_f64(void *h, int64_t *out) { sizes(static_cast<HBDIA<double> *>(h), out); }
void ref_matrix_sizes_f32(void *h, int64_t *out) { sizes(static_cast<HBDIA<float> *>(h), out); }
void ref_matrix_export_f64(void *h, int *offsets, int *blockStart, double *data, int *cooRow,
                           int *cooCol, double *cooVal, int *cooRowPtr, int *histBlocks,
                           int *histNnz) {
    export_layout(static_cast<HBDIA<double> *>(h), offsets, blockStart, data, cooRow, cooCol,
                  cooVal, cooRowPtr, histBlocks, histNnz);
}
void ref_matrix_export_f32(void *h, int *offsets, int *blockStart, float *data, int *cooRow,
                           int *cooCol, float *cooVal, int *cooRowPtr, int *histBlocks,
                           int *histNnz) {
    export_layout(static_cast<HBDIA<float> *>(h), offsets, blockStart, data, cooRow, cooCol,
                  cooVal, cooRowPtr, histBlocks, histNnz);
}
// ---- convertToDIAFormat / removeCOODuplicates (src/Format/HBDIA.cpp:372-505)
void ref_matrix_remove_dups_f64(void *h) { static_cast<HBDIA<double> *>(h)->removeCOODuplicates(); }
void ref_matrix_convert_dia_f64(void *h, int cooUnique) {
    static_cast<HBDIA<double> *>(h)->convertToDIAFormat(cooUnique != 0);
}
// out: numDiagonals, diagonal length, numNonZeros, COO entries, isDIAFormat
void ref_matrix_dia_sizes_f64(void *h, int64_t *out) {
    auto *m = static_cast<HBDIA<double> *>(h);
    const auto &d = m->getDiagonals();
    out[0] = static_cast<int64_t>(m->getOffsets().size());
    out[1] = d.empty() ? 0 : static_cast<int64_t>(d[0].size());
    out[2] = m->getNumNonZeros();
    out[3] = static_cast<int64_t>(m->getValues().size());
    out[4] = m->getHasDIA() ? 1 : 0;
}
void ref_matrix_export_dia_f64(void *h, int *offsets, double *diagonals, int *rows, int *cols, double *vals) {
    auto *m = static_cast<HBDIA<double> *>(h);
    const auto &o = m->getOffsets();
    const auto &d = m->getDiagonals();
    std::copy(o.begin(), o.end(), offsets);
    size_t p = 0;
    for (const auto &diag : d)
        for (double v : diag) diagonals[p++] = v;
    std::copy(m->getRowIndices().begin(), m->getRowIndices().end(), rows);
    std::copy(m->getColIndices().begin(), m->getColIndices().end(), cols);
    std::copy(m->getValues().begin(), m->getValues().end(), vals);
}
void ref_matrix_destroy_f64(void *h) { delete static_cast<HBDIA<double> *>(h); }
void ref_matrix_destroy_f32(void *h) { delete static_cast<HBDIA<float> *>(h); }

// COO export of the matrix's own input arrays (after create3DStencil27Point / loadMTX).
void ref_coo_sizes_f64(void *h, int64_t *out) {
    auto *m = static_cast<HBDIA<double> *>(h);
    out[0] = static_cast<int64_t>(m->getValues().size());
    out[1] = m->getNumRows();
    out[2] = m->getNumCols();
}
void ref_coo_export_f64(void *h, int *rows, int *cols, double *vals) {
    auto *m = static_cast<HBDIA<double> *>(h);
    const auto &r = m->getRowIndices();
    const auto &c = m->getColIndices();
    const auto &v = m->getValues();
    if (r.empty()) return;
    std::memcpy(rows, r.data(), r.size() * sizeof(int));
    std::memcpy(cols, c.data(), c.size() * sizeof(int));
    std::memcpy(vals, v.data(), v.size() * sizeof(double));
}

// create3DStencil27Point (src/Format/HBDIA.cpp:1416-1607)
void *ref_stencil27_f64(int nx, int ny, int nz, double noise, int iteration) {
    auto *m = new HBDIA<double>();
    m->create3DStencil27Point(nx, ny, nz, noise, iteration);
    return m;
}

// loadMTX (src/Format/HBDIA.cpp:161-263)
void *ref_load_mtx_f64(const char *path, int *ok) {
    auto *m = new HBDIA<double>();
    *ok = m->loadMTX(std::string(path)) ? 1 : 0;
    return m;
}

// ---- the reference's CPU COO SpMV, cpu_coo_spmv_kernel<T> (src/Operations/HBDIASpMV.cpp:36-99)
void *ref_cpu_coo_create_f64(const int *rows, const int *cols, const double *vals, int64_t nnz) {
    auto *h = new CooHolder<double>();
    h->rows.assign(rows, rows + nnz);
    h->cols.assign(cols, cols + nnz);
    h->vals.assign(vals, vals + nnz);
    return h;
}
void *ref_cpu_coo_create_f32(const int *rows, const int *cols, const float *vals, int64_t nnz) {
    auto *h = new CooHolder<float>();
    h->rows.assign(rows, rows + nnz);
    h->cols.assign(cols, cols + nnz);
    h->vals.assign(vals, vals + nnz);
    return h;
}
void ref_cpu_coo_spmv_f64(void *h, const double *x, int numRows, double *y) {
    auto *c = static_cast<CooHolder<double> *>(h);
    cpu_coo_spmv_kernel<double>(c->rows, c->cols, c->vals, x, numRows, y);
}
void ref_cpu_coo_spmv_f32(void *h, const float *x, int numRows, float *y) {
    auto *c = static_cast<CooHolder<float> *>(h);
    cpu_coo_spmv_kernel<float>(c->rows, c->cols, c->vals, x, numRows, y);
}
void ref_cpu_coo_destroy_f64(void *h) { delete static_cast<CooHolder<double> *>(h); }
void ref_cpu_coo_destroy_f32(void *h) { delete static_cast<CooHolder<float> *>(h); }
int ref_omp_max_threads(void) { return omp_get_max_threads(); }
void ref_omp_set_threads(int n) { omp_set_num_threads(n); }

// ---- the reference's own GPU path, hbdiaSpMV (src/Operations/HBDIASpMV.cpp:186-251).
// Needs a GPU.  Builds a NON-partial matrix so convertToHBDIAFormat uploads
// (prepareForGPU), then runs one hbdiaSpMV and reads y back.  y starts at 0,
// as in every reference caller (simple_hbdia_example.cpp:27).
int ref_gpu_spmv_f64(const int *rows, const int *cols, const double *vals, int64_t nnz,
                     int numRows, int numCols, int bw, int thr, const double *x, double *y,
                     int execCOOCPU, int execCOOGPU) {
    try {
        HBDIA<double> m(std::vector<int>(rows, rows + nnz), std::vector<int>(cols, cols + nnz),
                        std::vector<double>(vals, vals + nnz), numRows, numCols);
        m.convertToHBDIAFormat(bw, thr);
        if (execCOOGPU) m.initializeCuSparse();
        HBDIAVector<double> vx(std::vector<double>(x, x + numRows));
        HBDIAVector<double> vy(std::vector<double>(numRows, 0.0));
        hbdiaSpMV<double>(m, vx, vy, execCOOCPU != 0, execCOOGPU != 0);
        if (cudaDeviceSynchronize() != cudaSuccess) return -3;
        if (cudaMemcpy(y, vy.getDeviceLocalPtr(), sizeof(double) * numRows,
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            return -3;
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference hbdiaSpMV threw: %s\n", e.what());
        return -1;
    }
}

// ---- a matrix converted by the reference on a GPU (convertToHBDIAFormat ends in
// prepareForGPU for non-partial matrices, src/Format/HBDIA.cpp:715-717): its own
// device arrays, and its own hbdiaSpMV on them
void *ref_gpu_matrix_f64(const int *rows, const int *cols, const double *vals, int64_t nnz, int numRows,
                         int numCols, int bw, int thr) {
    try {
        auto *m = new HBDIA<double>(std::vector<int>(rows, rows + nnz), std::vector<int>(cols, cols + nnz),
                                    std::vector<double>(vals, vals + nnz), numRows, numCols);
        m->convertToHBDIAFormat(bw, thr);
        return m;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference conversion threw: %s\n", e.what());
        return nullptr;
    }
}

// sizes: numBlocks, totalOffsets, numCoo; ptrs: values, offsets, blockStart, cooRow, cooCol, cooVal, cooRowPtr
void ref_gpu_matrix_arrays_f64(void *h, int64_t *sizes, const void **ptrs) {
    const auto *m = static_cast<const HBDIA<double> *>(h);
    int64_t total = 0;
    for (const auto &b : m->getOffsetsPerBlock()) total += static_cast<int64_t>(b.size());
    sizes[0] = m->getNumBlocks();
    sizes[1] = total;
    sizes[2] = static_cast<int64_t>(m->getCpuValues().size());
    ptrs[0] = m->getHBDIADataDevice();
    ptrs[1] = m->getFlattenedOffsetsDevice();
    ptrs[2] = m->getBlockStartIndicesDevice();
    ptrs[3] = m->getCpuRowIndicesDevice();
    ptrs[4] = m->getCpuColIndicesDevice();
    ptrs[5] = m->getCpuValuesDevice();
    ptrs[6] = m->getCpuRowPtrDevice();
}

int ref_gpu_matrix_spmv_f64(void *h, const double *x, double *y, int execCOOCPU) {
    try {
        auto &m = *static_cast<HBDIA<double> *>(h);
        const int n = m.getNumRows();
        HBDIAVector<double> vx(std::vector<double>(x, x + n));
        HBDIAVector<double> vy(std::vector<double>(n, 0.0));
        hbdiaSpMV<double>(m, vx, vy, execCOOCPU != 0, false);
        if (cudaDeviceSynchronize() != cudaSuccess) return -3;
        if (cudaMemcpy(y, vy.getDeviceLocalPtr(), sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return -3;
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference hbdiaSpMV threw: %s\n", e.what());
        return -1;
    }
}

// ---- row partitioning, as BasicDistributor::scatterMatrix / receiveMatrix do
// it for one rank (src/DataExchange/BasicDistributor.cpp:17-146): the
// extractor's partition, the partial-matrix constructor, convertToHBDIAFormat,
// analyzeDataRanges and extractPartialMatrixMetadata -- all host code.
struct RefPartition {
    HBDIA<double> *m = nullptr;
    std::vector<int> rows, cols;
    std::vector<double> vals;
    int rowStart = 0, numLocalRows = 0;
    std::vector<std::tuple<int, int>> data;
    std::vector<std::vector<std::tuple<int, int>>> proc;
    int total = 0;
};

void *ref_partition_f64(const int *rows, const int *cols, const double *vals, int64_t nnz, int n, int P,
                        int part, int bw, int thr) {
    try {
        HBDIA<double> g(std::vector<int>(rows, rows + nnz), std::vector<int>(cols, cols + nnz),
                        std::vector<double>(vals, vals + nnz), n, n);
        BasicExtractor<double> ex;
        if (!ex.createMatrixPartitions(g, P)) return nullptr;
        const auto &pt = ex.getPartitions()[part];
        const auto &md = ex.getMatrixData()[part];
        auto *h = new RefPartition();
        h->rows = pt.localRowIndices;
        h->cols = pt.localColIndices;
        h->vals = pt.localValues;
        h->rowStart = pt.globalRowMapping.empty() ? 0 : pt.globalRowMapping[0];
        h->numLocalRows = md.numLocalRows;
        h->m = new HBDIA<double>(pt.localRowIndices, pt.localColIndices, pt.localValues, md.numLocalRows,
                                 md.numLocalCols, pt.globalRowMapping, true, md.numGlobalRows, md.numGlobalCols,
                                 md.numGlobalNonZeros, part, P);
        h->m->convertToHBDIAFormat(bw, thr);
        h->m->analyzeDataRanges();
        ex.extractPartialMatrixMetadata(*h->m, P);
        const auto &meta = h->m->getPartialMatrixMetadata();
        h->data = meta.dataRanges;
        h->proc = meta.processDataRanges;
        h->total = meta.totalBufferSize;
        return h;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "oracle: reference partitioning threw: %s\n", e.what());
        return nullptr;
    }
}

// out: rowStart, numLocalRows, local nnz, #data ranges, #process segments, totalBufferSize
void ref_partition_sizes(void *hp, int64_t *out) {
    auto *h = static_cast<RefPartition *>(hp);
    int64_t segs = 0;
    for (const auto &v : h->proc) segs += static_cast<int64_t>(v.size());
    out[0] = h->rowStart;
    out[1] = h->numLocalRows;
    out[2] = static_cast<int64_t>(h->vals.size());
    out[3] = static_cast<int64_t>(h->data.size());
    out[4] = segs;
    out[5] = h->total;
}

void ref_partition_export(void *hp, int *rows, int *cols, double *vals, int *data, int *proc) {
    auto *h = static_cast<RefPartition *>(hp);
    if (!h->vals.empty()) {
        std::memcpy(rows, h->rows.data(), h->rows.size() * sizeof(int));
        std::memcpy(cols, h->cols.data(), h->cols.size() * sizeof(int));
        std::memcpy(vals, h->vals.data(), h->vals.size() * sizeof(double));
    }
    for (size_t i = 0; i < h->data.size(); ++i) {
        data[2 * i] = std::get<0>(h->data[i]);
        data[2 * i + 1] = std::get<1>(h->data[i]);
    }
    size_t k = 0;
    for (size_t p = 0; p < h->proc.size(); ++p)
        for (const auto &t : h->proc[p]) {
            proc[3 * k] = static_cast<int>(p);
            proc[3 * k + 1] = std::get<0>(t);
            proc[3 * k + 2] = std::get<1>(t);
            ++k;
        }
}

void *ref_partition_matrix(void *hp) { return static_cast<RefPartition *>(hp)->m; }

void ref_partition_destroy(void *hp) {
    auto *h = static_cast<RefPartition *>(hp);
    delete h->m;
    delete h;
}

}  // extern "C"
