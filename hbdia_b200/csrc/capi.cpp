// The C ABI (include/hbdia_b200.h): matrix and vector handles, conversion,
// SpMV entry points and workload generators.  Exceptions never cross the ABI;
// they become hbdia_status codes with a per-thread message.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "handles.hpp"
#include "hbdia_internal.hpp"

using hbdia::Error;

struct hbdia_batch {
    hbdia::Batch *B = nullptr;
};

struct hbdia_server {
    hbdia::Server *S = nullptr;
};

struct hbdia_halo {
    hbdia::Halo *H = nullptr;
};

struct hbdia_plan {
    hbdia::DevicePlan P;
};

namespace {

thread_local std::string g_err;

void set_err(const char *m) { g_err = m ? m : ""; }

template <typename F>
int guarded(F &&f) {
    try {
        f();
        g_err.clear();
        return HBDIA_OK;
    } catch (const Error &e) {
        set_err(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_err("out of host memory");
        return HBDIA_ERR_NO_MEMORY;
    } catch (const std::exception &e) {
        set_err(e.what());
        return HBDIA_ERR_RUNTIME;
    }
}

size_t esize(int32_t dtype) { return dtype == HBDIA_F32 ? sizeof(float) : sizeof(double); }

void need(bool ok, int status, const char *msg) {
    if (!ok) throw Error(status, msg);
}

int64_t coo_nnz(const hbdia_matrix *m) {
    return m->dtype == HBDIA_F32 ? static_cast<int64_t>(m->c32.vals.size())
                                 : static_cast<int64_t>(m->c64.vals.size());
}
int32_t num_rows(const hbdia_matrix *m) { return m->dtype == HBDIA_F32 ? m->c32.numRows : m->c64.numRows; }
int32_t num_cols(const hbdia_matrix *m) { return m->dtype == HBDIA_F32 ? m->c32.numCols : m->c64.numCols; }

template <typename T>
void fill_coo(hbdia::Coo<T> &c, const int32_t *r, const int32_t *col, const void *v, int64_t nnz,
              int32_t nR, int32_t nC) {
    // HBDIA(rows, cols, vals[, numRows, numCols]) (src/Format/HBDIA.cpp:23-80)
    need(nnz >= 0, HBDIA_ERR_INVALID_ARGUMENT, "nnz must be non-negative");
    need(nnz == 0 || (r && col && v), HBDIA_ERR_INVALID_ARGUMENT, "null COO array");
    if (nnz > 2147483647LL) throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^31-1 entries");
    const bool infer = nR <= 0 && nC <= 0;
    if (!infer && (nR <= 0 || nC <= 0))
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "Matrix dimensions must be positive");
    c.rows.assign(r, r + nnz);
    c.cols.assign(col, col + nnz);
    c.vals.assign(static_cast<const T *>(v), static_cast<const T *>(v) + nnz);
    c.nnzPerRow.clear();
    if (infer) {
        int32_t mr = 0, mc = 0;
        for (int64_t i = 0; i < nnz; ++i) {
            // the reference does not check signs here; a negative index has no
            // place in the layout, so it is rejected like an out-of-range one
            if (r[i] < 0 || col[i] < 0)
                throw Error(HBDIA_ERR_OUT_OF_RANGE, "negative index at entry " + std::to_string(i));
            mr = std::max(mr, r[i] + 1);
            mc = std::max(mc, col[i] + 1);
        }
        c.numRows = mr;
        c.numCols = mc;
        return;
    }
    for (int64_t i = 0; i < nnz; ++i) {
        if (r[i] < 0 || r[i] >= nR)
            throw Error(HBDIA_ERR_OUT_OF_RANGE, "Row index " + std::to_string(r[i]) +
                                                     " is out of range [0, " + std::to_string(nR - 1) + "]");
        if (col[i] < 0 || col[i] >= nC)
            throw Error(HBDIA_ERR_OUT_OF_RANGE, "Column index " + std::to_string(col[i]) +
                                                     " is out of range [0, " + std::to_string(nC - 1) + "]");
    }
    c.numRows = nR;
    c.numCols = nC;
}

void free_host_pipeline(hbdia_matrix *m) {
    for (int d = 0; d < hbdia_matrix::kHostDepth; ++d) {
        if (m->pipeX[d]) cudaFree(m->pipeX[d]);
        if (m->pipeY[d]) cudaFree(m->pipeY[d]);
        if (m->pipeStream[d]) cudaStreamDestroy(static_cast<cudaStream_t>(m->pipeStream[d]));
        m->pipeX[d] = m->pipeY[d] = m->pipeStream[d] = nullptr;
    }
}

// The public storage code of a plan (hbdia_value_storage).
int32_t plan_storage_code(const hbdia::DevicePlan &P) {
    if (!P.quadLayout) return P.storage;
    return P.storage == HBDIA_STORE_F32 ? HBDIA_STORE_F32_QUAD : HBDIA_STORE_BF16_QUAD;
}

void free_block_sizes(hbdia_matrix *m) {
    if (m->blockSizesDev) cudaFree(m->blockSizesDev);
    m->blockSizesDev = nullptr;
}

void reset_hbdia(hbdia_matrix *m) {
    free_host_pipeline(m);
    free_block_sizes(m);
    hbdia::free_plan(m->plan);
    hbdia::free_plan(m->innerPlan);
    hbdia::cg_free(m->cg);
    m->cg = nullptr;
    m->L64 = hbdia::HostLayout<double>();
    m->L32 = hbdia::HostLayout<float>();
    m->hasHBDIA = false;
    m->hostLayout = false;
    m->part.hasMetadata = false;
}

void prepare(hbdia_matrix *m, int32_t storage) {
    need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
    need(m->hostLayout, HBDIA_ERR_NOT_CONVERTED, "no host layout to upload");
    hbdia::ColumnWindow w, *W = nullptr;
    if (m->part.partial) {  // the plan reads x through the rank's window
        w.lo = m->part.windowLo;
        w.len = m->part.windowLen;
        w.rowBase = m->dtype == HBDIA_F32 ? m->c32.rowBase : m->c64.rowBase;
        W = &w;
    }
    free_block_sizes(m);
    if (m->dtype == HBDIA_F32) hbdia::build_plan(m->L32, storage, m->plan, W);
    else hbdia::build_plan(m->L64, storage, m->plan, W);
}

void ensure_device(hbdia_matrix *m) {
    if (!m->plan.base) prepare(m, HBDIA_STORE_NATIVE);
}

}  // namespace

int hbdia::record_error(int status, const std::string &msg) {
    g_err = msg;
    return status;
}

extern "C" {

const char *hbdia_last_error(void) { return g_err.c_str(); }
const char *hbdia_version(void) { return "hbdia_b200 0.1 (sm_100a)"; }

int hbdia_set_device(int32_t device) {
    return guarded([&] { hbdia::check_cuda(cudaSetDevice(device), "cudaSetDevice"); });
}

int hbdia_get_device(int32_t *device) {
    return guarded([&] {
        need(device != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        int d = 0;
        hbdia::check_cuda(cudaGetDevice(&d), "cudaGetDevice");
        *device = d;
    });
}

const char *hbdia_status_string(int s) {
    switch (s) {
        case HBDIA_OK: return "HBDIA_OK";
        case HBDIA_ERR_INVALID_ARGUMENT: return "HBDIA_ERR_INVALID_ARGUMENT";
        case HBDIA_ERR_OUT_OF_RANGE: return "HBDIA_ERR_OUT_OF_RANGE";
        case HBDIA_ERR_RUNTIME: return "HBDIA_ERR_RUNTIME";
        case HBDIA_ERR_CUDA: return "HBDIA_ERR_CUDA";
        case HBDIA_ERR_NO_MEMORY: return "HBDIA_ERR_NO_MEMORY";
        case HBDIA_ERR_NOT_CONVERTED: return "HBDIA_ERR_NOT_CONVERTED";
        case HBDIA_ERR_UNSUPPORTED: return "HBDIA_ERR_UNSUPPORTED";
        case HBDIA_ERR_DEVICE_TIMEOUT: return "HBDIA_ERR_DEVICE_TIMEOUT";
        default: return "HBDIA_ERR_UNKNOWN";
    }
}

int hbdia_matrix_create_empty(hbdia_dtype dtype, hbdia_matrix **out) {
    return guarded([&] {
        need(out != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null output handle");
        need(dtype == HBDIA_F64 || dtype == HBDIA_F32, HBDIA_ERR_INVALID_ARGUMENT, "unknown dtype");
        auto *m = new hbdia_matrix();
        m->dtype = dtype;
        *out = m;
    });
}

int hbdia_matrix_create(hbdia_dtype dtype, const int32_t *rows, const int32_t *cols, const void *values,
                        int64_t nnz, int32_t numRows, int32_t numCols, hbdia_matrix **out) {
    return guarded([&] {
        need(out != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null output handle");
        need(dtype == HBDIA_F64 || dtype == HBDIA_F32, HBDIA_ERR_INVALID_ARGUMENT, "unknown dtype");
        std::unique_ptr<hbdia_matrix> m(new hbdia_matrix());
        m->dtype = dtype;
        if (dtype == HBDIA_F32) fill_coo(m->c32, rows, cols, values, nnz, numRows, numCols);
        else fill_coo(m->c64, rows, cols, values, nnz, numRows, numCols);
        m->hasCOO = true;
        *out = m.release();
    });
}

void hbdia_matrix_destroy(hbdia_matrix *m) {
    if (!m) return;
    reset_hbdia(m);
    delete m;
}

int hbdia_matrix_stencil27(hbdia_matrix *m, int32_t nx, int32_t ny, int32_t nz, double noise,
                           int32_t iteration) {
    return guarded([&] {
        need(m && nx > 0 && ny > 0 && nz > 0, HBDIA_ERR_INVALID_ARGUMENT, "bad stencil arguments");
        need(static_cast<int64_t>(nx) * ny * nz * 27 < 2147483647LL, HBDIA_ERR_UNSUPPORTED,
             "grid too large for the reference's int arithmetic");
        reset_hbdia(m);
        if (m->dtype == HBDIA_F32) hbdia::reference_stencil27(nx, ny, nz, noise, iteration, m->c32);
        else hbdia::reference_stencil27(nx, ny, nz, noise, iteration, m->c64);
        m->hasCOO = true;
    });
}

int hbdia_matrix_load_mtx(hbdia_matrix *m, const char *path, int32_t numRows, int32_t numCols,
                          int32_t *ok) {
    return guarded([&] {
        need(m && path && ok, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        bool r;
        if (m->dtype == HBDIA_F32) {
            hbdia::Coo<float> c;
            r = hbdia::load_mtx(path, numRows, numCols, c);
            if (r || !c.vals.empty()) { reset_hbdia(m); m->c32 = std::move(c); m->hasCOO = true; }
        } else {
            hbdia::Coo<double> c;
            r = hbdia::load_mtx(path, numRows, numCols, c);
            if (r || !c.vals.empty()) { reset_hbdia(m); m->c64 = std::move(c); m->hasCOO = true; }
        }
        *ok = r ? 1 : 0;
    });
}

int hbdia_matrix_convert(hbdia_matrix *m, int32_t blockWidth, int32_t threshold, int64_t maxCoo,
                         int32_t cooIsUnique, int32_t execMode, int32_t upload) {
    (void)cooIsUnique;  // the reference ignores it too (src/Format/HBDIA.cpp:531-534)
    (void)execMode;     // the COO remainder always runs fused on the GPU
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        // early returns of src/Format/HBDIA.cpp:511-524
        if (m->hasHBDIA || !m->hasCOO || coo_nnz(m) == 0) return;
        need(blockWidth > 0, HBDIA_ERR_INVALID_ARGUMENT, "blockWidth must be positive");
        if (m->dtype == HBDIA_F32) hbdia::convert_to_hbdia(m->c32, blockWidth, threshold, maxCoo, m->L32);
        else hbdia::convert_to_hbdia(m->c64, blockWidth, threshold, maxCoo, m->L64);
        if (m->part.partial) {  // BasicDistributor::receiveMatrix's analyzeDataRanges + metadata
            if (m->dtype == HBDIA_F32) hbdia::partial_metadata(m->c32, m->L32, m->part);
            else hbdia::partial_metadata(m->c64, m->L64, m->part);
        }
        m->hasHBDIA = true;
        m->hostLayout = true;
        m->blockWidth = blockWidth;
        m->threshold = threshold;
        m->maxCoo = maxCoo;
        if (upload) prepare(m, HBDIA_STORE_NATIVE);
    });
}

int hbdia_matrix_prepare_gpu(hbdia_matrix *m, int32_t storage) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        prepare(m, storage);
    });
}

int hbdia_matrix_remove_duplicates(hbdia_matrix *m) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        if (!m->hasCOO) return;  // "No COO format available" (src/Format/HBDIA.cpp:374-377)
        if (m->dtype == HBDIA_F32) hbdia::remove_coo_duplicates(m->c32);
        else hbdia::remove_coo_duplicates(m->c64);
    });
}

int hbdia_matrix_convert_dia(hbdia_matrix *m, int32_t cooIsUnique) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        // early returns of src/Format/HBDIA.cpp:416-429
        if (m->hasDIA || !m->hasCOO) return;
        if (coo_nnz(m) == 0) {
            m->hasDIA = true;
            return;
        }
        if (m->dtype == HBDIA_F32) hbdia::convert_to_dia(m->c32, cooIsUnique != 0, m->diaOffsets, m->dia32, m->diaLength);
        else hbdia::convert_to_dia(m->c64, cooIsUnique != 0, m->diaOffsets, m->dia64, m->diaLength);
        m->hasDIA = true;
    });
}

int hbdia_matrix_dia_info(const hbdia_matrix *m, int32_t *hasDIA, int32_t *numDiagonals, int32_t *diagLength) {
    return guarded([&] {
        need(m && hasDIA && numDiagonals && diagLength, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *hasDIA = m->hasDIA;
        *numDiagonals = static_cast<int32_t>(m->diaOffsets.size());
        *diagLength = m->diaLength;
    });
}

int hbdia_matrix_export_dia(const hbdia_matrix *m, int32_t *offsets, void *diagonals) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->hasDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in DIA format");
        if (offsets && !m->diaOffsets.empty())
            std::memcpy(offsets, m->diaOffsets.data(), m->diaOffsets.size() * sizeof(int32_t));
        if (diagonals) {
            if (m->dtype == HBDIA_F32 && !m->dia32.empty())
                std::memcpy(diagonals, m->dia32.data(), m->dia32.size() * sizeof(float));
            else if (m->dtype == HBDIA_F64 && !m->dia64.empty())
                std::memcpy(diagonals, m->dia64.data(), m->dia64.size() * sizeof(double));
        }
    });
}

int hbdia_matrix_storage_costs(const hbdia_matrix *m, hbdia_storage_costs *out) {
    return guarded([&] {
        need(m && out, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
        const int64_t vb = static_cast<int64_t>(esize(m->dtype));
        const auto &npr = m->dtype == HBDIA_F32 ? m->c32.nnzPerRow : m->c64.nnzPerRow;
        if (m->hostLayout) {
            auto go = [&](const auto &L) {
                hbdia::storage_costs(vb, L.numRows, L.numCols, coo_nnz(m), L.numberDiagonals, L.numBlocks,
                                     L.blockWidth, static_cast<int64_t>(L.data.size()),
                                     static_cast<int64_t>(L.cooRow.size()), L.histBlocks, npr, *out);
            };
            if (m->dtype == HBDIA_F32) go(m->L32);
            else go(m->L64);
        } else {
            const hbdia::DevicePlan &P = m->plan;
            hbdia::storage_costs(vb, P.n, P.numCols, coo_nnz(m), m->devMeta.numberDiagonals, P.numBlocks, P.bw,
                                 P.slots, P.nCoo, m->devMeta.histBlocks, npr, *out);
        }
    });
}

int hbdia_matrix_convert_on_device(hbdia_matrix *m, int32_t blockWidth, int32_t threshold, int64_t maxCoo,
                                   int32_t storage) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        // the same early returns as convertToHBDIAFormat (src/Format/HBDIA.cpp:511-524)
        if (m->hasHBDIA || !m->hasCOO || coo_nnz(m) == 0) return;
        need(blockWidth > 0, HBDIA_ERR_INVALID_ARGUMENT, "blockWidth must be positive");
        need(!m->part.partial, HBDIA_ERR_UNSUPPORTED, "partial matrices convert on the host (hbdia_matrix_convert)");
        if (m->dtype == HBDIA_F32)
            hbdia::convert_on_device(m->c32, blockWidth, threshold, maxCoo, storage, m->plan, m->devMeta);
        else hbdia::convert_on_device(m->c64, blockWidth, threshold, maxCoo, storage, m->plan, m->devMeta);
        m->hasHBDIA = true;
        m->hostLayout = false;
        m->blockWidth = blockWidth;
        m->threshold = threshold;
        m->maxCoo = maxCoo;
    });
}

int hbdia_matrix_get_info(const hbdia_matrix *m, hbdia_matrix_info *info) {
    return guarded([&] {
        need(m && info, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia_matrix_info I;
        std::memset(&I, 0, sizeof(I));
        I.dtype = m->dtype;
        I.numRows = num_rows(m);
        I.numCols = num_cols(m);
        I.hasCOO = m->hasCOO;
        I.numNonZeros = coo_nnz(m);
        I.hasHBDIA = m->hasHBDIA;
        I.onDevice = m->plan.base != nullptr;
        I.blockWidth = m->blockWidth;
        I.threshold = m->threshold;
        I.maxCooEntries = m->maxCoo;
        I.storage = plan_storage_code(m->plan);
        I.deviceBytes = static_cast<int64_t>(m->plan.bytes);
        I.bytesPerSpmv = m->plan.bytesPerSpmv;
        if (m->hostLayout) {
            auto fill = [&](const auto &L) {
                I.numBlocks = L.numBlocks;
                I.numberDiagonals = L.numberDiagonals;
                I.totalOffsets = static_cast<int64_t>(L.offsets.size());
                I.numSlots = static_cast<int64_t>(L.data.size());
                I.numCoo = static_cast<int64_t>(L.cooRow.size());
                I.histogramLength = static_cast<int32_t>(L.histBlocks.size());
            };
            if (m->dtype == HBDIA_F32) fill(m->L32);
            else fill(m->L64);
        } else if (m->plan.base) {
            I.numBlocks = m->plan.numBlocks;
            I.totalOffsets = m->plan.totalOffsets;
            I.numSlots = m->plan.slots;
            I.numCoo = m->plan.nCoo;
            I.numberDiagonals = m->devMeta.numberDiagonals;
            I.histogramLength = static_cast<int32_t>(m->devMeta.histBlocks.size());
        }
        *info = I;
    });
}

int hbdia_matrix_export_layout(const hbdia_matrix *m, int32_t *offsets, int32_t *blockStart, void *data,
                               int32_t *cooRow, int32_t *cooCol, void *cooVal, int32_t *cooRowPtr,
                               int32_t *histBlocks, int32_t *histNnz) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "no HBDIA layout");
        auto cp = [](void *dst, const auto &v) {
            if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
        };
        if (!m->hostLayout) {
            // a layout the GPU converter built: read it back from the device
            const hbdia::DevicePlan &P = m->plan;
            need(P.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "no HBDIA layout");
            need(P.storage == HBDIA_STORE_NATIVE, HBDIA_ERR_UNSUPPORTED,
                 "a reduced-storage device layout has no exact values to export");
            const size_t es = esize(m->dtype);
            auto down = [](void *dst, const void *src, size_t bytes) {
                if (dst && bytes) hbdia::check_cuda(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy(export)");
            };
            down(offsets, P.offs, sizeof(int32_t) * P.totalOffsets);
            down(blockStart, P.blkOff, sizeof(int32_t) * (static_cast<size_t>(P.numBlocks) + 1));
            down(data, P.vals, es * P.slots);
            down(cooRow, P.cooRow, sizeof(int32_t) * P.nCoo);
            down(cooCol, P.cooCol, sizeof(int32_t) * P.nCoo);
            down(cooVal, P.cooVal, es * P.nCoo);
            down(cooRowPtr, P.cooRowPtr, sizeof(int32_t) * (static_cast<size_t>(P.n) + 1));
            cp(histBlocks, m->devMeta.histBlocks);
            cp(histNnz, m->devMeta.histNnz);
            return;
        }
        auto go = [&](const auto &L) {
            cp(offsets, L.offsets);
            cp(blockStart, L.blockStart);
            cp(data, L.data);
            cp(cooRow, L.cooRow);
            cp(cooCol, L.cooCol);
            cp(cooVal, L.cooVal);
            cp(cooRowPtr, L.cooRowPtr);
            cp(histBlocks, L.histBlocks);
            cp(histNnz, L.histNnz);
        };
        if (m->dtype == HBDIA_F32) go(m->L32);
        else go(m->L64);
    });
}

int hbdia_matrix_export_coo(const hbdia_matrix *m, int32_t *rows, int32_t *cols, void *values) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        auto go = [&](const auto &c) {
            if (rows && !c.rows.empty()) std::memcpy(rows, c.rows.data(), c.rows.size() * 4);
            if (cols && !c.cols.empty()) std::memcpy(cols, c.cols.data(), c.cols.size() * 4);
            if (values && !c.vals.empty()) std::memcpy(values, c.vals.data(), c.vals.size() * sizeof(c.vals[0]));
        };
        if (m->dtype == HBDIA_F32) go(m->c32);
        else go(m->c64);
    });
}

int hbdia_matrix_export_nnz_per_row(const hbdia_matrix *m, int32_t *nnzPerRow) {
    return guarded([&] {
        need(m && nnzPerRow, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        const auto &v = m->dtype == HBDIA_F32 ? m->c32.nnzPerRow : m->c64.nnzPerRow;
        if (!v.empty()) std::memcpy(nnzPerRow, v.data(), v.size() * 4);
    });
}

int hbdia_allocation_count(int64_t *device, int64_t *pinnedHost) {
    return guarded([&] {
        need(device && pinnedHost, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::allocation_counts(device, pinnedHost);
    });
}

int hbdia_matrix_device_arrays(hbdia_matrix *m, hbdia_device_arrays *a) {
    return guarded([&] {
        need(m && a, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        const hbdia::DevicePlan &P = m->plan;
        need(P.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        if (!m->blockSizesDev && P.numBlocks > 0) {
            // blockSizes[b] = blockStart[b + 1] - blockStart[b] (src/Format/HBDIA.cpp:741)
            std::vector<int32_t> start(static_cast<size_t>(P.numBlocks) + 1), sizes(P.numBlocks);
            hbdia::check_cuda(cudaMemcpy(start.data(), P.blkOff, start.size() * sizeof(int32_t),
                                         cudaMemcpyDeviceToHost), "cudaMemcpy(block starts)");
            for (int32_t b = 0; b < P.numBlocks; ++b) sizes[b] = start[b + 1] - start[b];
            int32_t *d = nullptr;
            hbdia::check_cuda(hbdia::dev_alloc(&d, sizes.size() * sizeof(int32_t)), "cudaMalloc(block sizes)");
            const cudaError_t e = cudaMemcpy(d, sizes.data(), sizes.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(d);
                hbdia::check_cuda(e, "cudaMemcpy(block sizes)");
            }
            m->blockSizesDev = d;
        }
        std::memset(a, 0, sizeof(*a));
        a->hbdiaData = P.storage == HBDIA_STORE_NATIVE ? P.vals : nullptr;
        if (m->part.partial) a->flattenedVectorOffsets = P.offs;
        else a->flattenedOffsets = P.offs;
        a->blockStartIndices = P.blkOff;
        a->blockSizes = m->blockSizesDev;
        if (P.nCoo > 0) {
            a->cpuRowIndices = P.cooRow;
            a->cpuColIndices = P.cooCol;
            a->cpuValues = P.cooVal;
            a->cpuRowPtr = P.cooRowPtr;
        }
    });
}

int hbdia_matrix_stream(const hbdia_matrix *m, void **stream) {
    return guarded([&] {
        need(m && stream, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        *stream = m->plan.stream;
    });
}

}  // extern "C"

namespace {
int32_t read_status(const hbdia_matrix *m, bool clear) {
    int32_t bits = 0;
    if (!m->plan.status) return 0;
    hbdia::check_cuda(cudaStreamSynchronize(static_cast<cudaStream_t>(m->plan.stream)), "cudaStreamSynchronize");
    hbdia::check_cuda(cudaMemcpy(&bits, m->plan.status, sizeof(bits), cudaMemcpyDeviceToHost), "cudaMemcpy(status)");
    if (clear && bits) hbdia::check_cuda(cudaMemset(m->plan.status, 0, sizeof(bits)), "cudaMemset(status)");
    return bits;
}
void throw_if_timeout(int32_t bits) {
    if (bits)
        throw Error(HBDIA_ERR_DEVICE_TIMEOUT, "a bounded wait in the SpMV kernel ran out (status bits " +
                                                  std::to_string(bits) + "); the result is invalid");
}
}  // namespace

extern "C" {

int hbdia_matrix_synchronize(const hbdia_matrix *m) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        if (m->plan.stream) {
            hbdia::check_cuda(cudaStreamSynchronize(static_cast<cudaStream_t>(m->plan.stream)),
                              "cudaStreamSynchronize");
            throw_if_timeout(read_status(m, true));
        }
    });
}

int hbdia_matrix_device_status(const hbdia_matrix *m, int32_t *bits) {
    return guarded([&] {
        need(m && bits, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *bits = read_status(m, false);
    });
}

int hbdia_matrix_set_kernel(hbdia_matrix *m, int32_t kernel) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(kernel >= HBDIA_KERNEL_AUTO && kernel <= HBDIA_KERNEL_QUAD, HBDIA_ERR_INVALID_ARGUMENT,
             "unknown kernel");
        m->plan.kernel = kernel;
    });
}

int hbdia_matrix_selected_kernel(const hbdia_matrix *m, const void *x, int32_t *kernel) {
    return guarded([&] {
        need(m && kernel, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        *kernel = hbdia::select_kernel(m->plan, x);
    });
}

int hbdia_matrix_set_tuning(hbdia_matrix *m, int32_t key, int32_t value) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        if (key == HBDIA_TUNE_UNROLL) {
            need(value == 0 || value == 9 || value == 27, HBDIA_ERR_INVALID_ARGUMENT, "unroll must be 0, 9 or 27");
            m->plan.unroll = value;
            return;
        }
        if (key == HBDIA_TUNE_PREFETCH) {
            need(value >= -1 && value <= 1, HBDIA_ERR_INVALID_ARGUMENT, "prefetch must be -1, 0 or 1");
            m->plan.prefetchL2 = value;
            return;
        }
        if (key == HBDIA_TUNE_TAIL) {
            need(value >= -1 && value <= 1, HBDIA_ERR_INVALID_ARGUMENT, "tail must be -1, 0 or 1");
            m->plan.maskedTail = value;
            return;
        }
        if (key == HBDIA_TUNE_QUAD_GROUP) {
            need(value == 0 || value == 1 || value == 2 || value == 4 || value == 8, HBDIA_ERR_INVALID_ARGUMENT,
                 "quad group must be 0, 1, 2, 4 or 8");
            m->plan.quadGroup = value;
            return;
        }
        if (key == HBDIA_TUNE_STAGES) {
            need(value >= 0 && value <= 5, HBDIA_ERR_INVALID_ARGUMENT, "stage configuration must be 0-5");
            m->plan.xsConfig = value;
            return;
        }
        if (key == HBDIA_TUNE_SPMM_TILE) {
            need(value == 0 || value == 2 || value == 4 || value == 8 || value == 16 || value == 32,
                 HBDIA_ERR_INVALID_ARGUMENT, "SpMM tile must be 0, 2, 4, 8, 16 or 32");
            m->plan.spmmTileForced = value;
            return;
        }
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "unknown tuning key");
    });
}

int hbdia_matrix_autotune(hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                          void *stream, int32_t force, hbdia_tune_result *out) {
    return guarded([&] {
        need(m && X && Y, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia_tune_result r;
        std::memset(&r, 0, sizeof(r));
        hbdia::autotune(m->plan, X, ldx, Y, ldy, k, stream, force != 0, &r.kernel, &r.unroll, &r.spmmTile,
                        &r.fromCache, &r.msPerCall);
        if (out) *out = r;
    });
}

int hbdia_autotune_clear(void) {
    return guarded([&] { hbdia::autotune_clear_cache(); });
}

int hbdia_matrix_set_wait_timeout(hbdia_matrix *m, uint64_t ns) {
    return guarded([&] {
        need(m != nullptr && ns > 0, HBDIA_ERR_INVALID_ARGUMENT, "bad timeout");
        m->plan.waitTimeoutNs = ns;
    });
}

int hbdia_matrix_test_skip_tile(hbdia_matrix *m, int32_t tile) {
    return guarded([&] {
        need(m != nullptr && tile >= -1, HBDIA_ERR_INVALID_ARGUMENT, "bad tile");
        m->plan.skipTile = tile;
    });
}

// ---------------------------------------------------------------- vectors
int hbdia_vector_create(hbdia_dtype dtype, const void *host, int64_t n, hbdia_vector **out) {
    return guarded([&] {
        need(out != nullptr && n >= 0, HBDIA_ERR_INVALID_ARGUMENT, "bad vector arguments");
        need(dtype == HBDIA_F64 || dtype == HBDIA_F32, HBDIA_ERR_INVALID_ARGUMENT, "unknown dtype");
        std::unique_ptr<hbdia_vector> v(new hbdia_vector());
        v->dtype = dtype;
        v->n = n;
        const size_t bytes = static_cast<size_t>(n) * esize(dtype);
        hbdia::check_cuda(hbdia::dev_alloc(&v->d, bytes ? bytes : 256), "cudaMalloc(vector)");
        int err = host && bytes ? cudaMemcpy(v->d, host, bytes, cudaMemcpyHostToDevice)
                                : cudaMemset(v->d, 0, bytes ? bytes : 256);
        if (err != cudaSuccess) {
            cudaFree(v->d);
            hbdia::check_cuda(err, "vector initialisation");
        }
        *out = v.release();
    });
}

void hbdia_vector_destroy(hbdia_vector *v) {
    if (!v) return;
    if (v->d) cudaFree(v->d);
    if (v->cooResult) cudaFree(v->cooResult);
    delete v;
}

int hbdia_vector_device_ptr(const hbdia_vector *v, void **p) {
    return guarded([&] {
        need(v && p, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *p = v->d;
    });
}

int hbdia_vector_coo_results_ptr(hbdia_vector *v, void **p) {
    return guarded([&] {
        need(v && p, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        if (!v->cooResult) {
            const size_t bytes = static_cast<size_t>(v->n) * esize(v->dtype);
            void *d = nullptr;
            hbdia::check_cuda(hbdia::dev_alloc(&d, bytes ? bytes : 256), "cudaMalloc(COO result buffer)");
            const cudaError_t e = cudaMemset(d, 0, bytes ? bytes : 256);
            if (e != cudaSuccess) {
                cudaFree(d);
                hbdia::check_cuda(e, "cudaMemset(COO result buffer)");
            }
            v->cooResult = d;
        }
        *p = v->cooResult;
    });
}

int hbdia_vector_size(const hbdia_vector *v, int64_t *n) {
    return guarded([&] {
        need(v && n, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *n = v->n;
    });
}

int hbdia_vector_upload(hbdia_vector *v, const void *host) {
    return guarded([&] {
        need(v && host, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::check_cuda(cudaMemcpy(v->d, host, v->n * esize(v->dtype), cudaMemcpyHostToDevice),
                          "cudaMemcpy(vector upload)");
    });
}

int hbdia_vector_download(const hbdia_vector *v, void *host) {
    return guarded([&] {
        need(v && host, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        hbdia::check_cuda(cudaMemcpy(host, v->d, v->n * esize(v->dtype), cudaMemcpyDeviceToHost),
                          "cudaMemcpy(vector download)");
    });
}

// ---------------------------------------------------------------- SpMV
int hbdia_spmv(hbdia_matrix *m, const hbdia_vector *x, hbdia_vector *y, int32_t execCOOCPU,
               int32_t execCOOGPU) {
    return guarded([&] {
        need(m && x && y, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(x->dtype == m->dtype && y->dtype == m->dtype, HBDIA_ERR_INVALID_ARGUMENT,
             "vector and matrix value types differ");
        const int32_t nR = num_rows(m), nC = num_cols(m);
        need(x->n >= std::max(nR, nC), HBDIA_ERR_INVALID_ARGUMENT, "input vector shorter than the matrix");
        need(y->n >= nR, HBDIA_ERR_INVALID_ARGUMENT, "output vector shorter than the matrix");
        if (!m->hasHBDIA) {
            need(coo_nnz(m) == 0, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
            // an empty matrix: y = 0
            hbdia::check_cuda(cudaMemset(y->d, 0, static_cast<size_t>(nR) * esize(m->dtype)), "cudaMemset");
            return;
        }
        const int64_t nCoo = m->hostLayout ? (m->dtype == HBDIA_F32 ? (int64_t)m->L32.cooRow.size()
                                                                    : (int64_t)m->L64.cooRow.size())
                                           : m->plan.nCoo;
        if (nCoo > 0 && !execCOOCPU && !execCOOGPU)
            throw Error(HBDIA_ERR_RUNTIME, "Invalid COO execution flags");
        ensure_device(m);
        hbdia::launch_spmv(m->plan, x->d, y->d, nullptr);
    });
}

int hbdia_spmv_device(const hbdia_matrix *m, const void *x, void *y, void *stream) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        hbdia::launch_spmv(m->plan, x, y, stream);
    });
}

int hbdia_spmm_device(const hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                      void *stream) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        hbdia::launch_spmm(m->plan, X, ldx, Y, ldy, k, stream);
    });
}

int hbdia_spmm_device_colmajor(const hbdia_matrix *m, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k,
                               void *stream) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        hbdia::launch_spmm(m->plan, X, ldx, Y, ldy, k, stream, true);
    });
}

int hbdia_spmv_list_device(const hbdia_matrix *m, const void *const *x, void *const *y, int32_t k, void *stream) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        need(m->plan.base != nullptr, HBDIA_ERR_NOT_CONVERTED, "matrix has no device layout");
        hbdia::launch_spmv_list(m->plan, x, y, k, stream);
    });
}

int hbdia_spmv_host(hbdia_matrix *m, const void *xh, void *yh) {
    return guarded([&] {
        need(m && xh && yh, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
        ensure_device(m);
        std::lock_guard<std::mutex> lk(m->hostMu);
        hbdia::DevicePlan &P = m->plan;
        const size_t es = esize(m->dtype);
        const size_t xb = static_cast<size_t>(std::max(P.n, P.numCols)) * es;
        const size_t yb = static_cast<size_t>(P.n) * es;
        if (!P.xScratch) hbdia::check_cuda(hbdia::dev_alloc(&P.xScratch, xb), "cudaMalloc(x scratch)");
        if (!P.yScratch) hbdia::check_cuda(hbdia::dev_alloc(&P.yScratch, yb), "cudaMalloc(y scratch)");
        cudaStream_t s = static_cast<cudaStream_t>(P.stream);
        hbdia::check_cuda(cudaMemcpyAsync(P.xScratch, xh, xb, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(x)");
        hbdia::launch_spmv(P, P.xScratch, P.yScratch, s);
        hbdia::check_cuda(cudaMemcpyAsync(yh, P.yScratch, yb, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync(y)");
        hbdia::check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        throw_if_timeout(read_status(m, true));
    });
}

int hbdia_spmv_host_many(hbdia_matrix *m, const void *const *xh, void *const *yh, int32_t count) {
    return guarded([&] {
        need(m != nullptr && count >= 0, HBDIA_ERR_INVALID_ARGUMENT, "bad argument");
        need(count == 0 || (xh && yh), HBDIA_ERR_INVALID_ARGUMENT, "null vector list");
        for (int32_t j = 0; j < count; ++j) need(xh[j] && yh[j], HBDIA_ERR_INVALID_ARGUMENT, "null vector");
        need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
        if (count == 0) return;
        ensure_device(m);
        std::lock_guard<std::mutex> lk(m->hostMu);
        hbdia::DevicePlan &P = m->plan;
        const size_t es = esize(m->dtype);
        const size_t xb = static_cast<size_t>(std::max(P.n, P.numCols)) * es;
        const size_t yb = static_cast<size_t>(P.n) * es;
        constexpr int D = hbdia_matrix::kHostDepth;
        const int depth = std::min<int32_t>(D, count);
        for (int d = 0; d < depth; ++d) {
            if (!m->pipeStream[d]) {
                cudaStream_t s = nullptr;
                hbdia::check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate(pipeline)");
                m->pipeStream[d] = s;
            }
            if (!m->pipeX[d]) hbdia::check_cuda(hbdia::dev_alloc(&m->pipeX[d], xb), "cudaMalloc(pipeline x)");
            if (!m->pipeY[d]) hbdia::check_cuda(hbdia::dev_alloc(&m->pipeY[d], yb), "cudaMalloc(pipeline y)");
        }
        // step j on stage j % depth: its copy in, SpMV and copy out are ordered
        // on that stage's stream (so the stage's buffers are free again when
        // step j + depth starts), while different stages overlap -- one
        // step's upload runs beside another's download and kernel
        std::string err;
        int status = HBDIA_OK;
        try {
            for (int32_t j = 0; j < count; ++j) {
                const int d = j % depth;
                cudaStream_t s = static_cast<cudaStream_t>(m->pipeStream[d]);
                hbdia::check_cuda(cudaMemcpyAsync(m->pipeX[d], xh[j], xb, cudaMemcpyHostToDevice, s),
                                  "cudaMemcpyAsync(x)");
                hbdia::launch_spmv(P, m->pipeX[d], m->pipeY[d], s);
                hbdia::check_cuda(cudaMemcpyAsync(yh[j], m->pipeY[d], yb, cudaMemcpyDeviceToHost, s),
                                  "cudaMemcpyAsync(y)");
            }
        } catch (const hbdia::Error &e) {
            status = e.status;
            err = e.what();
        }
        for (int d = 0; d < depth; ++d) {  // always drain what was issued
            const cudaError_t rc = cudaStreamSynchronize(static_cast<cudaStream_t>(m->pipeStream[d]));
            if (rc != cudaSuccess && status == HBDIA_OK) {
                status = HBDIA_ERR_CUDA;
                err = cudaGetErrorString(rc);
            }
        }
        if (status != HBDIA_OK) throw hbdia::Error(status, err);
        throw_if_timeout(read_status(m, true));
    });
}

// ---------------------------------------------------------------- solver
int hbdia_cg_solve(hbdia_matrix *m, const double *b, double *x, const hbdia_cg_options *opt, void *stream,
                   hbdia_cg_result *out) {
    return guarded([&] {
        need(m && b && x && opt, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(m->dtype == HBDIA_F64, HBDIA_ERR_UNSUPPORTED, "the CG solver needs a double matrix");
        need(m->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
        need(num_rows(m) == num_cols(m), HBDIA_ERR_INVALID_ARGUMENT, "CG needs a square matrix");
        need(!m->part.partial, HBDIA_ERR_UNSUPPORTED, "CG runs on whole matrices, not on one rank's rows");
        need(opt->tol > 0 && opt->updateFactor > 0 && opt->updateFactor < 1 && opt->maxUpdates >= 0 &&
                 opt->maxIterations > 0 && opt->checkEvery > 0,
             HBDIA_ERR_INVALID_ARGUMENT, "bad CG options");
        ensure_device(m);
        const hbdia::DevicePlan *it = &m->plan;
        if (opt->iterStorage != HBDIA_STORE_NATIVE) {
            const int32_t st = m->hostLayout ? hbdia::iteration_storage(m->L64, opt->iterStorage) : opt->iterStorage;
            if (!m->innerPlan.base || plan_storage_code(m->innerPlan) != st) {
                need(m->hostLayout, HBDIA_ERR_NOT_CONVERTED, "no host layout to build the iteration operator");
                hbdia::build_plan(m->L64, st, m->innerPlan);
                m->innerPlan.kernel = m->plan.kernel;
                m->innerPlan.unroll = m->plan.unroll;
            }
            it = &m->innerPlan;
        }
        m->cg = hbdia::cg_work(m->cg, num_rows(m));
        hbdia::CgParams prm;
        prm.tol = opt->tol;
        prm.updateFactor = opt->updateFactor;
        prm.maxUpdates = opt->maxUpdates;
        prm.maxIterations = opt->maxIterations;
        prm.checkEvery = opt->checkEvery;
        hbdia::CgStats st;
        hbdia::cg_solve(m->plan, *it, m->cg, b, x, prm, stream, &st);
        hbdia_cg_result r;
        std::memset(&r, 0, sizeof(r));
        r.updates = st.updates;
        r.iterations = st.iterations;
        r.relResidual = st.relResidual;
        r.seconds = st.seconds;
        r.converged = r.relResidual <= opt->tol;
        throw_if_timeout(read_status(m, true));
        if (out) *out = r;
    });
}

// ---------------------------------------------------------------- serving
void hbdia_server_default_options(hbdia_server_options *o) {
    if (o) hbdia::server_default_options(o);
}

int hbdia_server_create(const hbdia_server_options *o, hbdia_server **out) {
    return guarded([&] {
        need(out != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        hbdia_server_options d;
        hbdia::server_default_options(&d);
        auto s = std::make_unique<hbdia_server>();
        s->S = hbdia::server_create(o ? *o : d);
        *out = s.release();
    });
}

void hbdia_server_destroy(hbdia_server *s) {
    if (!s) return;
    hbdia::server_destroy(s->S);
    delete s;
}

int hbdia_server_add_matrix(hbdia_server *s, const hbdia_matrix *m, int32_t *id) {
    return guarded([&] {
        need(s && m && id, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(!m->part.partial, HBDIA_ERR_UNSUPPORTED, "the server serves whole matrices");
        *id = hbdia::server_add_matrix(s->S, m);
    });
}

int hbdia_server_submit(hbdia_server *s, int32_t matrix, int32_t kind, const double *x, double *y,
                        uint64_t *ticket) {
    return guarded([&] {
        need(s && ticket, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *ticket = hbdia::server_submit(s->S, matrix, kind, x, y, false);
    });
}

int hbdia_server_submit_device(hbdia_server *s, int32_t matrix, int32_t kind, const double *xDevice, double *yDevice,
                               uint64_t *ticket) {
    return guarded([&] {
        need(s && ticket, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *ticket = hbdia::server_submit(s->S, matrix, kind, xDevice, yDevice, true);
    });
}

int hbdia_server_pause(hbdia_server *s, int32_t paused) {
    return guarded([&] {
        need(s != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null server");
        hbdia::server_pause(s->S, paused != 0);
    });
}

int hbdia_server_wait(hbdia_server *s, uint64_t ticket, hbdia_request_info *info) {
    return guarded([&] {
        need(s != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null server");
        hbdia::server_wait(s->S, ticket, info);
    });
}

int hbdia_server_get_stats(hbdia_server *s, hbdia_server_stats *out) {
    return guarded([&] {
        need(s && out, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::server_stats(s->S, out);
    });
}

// ---------------------------------------------------------------- batches
int hbdia_batch_create(hbdia_matrix *const *mats, int32_t count, hbdia_batch **out) {
    return guarded([&] {
        need(mats && out && count > 0, HBDIA_ERR_INVALID_ARGUMENT, "null argument or empty batch");
        *out = nullptr;
        std::vector<const hbdia::DevicePlan *> plans(static_cast<size_t>(count));
        for (int32_t i = 0; i < count; ++i) {
            need(mats[i] != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix in batch");
            need(mats[i]->hasHBDIA, HBDIA_ERR_NOT_CONVERTED, "matrix is not in HBDIA format");
            plans[i] = &mats[i]->plan;
        }
        auto b = std::make_unique<hbdia_batch>();
        b->B = hbdia::batch_create(plans);
        *out = b.release();
    });
}

void hbdia_batch_destroy(hbdia_batch *b) {
    if (!b) return;
    hbdia::batch_free(b->B);
    delete b;
}

int hbdia_batch_bind(hbdia_batch *b, const void *const *X, const int64_t *ldx, void *const *Y, const int64_t *ldy,
                     const int32_t *k) {
    return guarded([&] {
        need(b != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null batch");
        hbdia::batch_bind(b->B, X, ldx, Y, ldy, k);
    });
}

int hbdia_batch_run(hbdia_batch *b, void *stream) {
    return guarded([&] {
        need(b != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null batch");
        hbdia::batch_run(b->B, stream);
    });
}

int hbdia_batch_set_config(hbdia_batch *b, const hbdia_batch_config *c) {
    return guarded([&] {
        need(b && c, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::batch_set_config(b->B, *c);
    });
}

int hbdia_batch_get_config(const hbdia_batch *b, hbdia_batch_config *c) {
    return guarded([&] {
        need(b && c, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::batch_get_config(b->B, *c);
    });
}

int hbdia_batch_autotune(hbdia_batch *b, void *stream, float *ms, int32_t *candidates) {
    return guarded([&] {
        need(b != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null batch");
        hbdia::batch_autotune(b->B, stream, ms, candidates);
    });
}

int hbdia_batch_info(const hbdia_batch *b, int32_t *count, int32_t *totalTiles, int64_t *bytesPerRun) {
    return guarded([&] {
        need(b && count && totalTiles && bytesPerRun, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        hbdia::batch_info(b->B, count, totalTiles, bytesPerRun);
    });
}

int hbdia_batch_stream(const hbdia_batch *b, void **stream) {
    return guarded([&] {
        need(b && stream, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        *stream = hbdia::batch_stream(b->B);
    });
}

// ---------------------------------------------------------------- workloads
int hbdia_generate_stencil27(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor,
                             double frac, double lo, double hi, uint64_t seed, int64_t *nnz,
                             int32_t *rows, int32_t *cols, double *values) {
    return guarded([&] {
        hbdia::generate_stencil(27, nx, ny, nz, center, neighbor, frac, lo, hi, seed, nnz, rows, cols, values);
    });
}

int hbdia_generate_stencil7(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor,
                            int64_t *nnz, int32_t *rows, int32_t *cols, double *values) {
    return guarded([&] {
        hbdia::generate_stencil(7, nx, ny, nz, center, neighbor, 0.0, 0.0, 0.0, 0, nnz, rows, cols, values);
    });
}

int hbdia_generate_banded(int32_t n, const int32_t *offsets, int32_t numOffsets, double lo, double hi,
                          double dropProb, double scatterFraction, uint64_t seed, int64_t *nnz,
                          int32_t *rows, int32_t *cols, double *values) {
    return guarded([&] {
        hbdia::generate_banded(n, offsets, numOffsets, lo, hi, dropProb, scatterFraction, seed, nnz, rows,
                               cols, values);
    });
}

int hbdia_generate_stencil27_spd(int32_t nx, int32_t ny, int32_t nz, double shift, double extraFraction,
                                 uint64_t seed, int64_t *nnz, int32_t *rows, int32_t *cols, double *values) {
    return guarded([&] {
        hbdia::generate_stencil27_spd(nx, ny, nz, shift, extraFraction, seed, nnz, rows, cols, values);
    });
}

int hbdia_fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed) {
    return guarded([&] {
        need(out != nullptr || n == 0, HBDIA_ERR_INVALID_ARGUMENT, "null output");
        hbdia::fill_uniform(out, n, lo, hi, seed);
    });
}

}  // extern "C"

// ------------------------------------------------------- row partitioning
int hbdia_matrix_create_partial(hbdia_dtype dtype, const int32_t *rows, const int32_t *cols, const void *values,
                                int64_t nnz, int32_t numLocalRows, int32_t numGlobalRows, int32_t numGlobalCols,
                                int64_t numGlobalNonZeros, int32_t globalRowStart, int32_t rank, int32_t size,
                                hbdia_matrix **out) {
    return guarded([&] {
        need(out != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null output handle");
        need(dtype == HBDIA_F64 || dtype == HBDIA_F32, HBDIA_ERR_INVALID_ARGUMENT, "unknown dtype");
        need(numLocalRows > 0 && numGlobalRows > 0 && numGlobalCols > 0, HBDIA_ERR_INVALID_ARGUMENT,
             "Matrix dimensions must be positive");
        need(numGlobalRows == numGlobalCols, HBDIA_ERR_UNSUPPORTED,
             "row partitioning needs a square matrix (x is partitioned like the rows)");
        need(globalRowStart >= 0 && static_cast<int64_t>(globalRowStart) + numLocalRows <= numGlobalRows,
             HBDIA_ERR_OUT_OF_RANGE, "the local rows lie outside the global matrix");
        need(size >= 1 && rank >= 0 && rank < size, HBDIA_ERR_INVALID_ARGUMENT, "bad rank / size");
        need(numGlobalRows / size >= 1, HBDIA_ERR_INVALID_ARGUMENT, "more processes than rows");
        std::unique_ptr<hbdia_matrix> m(new hbdia_matrix());
        m->dtype = dtype;
        // the partial constructor validates against numRows = numLocalRows and
        // numCols = numLocalCols = numGlobalCols (src/Format/HBDIA.cpp:140-153)
        if (dtype == HBDIA_F32) {
            fill_coo(m->c32, rows, cols, values, nnz, numLocalRows, numGlobalCols);
            m->c32.rowBase = globalRowStart;
        } else {
            fill_coo(m->c64, rows, cols, values, nnz, numLocalRows, numGlobalCols);
            m->c64.rowBase = globalRowStart;
        }
        m->hasCOO = true;
        m->part.partial = true;
        m->part.numGlobalRows = numGlobalRows;
        m->part.numGlobalCols = numGlobalCols;
        m->part.numGlobalNonZeros = numGlobalNonZeros;
        m->part.rank = rank;
        m->part.size = size;
        m->part.windowLo = globalRowStart;
        m->part.windowLen = numLocalRows;
        *out = m.release();
    });
}

int hbdia_matrix_partition(const hbdia_matrix *g, int32_t numProcesses, int32_t part, hbdia_matrix **out) {
    return guarded([&] {
        need(g && out, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        need(g->hasCOO, HBDIA_ERR_INVALID_ARGUMENT, "Matrix must be in COO format for partitioning");
        need(!g->part.partial, HBDIA_ERR_UNSUPPORTED, "the matrix is a partition already");
        std::unique_ptr<hbdia_matrix> m(new hbdia_matrix());
        m->dtype = g->dtype;
        int32_t nLocal, rb;
        if (g->dtype == HBDIA_F32) {
            hbdia::partition_rows(g->c32, numProcesses, part, m->c32);
            nLocal = m->c32.numRows;
            rb = m->c32.rowBase;
        } else {
            hbdia::partition_rows(g->c64, numProcesses, part, m->c64);
            nLocal = m->c64.numRows;
            rb = m->c64.rowBase;
        }
        m->hasCOO = true;
        m->part.partial = true;
        m->part.numGlobalRows = num_rows(g);
        m->part.numGlobalCols = num_cols(g);
        m->part.numGlobalNonZeros = coo_nnz(g);
        m->part.rank = part;
        m->part.size = numProcesses;
        m->part.windowLo = rb;
        m->part.windowLen = nLocal;
        *out = m.release();
    });
}

int hbdia_matrix_partial_info(const hbdia_matrix *m, hbdia_partial_info *info) {
    return guarded([&] {
        need(m && info, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        const hbdia::PartialMeta &p = m->part;
        hbdia_partial_info I;
        std::memset(&I, 0, sizeof(I));
        I.isPartial = p.partial;
        I.hasMetadata = p.hasMetadata;
        I.globalRowStart = m->dtype == HBDIA_F32 ? m->c32.rowBase : m->c64.rowBase;
        I.numGlobalRows = p.partial ? p.numGlobalRows : num_rows(m);
        I.numGlobalCols = p.partial ? p.numGlobalCols : num_cols(m);
        I.numGlobalNonZeros = p.partial ? p.numGlobalNonZeros : coo_nnz(m);
        I.rank = p.rank;
        I.size = p.size;
        I.numDataRanges = static_cast<int64_t>(p.dataRanges.size() / 2);
        I.numProcessRanges = static_cast<int64_t>(p.processRanges.size() / 3);
        I.totalBufferSize = p.totalBufferSize;
        I.leftBufferSize = p.leftBufferSize;
        I.rightBufferSize = p.rightBufferSize;
        I.windowStart = p.partial ? p.windowLo : 0;
        I.windowLength = p.partial ? p.windowLen : num_cols(m);
        *info = I;
    });
}

int hbdia_matrix_export_ranges(const hbdia_matrix *m, int32_t *dataRanges, int32_t *processRanges) {
    return guarded([&] {
        need(m != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null matrix");
        const hbdia::PartialMeta &p = m->part;
        if (dataRanges && !p.dataRanges.empty())
            std::memcpy(dataRanges, p.dataRanges.data(), p.dataRanges.size() * sizeof(int32_t));
        if (processRanges && !p.processRanges.empty())
            std::memcpy(processRanges, p.processRanges.data(), p.processRanges.size() * sizeof(int32_t));
    });
}

int hbdia_halo_create(int32_t elemBytes, const int64_t *srcOffset, const int64_t *dstOffset, const int64_t *length,
                      int32_t numSegments, int64_t srcLength, int64_t dstLength, hbdia_halo **out) {
    return guarded([&] {
        need(out != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null output handle");
        std::unique_ptr<hbdia_halo> h(new hbdia_halo());
        h->H = hbdia::halo_create(elemBytes, srcOffset, dstOffset, length, numSegments, srcLength, dstLength);
        *out = h.release();
    });
}

int hbdia_halo_copy(const hbdia_halo *h, const void *src, void *dst, void *stream) {
    return guarded([&] {
        need(h != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null halo");
        hbdia::halo_copy(h->H, src, dst, stream);
    });
}

int64_t hbdia_halo_elements(const hbdia_halo *h) { return h ? hbdia::halo_elements(h->H) : 0; }

void hbdia_halo_destroy(hbdia_halo *h) {
    if (!h) return;
    hbdia::halo_free(h->H);
    delete h;
}

// ---------------------------------------------------- borrowed device layouts
int hbdia_plan_create(const hbdia_layout_desc *desc, hbdia_plan **out) {
    return guarded([&] {
        need(desc && out, HBDIA_ERR_INVALID_ARGUMENT, "null argument");
        std::unique_ptr<hbdia_plan> p(new hbdia_plan());
        hbdia::borrow_plan(*desc, p->P);
        *out = p.release();
    });
}

int hbdia_plan_spmv(const hbdia_plan *p, const void *x, void *y, void *stream) {
    return guarded([&] {
        need(p != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null plan");
        hbdia::launch_spmv(p->P, x, y, stream);
    });
}

int hbdia_plan_spmm(const hbdia_plan *p, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t k, void *stream) {
    return guarded([&] {
        need(p != nullptr, HBDIA_ERR_INVALID_ARGUMENT, "null plan");
        hbdia::launch_spmm(p->P, X, ldx, Y, ldy, k, stream, false);
    });
}

void hbdia_plan_destroy(hbdia_plan *p) {
    if (!p) return;
    hbdia::free_plan(p->P);
    delete p;
}
