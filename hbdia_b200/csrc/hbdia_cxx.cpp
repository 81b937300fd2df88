// C++ drop-in API (include/hbdia/*.hpp) over the C ABI.  Status codes become
// the exceptions the reference throws for the same conditions.

#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "hbdia/Format/HBDIA.hpp"
#include "hbdia/Format/HBDIAVector.hpp"
#include "hbdia/Operations/HBDIASpMV.hpp"

namespace {

void raise(int status) {
    if (status == HBDIA_OK) return;
    const std::string msg = std::string(hbdia_status_string(status)) + ": " + hbdia_last_error();
    switch (status) {
        case HBDIA_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
        case HBDIA_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
        case HBDIA_ERR_NO_MEMORY: throw std::bad_alloc();
        default: throw std::runtime_error(msg);
    }
}

template <typename T>
constexpr hbdia_dtype dtype_of() {
    return std::is_same<T, float>::value ? HBDIA_F32 : HBDIA_F64;
}

template <typename T>
hbdia_matrix_info info_of(const hbdia_matrix *h) {
    hbdia_matrix_info i;
    raise(hbdia_matrix_get_info(h, &i));
    return i;
}

}  // namespace

// ---------------------------------------------------------------- HBDIA<T>
template <typename T>
HBDIA<T>::HBDIA() {
    raise(hbdia_matrix_create_empty(dtype_of<T>(), &h_));
}

template <typename T>
HBDIA<T>::HBDIA(const std::vector<int> &r, const std::vector<int> &c, const std::vector<T> &v) {
    if (r.size() != c.size() || r.size() != v.size())
        throw std::invalid_argument("Row indices, column indices, and values vectors must have the same size");
    raise(hbdia_matrix_create(dtype_of<T>(), r.data(), c.data(), v.data(), static_cast<int64_t>(v.size()), -1, -1,
                              &h_));
}

template <typename T>
HBDIA<T>::HBDIA(const std::vector<int> &r, const std::vector<int> &c, const std::vector<T> &v, int numRows,
                int numCols) {
    if (r.size() != c.size() || r.size() != v.size())
        throw std::invalid_argument("Row indices, column indices, and values vectors must have the same size");
    if (numRows <= 0 || numCols <= 0) throw std::invalid_argument("Matrix dimensions must be positive");
    raise(hbdia_matrix_create(dtype_of<T>(), r.data(), c.data(), v.data(), static_cast<int64_t>(v.size()),
                              numRows, numCols, &h_));
}

template <typename T>
HBDIA<T>::~HBDIA() {
    hbdia_matrix_destroy(h_);
}

template <typename T>
HBDIA<T>::HBDIA(HBDIA &&o) noexcept : h_(o.h_), executionMode_(o.executionMode_) {
    o.h_ = nullptr;
}

template <typename T>
HBDIA<T> &HBDIA<T>::operator=(HBDIA &&o) noexcept {
    if (this != &o) {
        hbdia_matrix_destroy(h_);
        h_ = o.h_;
        executionMode_ = o.executionMode_;
        o.h_ = nullptr;
        layoutCached_ = cooCached_ = diaCached_ = false;
    }
    return *this;
}

template <typename T>
bool HBDIA<T>::loadMTX(const std::string &f) {
    int32_t ok = 0;
    raise(hbdia_matrix_load_mtx(h_, f.c_str(), 0, 0, &ok));
    layoutCached_ = cooCached_ = diaCached_ = false;
    return ok != 0;
}

template <typename T>
bool HBDIA<T>::loadMTX(const std::string &f, int numRows, int numCols) {
    if (numRows <= 0 || numCols <= 0) return false;  // src/Format/HBDIA.cpp:267-271
    int32_t ok = 0;
    raise(hbdia_matrix_load_mtx(h_, f.c_str(), numRows, numCols, &ok));
    layoutCached_ = cooCached_ = diaCached_ = false;
    return ok != 0;
}

template <typename T>
void HBDIA<T>::create3DStencil27Point(int nx, int ny, int nz, double noise, int iteration) {
    raise(hbdia_matrix_stencil27(h_, nx, ny, nz, noise, iteration));
    layoutCached_ = cooCached_ = diaCached_ = false;
}

template <typename T>
void HBDIA<T>::convertToHBDIAFormat(int blockWidth, int threshold, int maxCoo, bool cooUnique,
                                    ExecutionMode execMode) {
    if (!isHBDIAFormat()) executionMode_ = execMode;
    raise(hbdia_matrix_convert(h_, blockWidth, threshold, maxCoo, cooUnique ? 1 : 0,
                               execMode == ExecutionMode::GPU_COO ? HBDIA_GPU_COO : HBDIA_CPU_COO, 1));
    layoutCached_ = false;
}

template <typename T>
void HBDIA<T>::prepareForGPU() {
    raise(hbdia_matrix_prepare_gpu(h_, HBDIA_STORE_NATIVE));
}

template <typename T>
void HBDIA<T>::prepareForGPU(hbdia_value_storage storage) {
    raise(hbdia_matrix_prepare_gpu(h_, storage));
}

template <typename T>
void HBDIA<T>::removeCOODuplicates() {
    raise(hbdia_matrix_remove_duplicates(h_));
    cooCached_ = false;
}

template <typename T>
void HBDIA<T>::convertToDIAFormat(bool cooUnique) {
    raise(hbdia_matrix_convert_dia(h_, cooUnique ? 1 : 0));
    cooCached_ = diaCached_ = false;  // without cooUnique the COO loses its duplicates
}

template <typename T>
bool HBDIA<T>::isDIAFormat() const {
    int32_t has = 0, nd = 0, len = 0;
    raise(hbdia_matrix_dia_info(h_, &has, &nd, &len));
    return has != 0;
}

template <typename T>
void HBDIA<T>::refreshDiaCache() const {
    if (diaCached_) return;
    int32_t has = 0, nd = 0, len = 0;
    raise(hbdia_matrix_dia_info(h_, &has, &nd, &len));
    diaOffsets_.assign(static_cast<size_t>(has ? nd : 0), 0);
    diagonals_.clear();
    if (has && nd > 0) {
        std::vector<T> flat(static_cast<size_t>(nd) * static_cast<size_t>(len));
        raise(hbdia_matrix_export_dia(h_, diaOffsets_.data(), flat.data()));
        diagonals_.resize(static_cast<size_t>(nd));
        for (int32_t d = 0; d < nd; ++d)
            diagonals_[d].assign(flat.begin() + static_cast<size_t>(d) * len,
                                 flat.begin() + static_cast<size_t>(d + 1) * len);
    }
    diaCached_ = true;
}

template <typename T>
const std::vector<std::vector<T>> &HBDIA<T>::getDiagonals() const { refreshDiaCache(); return diagonals_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getOffsets() const { refreshDiaCache(); return diaOffsets_; }

template <typename T>
hbdia_device_arrays HBDIA<T>::deviceArrays() const {
    hbdia_device_arrays a{};
    const hbdia_matrix_info i = info_of<T>(h_);
    if (!i.hasHBDIA) return a;  // nothing on the device yet: the reference's getters return null too
    const int status = hbdia_matrix_device_arrays(h_, &a);
    if (status == HBDIA_ERR_NOT_CONVERTED) return hbdia_device_arrays{};  // converted on the host only
    raise(status);
    return a;
}

template <typename T>
const T *HBDIA<T>::getHBDIADataDevice() const { return static_cast<const T *>(deviceArrays().hbdiaData); }
template <typename T>
const int *HBDIA<T>::getFlattenedOffsetsDevice() const { return deviceArrays().flattenedOffsets; }
template <typename T>
const int *HBDIA<T>::getBlockStartIndicesDevice() const { return deviceArrays().blockStartIndices; }
template <typename T>
const int *HBDIA<T>::getBlockSizesDevice() const { return deviceArrays().blockSizes; }
template <typename T>
const int *HBDIA<T>::getFlattenedVectorOffsetsDevice() const { return deviceArrays().flattenedVectorOffsets; }
template <typename T>
const int *HBDIA<T>::getCpuRowIndicesDevice() const { return deviceArrays().cpuRowIndices; }
template <typename T>
const int *HBDIA<T>::getCpuColIndicesDevice() const { return deviceArrays().cpuColIndices; }
template <typename T>
const T *HBDIA<T>::getCpuValuesDevice() const { return static_cast<const T *>(deviceArrays().cpuValues); }
template <typename T>
const int *HBDIA<T>::getCpuRowPtrDevice() const { return deviceArrays().cpuRowPtr; }

template <typename T>
bool HBDIA<T>::isCOOFormat() const { return info_of<T>(h_).hasCOO != 0; }
template <typename T>
bool HBDIA<T>::isHBDIAFormat() const { return info_of<T>(h_).hasHBDIA != 0; }
template <typename T>
int HBDIA<T>::getNumRows() const { return info_of<T>(h_).numRows; }
template <typename T>
int HBDIA<T>::getNumCols() const { return info_of<T>(h_).numCols; }
template <typename T>
int HBDIA<T>::getNumNonZeros() const { return static_cast<int>(info_of<T>(h_).numNonZeros); }
template <typename T>
int HBDIA<T>::getBlockWidth() const { return info_of<T>(h_).blockWidth; }
template <typename T>
int HBDIA<T>::getThreshold() const { return info_of<T>(h_).threshold; }
template <typename T>
int HBDIA<T>::getMaxCooEntries() const { return static_cast<int>(info_of<T>(h_).maxCooEntries); }
template <typename T>
int HBDIA<T>::getNumBlocks() const { return info_of<T>(h_).numBlocks; }
template <typename T>
int HBDIA<T>::getNumberDiagonals() const { return info_of<T>(h_).numberDiagonals; }

template <typename T>
void HBDIA<T>::refreshHostCache() const {
    if (layoutCached_) return;
    const hbdia_matrix_info i = info_of<T>(h_);
    if (!i.hasHBDIA) {
        data_.clear(); offsetsPerBlock_.clear(); cpuRow_.clear(); cpuCol_.clear(); cpuValues_.clear();
        cpuRowPtr_.clear(); histBlocks_.clear(); histNnz_.clear();
        return;
    }
    std::vector<int> offs(static_cast<size_t>(i.totalOffsets)), start(static_cast<size_t>(i.numBlocks) + 1);
    data_.assign(static_cast<size_t>(i.numSlots), T(0));
    cpuRow_.assign(static_cast<size_t>(i.numCoo), 0);
    cpuCol_.assign(static_cast<size_t>(i.numCoo), 0);
    cpuValues_.assign(static_cast<size_t>(i.numCoo), T(0));
    cpuRowPtr_.assign(static_cast<size_t>(i.numRows) + 1, 0);
    histBlocks_.assign(static_cast<size_t>(i.histogramLength), 0);
    histNnz_.assign(static_cast<size_t>(i.histogramLength), 0);
    raise(hbdia_matrix_export_layout(h_, offs.data(), start.data(), data_.data(), cpuRow_.data(), cpuCol_.data(),
                                     cpuValues_.data(), cpuRowPtr_.data(), histBlocks_.data(), histNnz_.data()));
    offsetsPerBlock_.assign(static_cast<size_t>(i.numBlocks), {});
    for (int b = 0; b < i.numBlocks; ++b) offsetsPerBlock_[b].assign(offs.begin() + start[b], offs.begin() + start[b + 1]);
    layoutCached_ = true;
}

template <typename T>
void HBDIA<T>::refreshCooCache() const {
    if (cooCached_) return;
    const hbdia_matrix_info i = info_of<T>(h_);
    rows_.assign(static_cast<size_t>(i.numNonZeros), 0);
    cols_.assign(static_cast<size_t>(i.numNonZeros), 0);
    values_.assign(static_cast<size_t>(i.numNonZeros), T(0));
    raise(hbdia_matrix_export_coo(h_, rows_.data(), cols_.data(), values_.data()));
    nnzPerRow_.assign(static_cast<size_t>(i.numRows), 0);
    raise(hbdia_matrix_export_nnz_per_row(h_, nnzPerRow_.data()));
    cooCached_ = true;
}

template <typename T>
const std::vector<T> &HBDIA<T>::getValues() const { refreshCooCache(); return values_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getRowIndices() const { refreshCooCache(); return rows_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getColIndices() const { refreshCooCache(); return cols_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getNnzPerRow() const { refreshCooCache(); return nnzPerRow_; }
template <typename T>
const std::vector<T> &HBDIA<T>::getHBDIAData() const { refreshHostCache(); return data_; }
template <typename T>
const std::vector<std::vector<int>> &HBDIA<T>::getOffsetsPerBlock() const { refreshHostCache(); return offsetsPerBlock_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getCpuRowIndices() const { refreshHostCache(); return cpuRow_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getCpuColIndices() const { refreshHostCache(); return cpuCol_; }
template <typename T>
const std::vector<T> &HBDIA<T>::getCpuValues() const { refreshHostCache(); return cpuValues_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getCpuRowPtr() const { refreshHostCache(); return cpuRowPtr_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getHistogramBlocks() const { refreshHostCache(); return histBlocks_; }
template <typename T>
const std::vector<int> &HBDIA<T>::getHistogramNnz() const { refreshHostCache(); return histNnz_; }

template <typename T>
void *HBDIA<T>::getBDIAStream() const {
    void *s = nullptr;
    raise(hbdia_matrix_stream(h_, &s));
    return s;
}

template <typename T>
void HBDIA<T>::synchronize() const {
    raise(hbdia_matrix_synchronize(h_));
}

// ---------------------------------------------------------------- HBDIAVector<T>
template <typename T>
HBDIAVector<T>::HBDIAVector() {}  // no device buffer until assigned

template <typename T>
HBDIAVector<T>::HBDIAVector(const std::vector<T> &localData) : localVector_(localData) {
    raise(hbdia_vector_create(dtype_of<T>(), localData.data(), static_cast<int64_t>(localData.size()), &h_));
}

template <typename T>
HBDIAVector<T>::HBDIAVector(const std::vector<T> &localData, bool, bool, bool, bool) : HBDIAVector(localData) {}

template <typename T>
HBDIAVector<T>::~HBDIAVector() {
    hbdia_vector_destroy(h_);
}

template <typename T>
HBDIAVector<T>::HBDIAVector(HBDIAVector &&o) noexcept : localVector_(std::move(o.localVector_)), h_(o.h_) {
    o.h_ = nullptr;
}

template <typename T>
HBDIAVector<T> &HBDIAVector<T>::operator=(HBDIAVector &&o) noexcept {
    if (this != &o) {
        hbdia_vector_destroy(h_);
        localVector_ = std::move(o.localVector_);
        h_ = o.h_;
        o.h_ = nullptr;
    }
    return *this;
}

template <typename T>
T *HBDIAVector<T>::getDeviceDataPtr() const {
    void *p = nullptr;
    raise(hbdia_vector_device_ptr(h_, &p));
    return static_cast<T *>(p);
}

template <typename T>
T *HBDIAVector<T>::getDeviceCOOResultsPtr() const {
    void *p = nullptr;
    raise(hbdia_vector_coo_results_ptr(h_, &p));
    return static_cast<T *>(p);
}

template <typename T>
void HBDIAVector<T>::copyToHost(std::vector<T> &out) const {
    int64_t n = 0;
    raise(hbdia_vector_size(h_, &n));
    out.resize(static_cast<size_t>(n));
    raise(hbdia_vector_download(h_, out.data()));
}

template <typename T>
void HBDIAVector<T>::copyFromHost(const std::vector<T> &in) {
    int64_t n = 0;
    raise(hbdia_vector_size(h_, &n));
    if (static_cast<int64_t>(in.size()) != n) throw std::invalid_argument("size mismatch");
    raise(hbdia_vector_upload(h_, in.data()));
    localVector_ = in;
}

// ---------------------------------------------------------------- hbdiaSpMV
template <typename T>
bool hbdiaSpMV(HBDIA<T> &matrix, const HBDIAVector<T> &x, HBDIAVector<T> &y, bool execCooCPU, bool execCooGPU) {
    raise(hbdia_spmv(matrix.handle(), x.handle(), y.handle(), execCooCPU ? 1 : 0, execCooGPU ? 1 : 0));
    return true;
}

template class HBDIA<double>;
template class HBDIA<float>;
template class HBDIAVector<double>;
template class HBDIAVector<float>;
template bool hbdiaSpMV<double>(HBDIA<double> &, const HBDIAVector<double> &, HBDIAVector<double> &, bool, bool);
template bool hbdiaSpMV<float>(HBDIA<float> &, const HBDIAVector<float> &, HBDIAVector<float> &, bool, bool);
