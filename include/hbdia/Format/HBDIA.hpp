// Drop-in HBDIA<T> (reference: include/Format/HBDIA.hpp:24-291) for the SpMV
// path, implemented over the C ABI of libhbdia_b200.so (hbdia_b200.h).
//
// The tree include/hbdia/ has the reference's include/ shape (Format/,
// Operations/, types.hpp), so a program written against the reference's
// headers compiles against these when this tree stands where the reference's
// include/ stood (plus -I for hbdia_b200.h and the CUDA headers).
//
// Same names, arguments and defaults as the reference for construction,
// matrix sources, conversion, the host-layout getters (whose contents are
// bit-identical to the reference's), the DIA format and the GPU getters.
// Differences, all deliberate:
//  * move-only: the reference's implicit copy would free device memory twice;
//  * errors throw instead of exit(1) (include/types.hpp:37-44);
//  * the COO remainder always runs on the GPU inside the fused SpMV, so
//    initializeCuSparse() has nothing to do and ExecutionMode is ignored;
//  * the multi-process (partial matrix / MPI) members are not part of this
//    single-GPU C++ layer (the C ABI has the row partitioning).
#ifndef HBDIA_B200_HBDIA_HPP
#define HBDIA_B200_HBDIA_HPP

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "hbdia_b200.h"
#include "../types.hpp"

template <typename T>
class HBDIAVector;

template <typename T>
class HBDIA {
public:
    HBDIA();
    HBDIA(const std::vector<int> &rowIndices, const std::vector<int> &colIndices, const std::vector<T> &values);
    HBDIA(const std::vector<int> &rowIndices, const std::vector<int> &colIndices, const std::vector<T> &values,
          int numRows, int numCols);
    ~HBDIA();
    HBDIA(const HBDIA &) = delete;
    HBDIA &operator=(const HBDIA &) = delete;
    HBDIA(HBDIA &&other) noexcept;
    HBDIA &operator=(HBDIA &&other) noexcept;

    // format loading (src/Format/HBDIA.cpp:161-370, :1416-1607)
    bool loadMTX(const std::string &filename);
    bool loadMTX(const std::string &filename, int numRows, int numCols);
    void create3DStencil27Point(int nx, int ny, int nz, double noise = 0.0, int iteration = 0);

    // format conversion (src/Format/HBDIA.cpp:414-718); convertToHBDIAFormat
    // uploads the device layout, as the reference does for a whole matrix
    void convertToDIAFormat(bool COOisUnique = false);
    bool isDIAFormat() const;
    bool isCOOFormat() const;
    bool isHBDIAFormat() const;
    void convertToHBDIAFormat(int blockWidth = DEFAULT_BLOCK_WIDTH, int threshold = DEFAULT_THRESHOLD,
                              int max_coo_entries = MAX_COO_ENTRIES, bool COOisUnique = false,
                              ExecutionMode execMode = ExecutionMode::GPU_COO);

    // sums entries with equal (row, col) and sorts the COO by (row, col)
    // (src/Format/HBDIA.cpp:372-412)
    void removeCOODuplicates();

    // dimensions and COO input
    int getNumRows() const;
    int getNumCols() const;
    int getNumNonZeros() const;
    const std::vector<T> &getValues() const;
    const std::vector<int> &getRowIndices() const;
    const std::vector<int> &getColIndices() const;
    const std::vector<int> &getNnzPerRow() const;

    // DIA format (include/Format/HBDIA.hpp:89-90): one diagonal of
    // min(numRows, numCols) values per offset, offsets ascending
    const std::vector<std::vector<T>> &getDiagonals() const;
    const std::vector<int> &getOffsets() const;

    // HBDIA host layout (include/Format/HBDIA.hpp:93-108)
    const std::vector<T> &getHBDIAData() const;
    const std::vector<std::vector<int>> &getOffsetsPerBlock() const;
    const std::vector<int> &getCpuRowIndices() const;
    const std::vector<int> &getCpuColIndices() const;
    const std::vector<T> &getCpuValues() const;
    const std::vector<int> &getCpuRowPtr() const;
    int getBlockWidth() const;
    int getThreshold() const;
    int getMaxCooEntries() const;
    int getNumBlocks() const;
    ExecutionMode getExecutionMode() const { return executionMode_; }
    int getNumberDiagonals() const;
    const std::vector<int> &getHistogramBlocks() const;
    const std::vector<int> &getHistogramNnz() const;
    bool getHasCOO() const { return isCOOFormat(); }
    bool getHasDIA() const { return isDIAFormat(); }
    bool getHasHBDIA() const { return isHBDIAFormat(); }

    // GPU getters (include/Format/HBDIA.hpp:155-165): the device arrays the
    // fused SpMV reads, owned by the matrix.  getHBDIADataDevice is null when
    // the values are held in a reduced storage format; the vector offsets are
    // null for a whole matrix, as in the reference; the COO ones are null
    // without a COO remainder.
    const T *getHBDIADataDevice() const;
    const int *getFlattenedOffsetsDevice() const;
    const int *getBlockStartIndicesDevice() const;
    const int *getBlockSizesDevice() const;
    const int *getFlattenedVectorOffsetsDevice() const;
    const int *getCpuRowIndicesDevice() const;
    const int *getCpuColIndicesDevice() const;
    const T *getCpuValuesDevice() const;
    const int *getCpuRowPtrDevice() const;

    // device side
    void prepareForGPU();
    // Addition to the reference's API: the device layout with another value
    // storage (HBDIA_STORE_F32, _BF16_SCALED and the quad-interleaved
    // _F32_QUAD / _BF16_QUAD keep the values narrow; x, y and the
    // accumulation stay in the matrix's type).
    void prepareForGPU(hbdia_value_storage storage);
    void initializeCuSparse() {}  // nothing to set up: the COO remainder is fused
    void *getBDIAStream() const;   // a cudaStream_t
    void synchronize() const;      // waits for the SpMVs on the matrix's stream

    hbdia_matrix *handle() const { return h_; }

private:
    void refreshHostCache() const;
    void refreshCooCache() const;
    void refreshDiaCache() const;
    hbdia_device_arrays deviceArrays() const;
    hbdia_matrix *h_ = nullptr;
    ExecutionMode executionMode_ = ExecutionMode::GPU_COO;
    // host copies handed out by the getters, filled on first use
    mutable bool layoutCached_ = false, cooCached_ = false, diaCached_ = false;
    mutable std::vector<T> data_, cpuValues_, values_;
    mutable std::vector<int> cpuRow_, cpuCol_, cpuRowPtr_, histBlocks_, histNnz_, rows_, cols_, nnzPerRow_;
    mutable std::vector<std::vector<int>> offsetsPerBlock_;
    mutable std::vector<int> diaOffsets_;
    mutable std::vector<std::vector<T>> diagonals_;
};

#endif
