// Row-partitioned distribution, host side: one rank's rows of a square matrix
// as a "partial matrix", and what that rank needs of the other ranks' x.
//
//  * partition_rows: BasicExtractor::partitionRowWise
//    (src/DataExchange/BasicExtractor.cpp:124-234) -- contiguous row ranges of
//    numRows / P rows, the last one taking the remainder; a partition keeps its
//    entries in input order, rows made local, columns global.
//  * partial_metadata:
//      - dataRanges, HBDIA::analyzeDataRanges (src/Format/HBDIA.cpp:1333-1414):
//        the merged ascending ranges of global columns the rank reads -- every
//        column of its COO input and, for every kept offset of every block,
//        the column each lane's row reads there (inside [0, numGlobalCols)).
//        Only lanes with a row are counted: the reference also reads the
//        global row mapping past its end for the lanes of a partial last
//        block, which has no defined result;
//      - processDataRanges, BasicExtractor::extractPartialMatrixMetadataRowWise
//        (BasicExtractor.cpp:269-333): each range split at the ranks' row
//        boundaries, in the reference's order, with totalBufferSize;
//      - the receive-buffer sizes of HBDIAVector(localData, matrix, rank, size)
//        (src/Format/HBDIAVector.cpp:39-66);
//      - this library's x window: the smallest column range holding the
//        rank's own rows and every data range.  The rank's plan reads x
//        through the window (x_window[c - lo] holds x[c]) with the fused
//        single-GPU kernels unchanged; only the data ranges owned by other
//        ranks travel.

#include <algorithm>
#include <limits>

#include "hbdia_internal.hpp"

namespace hbdia {

template <typename T>
void partition_rows(const Coo<T> &g, int32_t numProcesses, int32_t part, Coo<T> &local) {
    if (numProcesses <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "Invalid number of processes");
    if (part < 0 || part >= numProcesses) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "partition index out of range");
    const int64_t nnz = static_cast<int64_t>(g.vals.size());
    if (g.numRows <= 0 || g.numCols <= 0 || nnz == 0)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "Invalid matrix dimensions");
    if (g.numRows != g.numCols)
        throw Error(HBDIA_ERR_UNSUPPORTED, "row partitioning needs a square matrix (x is partitioned like the rows)");
    const int32_t rpp = g.numRows / numProcesses;
    if (rpp == 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "more processes than rows");
    const int32_t start = part * rpp;
    const int32_t count = rpp + (part == numProcesses - 1 ? g.numRows % numProcesses : 0);
    const int32_t end = start + count;
    local = Coo<T>();
    int64_t k = 0;
    for (int64_t i = 0; i < nnz; ++i) k += g.rows[i] >= start && g.rows[i] < end;
    local.rows.reserve(static_cast<size_t>(k));
    local.cols.reserve(static_cast<size_t>(k));
    local.vals.reserve(static_cast<size_t>(k));
    for (int64_t i = 0; i < nnz; ++i) {
        const int32_t r = g.rows[i];
        if (r < start || r >= end) continue;
        local.rows.push_back(r - start);
        local.cols.push_back(g.cols[i]);
        local.vals.push_back(g.vals[i]);
    }
    local.numRows = count;
    local.numCols = g.numCols;  // numLocalCols = numCols (BasicExtractor.cpp:147)
    local.rowBase = start;
}

void process_ranges(PartialMeta &m) {
    const int32_t P = m.size;
    const int32_t rpp = m.numGlobalRows / P;
    if (rpp <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "more processes than rows");
    m.processRanges.clear();
    m.totalBufferSize = 0;
    std::vector<std::vector<int32_t>> per(static_cast<size_t>(P));
    const size_t nr = m.dataRanges.size() / 2;
    for (size_t i = 0; i < nr; ++i) {
        const int32_t s = m.dataRanges[2 * i], e = m.dataRanges[2 * i + 1];
        m.totalBufferSize += e - s;
        const int32_t p0 = std::max(0, std::min(s / rpp, P - 1));
        const int32_t p1 = std::max(0, std::min((e - 1) / rpp, P - 1));
        int32_t cur = s;
        for (int32_t p = p0; p <= p1 && cur < e; ++p) {
            const int64_t boundary = p == P - 1 ? e : static_cast<int64_t>(p + 1) * rpp;
            const int32_t segEnd = static_cast<int32_t>(std::min<int64_t>(e, boundary));
            if (cur < segEnd) {
                per[p].push_back(cur);
                per[p].push_back(segEnd);
                cur = segEnd;
            }
        }
    }
    m.leftBufferSize = m.rightBufferSize = 0;
    for (int32_t p = 0; p < P; ++p) {
        for (size_t j = 0; j < per[p].size(); j += 2) {
            m.processRanges.push_back(p);
            m.processRanges.push_back(per[p][j]);
            m.processRanges.push_back(per[p][j + 1]);
            const int64_t len = per[p][j + 1] - per[p][j];
            if (p < m.rank) m.leftBufferSize += len;
            else if (p > m.rank) m.rightBufferSize += len;
        }
    }
}

template <typename T>
void partial_metadata(const Coo<T> &c, const HostLayout<T> &L, PartialMeta &m) {
    const int32_t nGC = m.numGlobalCols;
    const int32_t rb = c.rowBase;
    // coverage of [0, nGC) as a difference array: +1 at a range's start,
    // -1 past its end
    std::vector<int32_t> diff(static_cast<size_t>(nGC) + 1, 0);
    for (int32_t col : c.cols) {
        diff[col]++;
        diff[static_cast<size_t>(col) + 1]--;
    }
    const int32_t bw = L.blockWidth;
    for (int32_t b = 0; b < L.numBlocks; ++b) {
        const int64_t row0 = static_cast<int64_t>(b) * bw;
        const int64_t lanes = std::min<int64_t>(bw, L.numRows - row0);
        for (int32_t k = L.blockStart[b]; k < L.blockStart[b + 1]; ++k) {
            const int64_t g0 = rb + row0 + L.offsets[k];
            const int64_t lo = std::max<int64_t>(g0, 0), hi = std::min<int64_t>(g0 + lanes, nGC);
            if (lo < hi) {
                diff[lo]++;
                diff[hi]--;
            }
        }
    }
    m.dataRanges.clear();
    int64_t run = 0;
    int32_t open = -1;
    for (int32_t col = 0; col <= nGC; ++col) {
        run += diff[col];
        const bool covered = col < nGC && run > 0;
        if (covered && open < 0) open = col;
        if (!covered && open >= 0) {
            m.dataRanges.push_back(open);
            m.dataRanges.push_back(col);
            open = -1;
        }
    }
    process_ranges(m);
    int64_t lo = rb, hi = static_cast<int64_t>(rb) + c.numRows;
    if (!m.dataRanges.empty()) {
        lo = std::min<int64_t>(lo, m.dataRanges.front());
        hi = std::max<int64_t>(hi, m.dataRanges.back());
    }
    m.windowLo = static_cast<int32_t>(lo);
    m.windowLen = static_cast<int32_t>(hi - lo);
    m.hasMetadata = true;
}

template void partition_rows<double>(const Coo<double> &, int32_t, int32_t, Coo<double> &);
template void partition_rows<float>(const Coo<float> &, int32_t, int32_t, Coo<float> &);
template void partial_metadata<double>(const Coo<double> &, const HostLayout<double> &, PartialMeta &);
template void partial_metadata<float>(const Coo<float> &, const HostLayout<float> &, PartialMeta &);

}  // namespace hbdia
