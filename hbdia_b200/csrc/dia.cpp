// DIA format and storage-cost analytics (host code).
//
//  * remove_coo_duplicates: removeCOODuplicates (src/Format/HBDIA.cpp:372-412)
//    -- entries with the same (row, col) become one whose value is
//    ((0 + v1) + v2) + ... in input order, and the COO comes out sorted by
//    (row, col), as the reference's std::map<pair<int,int>, T> leaves it.
//  * convert_to_dia: convertToDIAFormat (HBDIA.cpp:414-505) for a whole
//    (non-partial) matrix -- ascending distinct offsets col - row, one
//    diagonal of min(numRows, numCols) values per offset, value of (r, c) at
//    position r (positions past the diagonal length dropped), later entries
//    overwriting earlier ones.
//  * storage_costs: the byte counts the reference's benchmark prints and
//    saves (benchmarking/benchmark.cpp:171-215) for HBDIA, COO, DIA, SELL and
//    CSR storage of the matrix.
#include <algorithm>
#include <numeric>
#include <set>

#include "hbdia_internal.hpp"

namespace hbdia {

template <typename T>
void remove_coo_duplicates(Coo<T> &c) {
    const int64_t n = static_cast<int64_t>(c.vals.size());
    if (n == 0) return;
    std::vector<int64_t> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), int64_t(0));
    // (row, col) ascending, input order within equal keys
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        return c.rows[a] != c.rows[b] ? c.rows[a] < c.rows[b] : c.cols[a] < c.cols[b];
    });
    std::vector<int32_t> r, cc;
    std::vector<T> v;
    r.reserve(static_cast<size_t>(n));
    cc.reserve(static_cast<size_t>(n));
    v.reserve(static_cast<size_t>(n));
    for (int64_t i = 0; i < n;) {
        int64_t j = i;
        T sum = T(0);
        while (j < n && c.rows[order[j]] == c.rows[order[i]] && c.cols[order[j]] == c.cols[order[i]]) {
            sum = sum + c.vals[order[j]];
            ++j;
        }
        r.push_back(c.rows[order[i]]);
        cc.push_back(c.cols[order[i]]);
        v.push_back(sum);
        i = j;
    }
    c.rows.swap(r);
    c.cols.swap(cc);
    c.vals.swap(v);
}

template <typename T>
void convert_to_dia(Coo<T> &c, bool cooIsUnique, std::vector<int32_t> &offsets, std::vector<T> &diagonals,
                    int32_t &diagLength) {
    if (!cooIsUnique) remove_coo_duplicates(c);
    const int64_t n = static_cast<int64_t>(c.vals.size());
    std::set<int32_t> uniq;
    for (int64_t i = 0; i < n; ++i) uniq.insert(c.cols[i] - c.rows[i]);
    offsets.assign(uniq.begin(), uniq.end());
    diagLength = std::min(c.numRows, c.numCols);
    const double cells = static_cast<double>(offsets.size()) * diagLength;
    if (cells > 1e11) throw Error(HBDIA_ERR_RUNTIME, "Excessive memory requirement for DIA format");
    diagonals.assign(offsets.size() * static_cast<size_t>(diagLength), T(0));
    for (int64_t i = 0; i < n; ++i) {
        const int32_t off = c.cols[i] - c.rows[i];
        const int64_t d = std::lower_bound(offsets.begin(), offsets.end(), off) - offsets.begin();
        const int32_t pos = c.rows[i];
        if (pos >= 0 && pos < diagLength) diagonals[static_cast<size_t>(d) * diagLength + pos] = c.vals[i];
    }
}

void storage_costs(int64_t valueBytes, int32_t numRows, int32_t numCols, int64_t numNonZeros,
                   int32_t numberDiagonals, int32_t numBlocks, int32_t blockWidth, int64_t hbdiaSlots,
                   int64_t cooEntries, const std::vector<int32_t> &histBlocks, const std::vector<int32_t> &nnzPerRow,
                   hbdia_storage_costs &out) {
    const int64_t I = 4;  // sizeof(int)
    int64_t sumHistBlocks = 0;  // stored offsets: one per diagonal per block
    for (size_t i = 0; i < histBlocks.size(); ++i) sumHistBlocks += static_cast<int64_t>(i) * histBlocks[i];
    out.hbdia = hbdiaSlots * valueBytes + (static_cast<int64_t>(numBlocks) + 1) * I + sumHistBlocks * I +
                cooEntries * I * 2 + cooEntries * valueBytes;
    out.coo = numNonZeros * I * 2 + numNonZeros * valueBytes;
    out.dia = static_cast<int64_t>(numberDiagonals) * std::min(numRows, numCols) * valueBytes +
              static_cast<int64_t>(numberDiagonals) * I;
    // SELL-C with C = blockWidth from the per-row counts (which only the
    // 27-point stencil generator records, as in the reference)
    int64_t sell = 0;
    int32_t mx = 0;
    for (size_t i = 0; i < nnzPerRow.size(); ++i) {
        if (blockWidth > 0 && i % static_cast<size_t>(blockWidth) == 0 && i > 0) {
            sell += static_cast<int64_t>(mx) * blockWidth * valueBytes + static_cast<int64_t>(mx) * blockWidth * I;
            mx = 0;
        }
        mx = std::max(mx, nnzPerRow[i]);
    }
    sell += static_cast<int64_t>(mx) * blockWidth * valueBytes + static_cast<int64_t>(mx) * blockWidth * I;
    const int64_t numSlices = blockWidth > 0 ? (static_cast<int64_t>(numRows) + blockWidth - 1) / blockWidth : 0;
    sell += numSlices * I;
    out.sell = sell;
    out.csr = numNonZeros * valueBytes + numNonZeros * I + (static_cast<int64_t>(numRows) + 1) * I;
}

template void remove_coo_duplicates<double>(Coo<double> &);
template void remove_coo_duplicates<float>(Coo<float> &);
template void convert_to_dia<double>(Coo<double> &, bool, std::vector<int32_t> &, std::vector<double> &, int32_t &);
template void convert_to_dia<float>(Coo<float> &, bool, std::vector<int32_t> &, std::vector<float> &, int32_t &);

}  // namespace hbdia
