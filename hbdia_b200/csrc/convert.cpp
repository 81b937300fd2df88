// COO -> HBDIA conversion on the host, bit-exact with the reference's
// HBDIA<T>::convertToHBDIAFormat (src/Format/HBDIA.cpp:507-718), restated as
// a parallel (OpenMP) pipeline:
//
//   1. bucket entries by row block (for row-sorted input the buckets are just
//      contiguous ranges, found by binary search);
//   2. per block, the ascending distinct (offset, count) pairs -- what the
//      reference's std::map<int,int> per block holds (HBDIA.cpp:540-560);
//   3. the keep/drop filter (HBDIA.cpp:567-586).  Its `cpu_entries >=
//      max_coo_entries` clause depends on a running count across blocks; when
//      the total of all candidate counts cannot reach the limit the filter is
//      a per-offset test and runs in parallel, otherwise it runs sequentially
//      in the reference's block/offset order;
//   4. the fill (HBDIA.cpp:634-703): a kept slot is ASSIGNED (duplicates are
//      last-wins) and all other entries form the COO remainder in input
//      order.  For row-sorted input every (row, col) pair lives in one block,
//      so filling blocks in parallel, each in input order, gives the same
//      last-wins result; unsorted input is filled sequentially.
//
// Only the layout's contents are the reference's; the algorithm (no maps, no
// per-entry std::find) is this library's own.

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>

#include "hbdia_internal.hpp"

namespace hbdia {
namespace {

struct OffCount {
    int32_t off;
    int32_t cnt;
};

// Find `key` in the ascending unique list [list, list+n), starting with the
// slot after the previous hit (offsets of consecutive entries in a row are
// usually ascending), then by binary search.  Returns -1 when absent.
inline int64_t find_with_cursor(const int32_t *list, int64_t n, int32_t key, int64_t &cursor) {
    if (cursor < n && list[cursor] == key) return cursor++;
    const int32_t *p = std::lower_bound(list, list + n, key);
    if (p != list + n && *p == key) {
        cursor = (p - list) + 1;
        return p - list;
    }
    return -1;
}

// Distinct (offset, count) of one block's entries, ascending by offset.
template <typename EntryFn>
void block_histogram(int64_t j0, int64_t j1, const int32_t *R, const int32_t *C, int32_t rb, EntryFn entry,
                     std::vector<OffCount> &list, std::vector<int32_t> &scratch) {
    list.clear();
    size_t cursor = 0;
    bool overflow = false;
    for (int64_t j = j0; j < j1; ++j) {
        const int64_t i = entry(j);
        const int32_t off = C[i] - R[i] - rb;
        if (cursor < list.size() && list[cursor].off == off) {
            list[cursor++].cnt++;
            continue;
        }
        auto it = std::lower_bound(list.begin(), list.end(), off,
                                   [](const OffCount &a, int32_t k) { return a.off < k; });
        if (it != list.end() && it->off == off) {
            it->cnt++;
        } else {
            if (list.size() >= 512) {  // many distinct offsets: sort instead
                overflow = true;
                break;
            }
            it = list.insert(it, OffCount{off, 1});
        }
        cursor = static_cast<size_t>(it - list.begin()) + 1;
    }
    if (!overflow) return;
    scratch.clear();
    for (int64_t j = j0; j < j1; ++j) {
        const int64_t i = entry(j);
        scratch.push_back(C[i] - R[i] - rb);
    }
    std::sort(scratch.begin(), scratch.end());
    list.clear();
    for (size_t a = 0; a < scratch.size();) {
        size_t b = a;
        while (b < scratch.size() && scratch[b] == scratch[a]) ++b;
        list.push_back(OffCount{scratch[a], static_cast<int32_t>(b - a)});
        a = b;
    }
}

}  // namespace

template <typename T>
void convert_to_hbdia(const Coo<T> &coo, int32_t bw, int32_t thr, int64_t maxCoo,
                      HostLayout<T> &L) {
    if (bw <= 0) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "blockWidth must be positive");
    const int64_t nnz = static_cast<int64_t>(coo.vals.size());
    const int32_t nR = coo.numRows, nC = coo.numCols;
    const int32_t rb = coo.rowBase;  // 0 unless a partial matrix
    const int32_t *R = coo.rows.data();
    const int32_t *C = coo.cols.data();
    const T *V = coo.vals.data();

    L = HostLayout<T>();
    L.numRows = nR;
    L.numCols = nC;
    L.blockWidth = bw;
    L.threshold = thr;
    L.maxCoo = maxCoo;
    L.rowBase = rb;
    // maxNumBlocks = ceil(min(numRows, numCols) / blockWidth)   (HBDIA.cpp:537)
    const int32_t nb = static_cast<int32_t>((static_cast<int64_t>(std::min(nR, nC)) + bw - 1) / bw);
    L.numBlocks = nb;

    // ---- 1. bucket entries by block
    bool sorted = true;
#pragma omp parallel for reduction(&& : sorted) schedule(static)
    for (int64_t i = 1; i < nnz; ++i) sorted = sorted && (R[i - 1] <= R[i]);

    std::vector<int64_t> bstart(static_cast<size_t>(nb) + 1, 0);
    std::vector<int32_t> perm;  // unsorted input: entry indices grouped by block
    if (sorted) {
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b <= nb; ++b) {
            const int64_t rowKey = std::min<int64_t>(b * bw, std::numeric_limits<int32_t>::max());
            bstart[b] = std::lower_bound(R, R + nnz, rowKey,
                                         [](int32_t a, int64_t k) { return a < k; }) - R;
        }
    } else {
        for (int64_t i = 0; i < nnz; ++i) {
            const int32_t b = R[i] / bw;
            if (b < nb) bstart[b + 1]++;
        }
        for (int32_t b = 0; b < nb; ++b) bstart[b + 1] += bstart[b];
        perm.resize(static_cast<size_t>(bstart[nb]));
        std::vector<int64_t> fill(bstart.begin(), bstart.end() - 1);
        for (int64_t i = 0; i < nnz; ++i) {
            const int32_t b = R[i] / bw;
            if (b < nb) perm[fill[b]++] = static_cast<int32_t>(i);
        }
    }
    const int32_t *P = perm.data();
    auto entry = [sorted, P](int64_t j) -> int64_t { return sorted ? j : P[j]; };
    const int64_t inBlocks = bstart[nb];

    // ---- 2. distinct (offset, count) per block, stored in the block's own
    // entry range of uoff/ucnt (distinct <= entries)
    std::vector<int32_t> uoff(static_cast<size_t>(inBlocks)), ucnt(static_cast<size_t>(inBlocks));
    std::vector<int32_t> ndist(static_cast<size_t>(nb), 0);
#pragma omp parallel
    {
        std::vector<OffCount> list;
        std::vector<int32_t> scratch;
        list.reserve(64);
#pragma omp for schedule(dynamic, 256)
        for (int64_t b = 0; b < nb; ++b) {
            block_histogram(bstart[b], bstart[b + 1], R, C, rb, entry, list, scratch);
            for (size_t u = 0; u < list.size(); ++u) {
                uoff[bstart[b] + u] = list[u].off;
                ucnt[bstart[b] + u] = list[u].cnt;
            }
            ndist[b] = static_cast<int32_t>(list.size());
        }
    }

    // ---- 3. filter (HBDIA.cpp:571-583)
    std::vector<uint8_t> keep(static_cast<size_t>(inBlocks), 0);
    int64_t candidates = 0;
#pragma omp parallel for reduction(+ : candidates) schedule(static)
    for (int64_t b = 0; b < nb; ++b)
        for (int32_t u = 0; u < ndist[b]; ++u)
            if (ucnt[bstart[b] + u] < thr) candidates += ucnt[bstart[b] + u];
    if (candidates <= maxCoo) {
        // cpu_entries stays below max_coo_entries at every check
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < nb; ++b)
            for (int32_t u = 0; u < ndist[b]; ++u)
                keep[bstart[b] + u] = ucnt[bstart[b] + u] >= thr;
    } else {
        int64_t cpu_entries = 0;
        for (int64_t b = 0; b < nb; ++b) {
            for (int32_t u = 0; u < ndist[b]; ++u) {
                const int32_t c = ucnt[bstart[b] + u];
                if (c >= thr || cpu_entries >= maxCoo) keep[bstart[b] + u] = 1;
                else cpu_entries += c;
            }
        }
    }

    // numberDiagonals: distinct offsets over all blocks (HBDIA.cpp:563,585)
    {
        // offsets in [-(rb+nR-1), nC-1]
        const int64_t span = static_cast<int64_t>(rb) + nR + nC;
        std::vector<uint64_t> bits(static_cast<size_t>((span + 63) / 64), 0);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t b = 0; b < nb; ++b)
            for (int32_t u = 0; u < ndist[b]; ++u) {
                const int64_t k = static_cast<int64_t>(uoff[bstart[b] + u]) + rb + (nR - 1);
                __atomic_fetch_or(&bits[k >> 6], uint64_t(1) << (k & 63), __ATOMIC_RELAXED);
            }
        int64_t nd = 0;
#pragma omp parallel for reduction(+ : nd) schedule(static)
        for (int64_t w = 0; w < static_cast<int64_t>(bits.size()); ++w) nd += __builtin_popcountll(bits[w]);
        L.numberDiagonals = static_cast<int32_t>(nd);
    }

    // ---- kept offsets, flattened (prepareForGPU's form, HBDIA.cpp:733-760)
    std::vector<int64_t> kstart(static_cast<size_t>(nb) + 1, 0);
    for (int64_t b = 0; b < nb; ++b) {
        int64_t k = 0;
        for (int32_t u = 0; u < ndist[b]; ++u) k += keep[bstart[b] + u];
        kstart[b + 1] = kstart[b] + k;
    }
    const int64_t totalOffsets = kstart[nb];
    const int64_t slots = totalOffsets * bw;
    // storage guard (HBDIA.cpp:592-598)
    if (static_cast<double>(slots) > 1e11)
        throw Error(HBDIA_ERR_RUNTIME, "Excessive memory requirement for HBDIA format");
    if (totalOffsets > std::numeric_limits<int32_t>::max())
        throw Error(HBDIA_ERR_UNSUPPORTED, "more than 2^31-1 stored offsets");
    L.offsets.resize(static_cast<size_t>(totalOffsets));
    L.blockStart.resize(static_cast<size_t>(nb) + 1);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; ++b) {
        L.blockStart[b] = static_cast<int32_t>(kstart[b]);
        int64_t p = kstart[b];
        for (int32_t u = 0; u < ndist[b]; ++u)
            if (keep[bstart[b] + u]) L.offsets[p++] = uoff[bstart[b] + u];
    }
    L.blockStart[nb] = static_cast<int32_t>(totalOffsets);
    std::vector<int32_t>().swap(uoff);
    std::vector<int32_t>().swap(ucnt);
    std::vector<uint8_t>().swap(keep);

    // zero-filled value storage (HBDIA.cpp:600,617), filled in parallel
    L.data.resize(static_cast<size_t>(slots));

    // histograms (HBDIA.cpp:619-631)
    int32_t maxd = 0;
    for (int64_t b = 0; b < nb; ++b) maxd = std::max<int32_t>(maxd, L.blockStart[b + 1] - L.blockStart[b]);
    L.histBlocks.assign(static_cast<size_t>(maxd) + 1, 0);
    L.histNnz.assign(static_cast<size_t>(maxd) + 1, 0);
    for (int64_t b = 0; b < nb; ++b) L.histBlocks[L.blockStart[b + 1] - L.blockStart[b]]++;

    // ---- 4. fill (HBDIA.cpp:634-703)
    const int32_t *KO = L.offsets.data();
    const int32_t *KS = L.blockStart.data();
    T *D = L.data.data();
    if (sorted) {
        const int nthreads = omp_get_max_threads();
        std::vector<std::vector<int64_t>> hist(static_cast<size_t>(nthreads),
                                               std::vector<int64_t>(static_cast<size_t>(maxd) + 1, 0));
        std::vector<int64_t> cooCount(static_cast<size_t>(nb) + 1, 0);
#pragma omp parallel
        {
            std::vector<int64_t> &h = hist[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 256)
            for (int64_t b = 0; b < nb; ++b) {
                const int64_t nk = KS[b + 1] - KS[b];
                int64_t cursor = 0, ncoo = 0;
                for (int64_t i = bstart[b]; i < bstart[b + 1]; ++i) {
                    const int64_t idx = nk ? find_with_cursor(KO + KS[b], nk, C[i] - R[i] - rb, cursor) : -1;
                    if (idx >= 0) {
                        D[(static_cast<int64_t>(KS[b]) + idx) * bw + (R[i] % bw)] = V[i];
                        h[nk]++;
                    } else {
                        ++ncoo;
                    }
                }
                cooCount[b + 1] = ncoo;
            }
        }
        for (int t = 0; t < nthreads; ++t)
            for (int32_t d = 0; d <= maxd; ++d) L.histNnz[d] += static_cast<int32_t>(hist[t][d]);
        for (int64_t b = 0; b < nb; ++b) cooCount[b + 1] += cooCount[b];
        const int64_t tail = nnz - inBlocks;  // rows in blocks >= maxNumBlocks: all COO
        const int64_t nCoo = cooCount[nb] + tail;
        L.cooRow.resize(static_cast<size_t>(nCoo));
        L.cooCol.resize(static_cast<size_t>(nCoo));
        L.cooVal.resize(static_cast<size_t>(nCoo));
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t b = 0; b < nb; ++b) {
            if (cooCount[b + 1] == cooCount[b]) continue;
            const int64_t nk = KS[b + 1] - KS[b];
            int64_t cursor = 0, p = cooCount[b];
            for (int64_t i = bstart[b]; i < bstart[b + 1]; ++i) {
                const int64_t idx = nk ? find_with_cursor(KO + KS[b], nk, C[i] - R[i] - rb, cursor) : -1;
                if (idx < 0) {
                    L.cooRow[p] = R[i];
                    L.cooCol[p] = C[i];
                    L.cooVal[p] = V[i];
                    ++p;
                }
            }
        }
        if (tail > 0) {
            std::memcpy(&L.cooRow[cooCount[nb]], R + inBlocks, sizeof(int32_t) * tail);
            std::memcpy(&L.cooCol[cooCount[nb]], C + inBlocks, sizeof(int32_t) * tail);
            std::memcpy(&L.cooVal[cooCount[nb]], V + inBlocks, sizeof(T) * tail);
        }
    } else {
        for (int64_t i = 0; i < nnz; ++i) {
            const int32_t b = R[i] / bw;
            int64_t idx = -1, nk = 0, cursor = 0;
            if (b < nb) {
                nk = KS[b + 1] - KS[b];
                if (nk) idx = find_with_cursor(KO + KS[b], nk, C[i] - R[i] - rb, cursor);
            }
            if (idx >= 0) {
                D[(static_cast<int64_t>(KS[b]) + idx) * bw + (R[i] % bw)] = V[i];
                L.histNnz[nk]++;
            } else {
                L.cooRow.push_back(R[i]);
                L.cooCol.push_back(C[i]);
                L.cooVal.push_back(V[i]);
            }
        }
    }

    // CSR row pointer of the COO remainder, built exactly as the reference
    // does (it assumes non-decreasing rows, HBDIA.cpp:671-703)
    L.cooRowPtr.assign(static_cast<size_t>(nR) + 1, 0);
    {
        int32_t currentRow = -1;
        int32_t next = 0;
        const int64_t nCoo = static_cast<int64_t>(L.cooRow.size());
        for (int64_t e = 0; e < nCoo; ++e) {
            const int32_t r = L.cooRow[e];
            if (r != currentRow) {
                for (int32_t q = currentRow + 1; q <= r; ++q) L.cooRowPtr[q] = next;
                currentRow = r;
            }
            ++next;
        }
        for (int32_t q = currentRow + 1; q <= nR; ++q) L.cooRowPtr[q] = next;
        bool cs = true;
        for (int64_t e = 1; e < nCoo && cs; ++e) cs = L.cooRow[e - 1] <= L.cooRow[e];
        L.cooRowSorted = cs;
    }
}

std::vector<int64_t> stable_row_order(const std::vector<int32_t> &rows, int32_t numRows) {
    std::vector<int64_t> cnt(static_cast<size_t>(numRows) + 1, 0);
    for (int32_t r : rows) cnt[static_cast<size_t>(r) + 1]++;
    for (int32_t r = 0; r < numRows; ++r) cnt[r + 1] += cnt[r];
    std::vector<int64_t> order(rows.size());
    for (size_t e = 0; e < rows.size(); ++e) order[cnt[rows[e]]++] = static_cast<int64_t>(e);
    return order;
}

template void convert_to_hbdia<double>(const Coo<double> &, int32_t, int32_t, int64_t, HostLayout<double> &);
template void convert_to_hbdia<float>(const Coo<float> &, int32_t, int32_t, int64_t, HostLayout<float> &);

}  // namespace hbdia
