/* Test infrastructure only -- the ORACLE.  A plain-C, single-threaded
 * restatement of the reference's HBDIA conversion and SpMV, written for
 * clarity rather than speed.  tests/, __graft_entry__.smoke() and bench.py's
 * CPU baseline load it as the checker; the product (hbdia_b200) never does.
 *
 * Every function cites the reference code it restates (paths relative to the
 * reference project root).
 */
#include "hbdia_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_layout {
    int32_t numRows, numCols, bw, threshold;
    int32_t rowBase;         /* partial matrix: global row of local row 0 */
    int64_t maxCoo;
    int is_f32;
    int has_hbdia;
    int32_t numBlocks;       /* maxNumBlocks */
    int64_t totalOffsets;
    int64_t slots;
    int32_t *offsets;        /* kept offsets, ascending per block, flattened */
    int32_t *blockStart;     /* numBlocks+1 prefix in offset units */
    void *data;              /* slots values, [block][offsetIdx][lane] */
    int64_t nCoo;
    int32_t *cooRow, *cooCol;
    void *cooVal;
    int32_t *cooRowPtr;      /* numRows+1 */
    int32_t numberDiagonals;
    int32_t histLen;
    int32_t *histBlocks, *histNnz;
};

static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* Binary search in an ascending, duplicate-free list; -1 when absent.  The
 * reference uses std::find over the same list (src/Format/HBDIA.cpp:662),
 * which returns the same index because the list is unique. */
static int64_t find_offset(const int32_t *list, int64_t n, int32_t key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (list[mid] < key) lo = mid + 1; else hi = mid;
    }
    return (lo < n && list[lo] == key) ? lo : -1;
}

int orc_convert(const int32_t *rows, const int32_t *cols, const void *vals, int is_f32,
                int64_t nnz, int32_t numRows, int32_t numCols, int32_t bw, int32_t threshold,
                int64_t maxCoo, orc_layout **out) {
    return orc_convert_partial(rows, cols, vals, is_f32, nnz, numRows, numCols, 0, bw, threshold, maxCoo, out);
}

/* The partial-matrix form: offsets are col - (row + rowBase), the global row
 * taken from a contiguous global row mapping (src/Format/HBDIA.cpp:546-552,
 * 646-657); blocks, lanes and the COO remainder use local rows. */
int orc_convert_partial(const int32_t *rows, const int32_t *cols, const void *vals, int is_f32,
                        int64_t nnz, int32_t numRows, int32_t numCols, int32_t rowBase, int32_t bw,
                        int32_t threshold, int64_t maxCoo, orc_layout **out) {
    if (!out || bw <= 0 || numRows <= 0 || numCols <= 0 || nnz < 0 || rowBase < 0) return -1;
    orc_layout *h = (orc_layout *)calloc(1, sizeof(orc_layout));
    if (!h) return -1;
    const size_t esz = is_f32 ? sizeof(float) : sizeof(double);
    h->numRows = numRows; h->numCols = numCols; h->bw = bw; h->threshold = threshold;
    h->maxCoo = maxCoo; h->is_f32 = is_f32; h->rowBase = rowBase;
    *out = h;
    /* Empty matrix: the reference returns without converting
     * (src/Format/HBDIA.cpp:521-524). */
    if (nnz == 0) return 0;

    /* Step 2: maxNumBlocks = ceil(min(numRows, numCols) / bw)  (HBDIA.cpp:537) */
    const int32_t nb = (int32_t)(((int64_t)(numRows < numCols ? numRows : numCols) + bw - 1) / bw);
    h->numBlocks = nb;

    /* Step 3: per-block offset counts (HBDIA.cpp:540-560).  Entries are
     * bucketed by block (stable), then each bucket's offsets are sorted and
     * run-length counted; this yields the same ascending (offset, count)
     * sequence as iterating the reference's std::map<int,int>. */
    int64_t *bcount = (int64_t *)calloc((size_t)nb + 1, sizeof(int64_t));
    for (int64_t i = 0; i < nnz; ++i) {
        int32_t b = rows[i] / bw;
        if (b < nb) bcount[b + 1]++;
    }
    for (int32_t b = 0; b < nb; ++b) bcount[b + 1] += bcount[b];
    int32_t *boffs = (int32_t *)malloc(sizeof(int32_t) * (size_t)(bcount[nb] > 0 ? bcount[nb] : 1));
    int64_t *fillp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nb > 0 ? nb : 1));
    for (int32_t b = 0; b < nb; ++b) fillp[b] = bcount[b];
    for (int64_t i = 0; i < nnz; ++i) {
        int32_t b = rows[i] / bw;
        if (b < nb) boffs[fillp[b]++] = cols[i] - rows[i] - rowBase;
    }
    free(fillp);
    /* distinct (offset,count) per block, in place: uniq[] holds offsets,
     * ucnt[] counts; ustart[b]..ustart[b+1] the block's run */
    int64_t *ustart = (int64_t *)calloc((size_t)nb + 1, sizeof(int64_t));
    int64_t *ucnt = (int64_t *)malloc(sizeof(int64_t) * (size_t)(bcount[nb] > 0 ? bcount[nb] : 1));
    int32_t *uniq = (int32_t *)malloc(sizeof(int32_t) * (size_t)(bcount[nb] > 0 ? bcount[nb] : 1));
    int64_t nu = 0;
    for (int32_t b = 0; b < nb; ++b) {
        int64_t s = bcount[b], e = bcount[b + 1];
        qsort(boffs + s, (size_t)(e - s), sizeof(int32_t), cmp_i32);
        ustart[b] = nu;
        for (int64_t i = s; i < e;) {
            int64_t j = i;
            while (j < e && boffs[j] == boffs[i]) ++j;
            uniq[nu] = boffs[i];
            ucnt[nu] = j - i;
            ++nu;
            i = j;
        }
    }
    ustart[nb] = nu;

    /* Step 4: filter, blocks in order, offsets ascending (HBDIA.cpp:567-586):
     * keep if count >= threshold or the running COO count already reached
     * max_coo_entries; otherwise the entries go to the COO remainder. */
    char *keep = (char *)malloc((size_t)(nu > 0 ? nu : 1));
    int64_t cpu_entries = 0;
    int64_t kept = 0;
    for (int32_t b = 0; b < nb; ++b) {
        for (int64_t u = ustart[b]; u < ustart[b + 1]; ++u) {
            if (ucnt[u] >= threshold || cpu_entries >= maxCoo) { keep[u] = 1; ++kept; }
            else { keep[u] = 0; cpu_entries += ucnt[u]; }
        }
    }
    /* numberDiagonals: distinct offsets over all blocks (HBDIA.cpp:563,585) */
    {
        int32_t *all = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nu > 0 ? nu : 1));
        memcpy(all, uniq, sizeof(int32_t) * (size_t)nu);
        qsort(all, (size_t)nu, sizeof(int32_t), cmp_i32);
        int32_t nd = 0;
        for (int64_t i = 0; i < nu; ++i) if (i == 0 || all[i] != all[i - 1]) ++nd;
        h->numberDiagonals = nd;
        free(all);
    }

    /* Step 5: storage (HBDIA.cpp:589-614) */
    h->totalOffsets = kept;
    h->slots = kept * bw;
    if ((double)h->slots > 1e11) {
        free(bcount); free(boffs); free(ustart); free(ucnt); free(uniq); free(keep);
        return -2;
    }
    h->offsets = (int32_t *)malloc(sizeof(int32_t) * (size_t)(kept > 0 ? kept : 1));
    h->blockStart = (int32_t *)malloc(sizeof(int32_t) * ((size_t)nb + 1));
    {
        int64_t p = 0;
        for (int32_t b = 0; b < nb; ++b) {
            h->blockStart[b] = (int32_t)p;
            for (int64_t u = ustart[b]; u < ustart[b + 1]; ++u)
                if (keep[u]) h->offsets[p++] = uniq[u];
        }
        h->blockStart[nb] = (int32_t)p;
    }
    /* Step 6: zero fill (HBDIA.cpp:617) */
    h->data = calloc((size_t)(h->slots > 0 ? h->slots : 1), esz);

    /* histograms (HBDIA.cpp:619-631) */
    int32_t maxd = 0;
    for (int32_t b = 0; b < nb; ++b) {
        int32_t k = h->blockStart[b + 1] - h->blockStart[b];
        if (k > maxd) maxd = k;
    }
    h->histLen = maxd + 1;
    h->histBlocks = (int32_t *)calloc((size_t)h->histLen, sizeof(int32_t));
    h->histNnz = (int32_t *)calloc((size_t)h->histLen, sizeof(int32_t));
    for (int32_t b = 0; b < nb; ++b) h->histBlocks[h->blockStart[b + 1] - h->blockStart[b]]++;

    /* Step 7: fill pass in input order (HBDIA.cpp:634-703).  A kept
     * (block, offset) slot is ASSIGNED, so duplicates are last-wins; every
     * other entry is appended to the COO remainder in input order and the
     * CSR row pointer is built assuming rows arrive non-decreasing. */
    h->cooRow = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    h->cooCol = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    h->cooVal = malloc(esz * (size_t)(nnz > 0 ? nnz : 1));
    h->cooRowPtr = (int32_t *)calloc((size_t)numRows + 1, sizeof(int32_t));
    int32_t currentRow = -1;
    int64_t nextOffset = 0;
    for (int64_t i = 0; i < nnz; ++i) {
        const int32_t r = rows[i], c = cols[i];
        const int32_t b = r / bw, off = c - r - rowBase, lane = r % bw;
        int64_t idx = -1;
        if (b < nb && h->blockStart[b + 1] > h->blockStart[b])
            idx = find_offset(h->offsets + h->blockStart[b],
                              h->blockStart[b + 1] - h->blockStart[b], off);
        if (idx >= 0) {
            int64_t slot = ((int64_t)h->blockStart[b] + idx) * bw + lane;
            memcpy((char *)h->data + slot * esz, (const char *)vals + i * esz, esz);
            h->histNnz[h->blockStart[b + 1] - h->blockStart[b]]++;
        } else {
            if (r != currentRow) {
                for (int32_t q = currentRow + 1; q <= r; ++q) h->cooRowPtr[q] = (int32_t)nextOffset;
                currentRow = r;
            }
            h->cooRow[nextOffset] = r;
            h->cooCol[nextOffset] = c;
            memcpy((char *)h->cooVal + nextOffset * esz, (const char *)vals + i * esz, esz);
            ++nextOffset;
        }
    }
    for (int32_t q = currentRow + 1; q <= numRows; ++q) h->cooRowPtr[q] = (int32_t)nextOffset;
    h->nCoo = nextOffset;
    h->has_hbdia = 1;

    free(bcount); free(boffs); free(ustart); free(ucnt); free(uniq); free(keep);
    return 0;
}

void orc_sizes(const orc_layout *h, int64_t *s) {
    s[0] = h->numBlocks; s[1] = h->totalOffsets; s[2] = h->slots; s[3] = h->nCoo;
    s[4] = h->numberDiagonals; s[5] = h->histLen; s[6] = h->has_hbdia;
    s[7] = h->numRows; s[8] = h->numCols; s[9] = h->has_hbdia ? (int64_t)h->numRows + 1 : 0;
}

void orc_export(const orc_layout *h, int32_t *offsets, int32_t *blockStart, void *data,
                int32_t *cooRow, int32_t *cooCol, void *cooVal, int32_t *cooRowPtr,
                int32_t *histBlocks, int32_t *histNnz) {
    if (!h->has_hbdia) return;
    const size_t esz = h->is_f32 ? sizeof(float) : sizeof(double);
    memcpy(offsets, h->offsets, sizeof(int32_t) * (size_t)h->totalOffsets);
    memcpy(blockStart, h->blockStart, sizeof(int32_t) * ((size_t)h->numBlocks + 1));
    memcpy(data, h->data, esz * (size_t)h->slots);
    memcpy(cooRow, h->cooRow, sizeof(int32_t) * (size_t)h->nCoo);
    memcpy(cooCol, h->cooCol, sizeof(int32_t) * (size_t)h->nCoo);
    memcpy(cooVal, h->cooVal, esz * (size_t)h->nCoo);
    memcpy(cooRowPtr, h->cooRowPtr, sizeof(int32_t) * ((size_t)h->numRows + 1));
    memcpy(histBlocks, h->histBlocks, sizeof(int32_t) * (size_t)h->histLen);
    memcpy(histNnz, h->histNnz, sizeof(int32_t) * (size_t)h->histLen);
}

void orc_destroy(orc_layout *h) {
    if (!h) return;
    free(h->offsets); free(h->blockStart); free(h->data);
    free(h->cooRow); free(h->cooCol); free(h->cooVal); free(h->cooRowPtr);
    free(h->histBlocks); free(h->histNnz);
    free(h);
}

/* Per-row COO sums in list order.  For row-sorted COO this is exactly what
 * cpu_coo_spmv_kernel computes (src/Operations/HBDIASpMV.cpp:76-92): start at
 * zero, `row_sum += val * x[col]` with a separate multiply and add. */
#define ORC_SPMV_BODY(T, FMA)                                                             \
    const int32_t n = h->numRows, bw = h->bw;                                             \
    const T *data = (const T *)h->data;                                                   \
    const T *cv = (const T *)h->cooVal;                                                   \
    T *coo = (T *)calloc((size_t)n + 1, sizeof(T));                                       \
    for (int64_t e = 0; e < h->nCoo; ++e) {                                               \
        T p = cv[e] * x[h->cooCol[e]];                                                    \
        coo[h->cooRow[e]] = coo[h->cooRow[e]] + p;                                        \
    }                                                                                     \
    for (int32_t row = 0; row < n; ++row) {                                               \
        /* src/Operations/HBDIASpMV.cu:22-71: ascending offsets, skip stored zeros and  \
         * columns outside [0, numRows), fused multiply-add (nvcc contracts          \
         * `sum += v * x`). */                                                        \
        T sum = (T)0;                                                                     \
        const int32_t b = row / bw, lane = row % bw;                                      \
        if (h->has_hbdia && b < h->numBlocks) {                                           \
            for (int32_t k = h->blockStart[b]; k < h->blockStart[b + 1]; ++k) {           \
                T v = data[(int64_t)k * bw + lane];                                       \
                if (v == (T)0) continue;                                                  \
                int64_t col = (int64_t)row + h->offsets[k];                               \
                if (col < 0 || col >= n) continue;                                        \
                sum = FMA(v, x[col], sum);                                                \
            }                                                                             \
        }                                                                                 \
        /* merge, src/Operations/HBDIASpMV.cu:77-88 (only when COO work exists,     \
         * src/Operations/HBDIASpMV.cpp:235-250) */                                    \
        y[row] = (h->nCoo > 0) ? (T)(sum + coo[row]) : sum;                               \
    }                                                                                     \
    free(coo);

void orc_spmv_f64(const orc_layout *h, const double *x, double *y) { ORC_SPMV_BODY(double, fma) }
void orc_spmv_f32(const orc_layout *h, const float *x, float *y) { ORC_SPMV_BODY(float, fmaf) }

/* The same double-precision SpMV with the blocked-DIA values replaced by
 * `values` (same layout): the expected result of reduced-precision value
 * storage, where each stored value is first rounded and then widened. */
void orc_spmv_f64_values(const orc_layout *h, const double *values, double *y, const double *x) {
    orc_layout g = *h;
    g.data = (void *)values;
    orc_spmv_f64(&g, x, y);
}

/* A partial matrix's rows of y = A x over the GLOBAL x: the blocked-DIA
 * column of local row r at offset o is rowBase + r + o, skipped outside
 * [0, numGlobalCols); COO columns are global.  The operation order is
 * orc_spmv_f64's (src/Operations/HBDIASpMV.cu:22-71, HBDIASpMV.cpp:76-92,
 * HBDIASpMV.cu:77-88) -- the reference's kernel itself reads x at
 * localRow + offset (HBDIASpMV.cu:53-58), so for partial matrices this is the
 * arithmetic its distributed SpMV intends rather than what that kernel
 * computes. */
void orc_spmv_partial_f64(const orc_layout *h, int32_t numGlobalCols, const double *x, double *y) {
    const int32_t n = h->numRows, bw = h->bw;
    const double *data = (const double *)h->data;
    const double *cv = (const double *)h->cooVal;
    double *coo = (double *)calloc((size_t)n + 1, sizeof(double));
    for (int64_t e = 0; e < h->nCoo; ++e) {
        double p = cv[e] * x[h->cooCol[e]];
        coo[h->cooRow[e]] = coo[h->cooRow[e]] + p;
    }
    for (int32_t row = 0; row < n; ++row) {
        double sum = 0.0;
        const int32_t b = row / bw, lane = row % bw;
        if (h->has_hbdia && b < h->numBlocks) {
            for (int32_t k = h->blockStart[b]; k < h->blockStart[b + 1]; ++k) {
                double v = data[(int64_t)k * bw + lane];
                if (v == 0.0) continue;
                int64_t col = (int64_t)h->rowBase + row + h->offsets[k];
                if (col < 0 || col >= numGlobalCols) continue;
                sum = fma(v, x[col], sum);
            }
        }
        y[row] = (h->nCoo > 0) ? sum + coo[row] : sum;
    }
    free(coo);
}

void orc_coo_spmv_f64(const int32_t *rows, const int32_t *cols, const double *vals,
                      int64_t nnz, const double *x, int32_t numRows, double *y) {
    /* single-thread instance of src/Operations/HBDIASpMV.cpp:36-99 */
    double row_sum = 0.0;
    int32_t current = -1;
    for (int64_t i = 0; i < nnz; ++i) {
        const int32_t r = rows[i];
        if (r != current) {
            if (current >= 0 && current < numRows) y[current] = row_sum;
            current = r;
            row_sum = 0.0;
        }
        row_sum += vals[i] * x[cols[i]];
    }
    if (current >= 0 && current < numRows) y[current] = row_sum;
}

/* ------------------------------------------------------------------------
 * Seeded benchmark workloads, restated so that bench.py's reference arm and
 * the tests can build the bench matrix without the product library.  This
 * follows the product's own generator (hbdia_b200/csrc/generate.cpp,
 * generate_stencil / fill_uniform), which tests/test_oracle.py pins entry for
 * entry: MT19937-64 (Matsumoto & Nishimura's published generator, the one
 * std::mt19937_64 implements), a draw in [0, n) as the high 64 bits of
 * draw * n, a draw in [0, 1) as the top 53 bits times 2^-53. */
typedef struct {
    uint64_t mt[312];
    int idx;
} orc_mt64;

static void mt64_seed(orc_mt64 *g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = 312;
}

static uint64_t mt64_next(orc_mt64 *g) {
    if (g->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t v = (g->mt[i] & 0xFFFFFFFF80000000ULL) | (g->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t va = v >> 1;
            if (v & 1) va ^= 0xB5026F5AA96619E9ULL;
            g->mt[i] = g->mt[(i + 156) % 312] ^ va;
        }
        g->idx = 0;
    }
    uint64_t y = g->mt[g->idx++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

static uint64_t mt64_bounded(orc_mt64 *g, uint64_t n) {
    return (uint64_t)(((unsigned __int128)mt64_next(g) * n) >> 64);
}

static double mt64_unit(orc_mt64 *g) { return (double)(mt64_next(g) >> 11) * 0x1.0p-53; }

void orc_fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed) {
    orc_mt64 g;
    mt64_seed(&g, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * mt64_unit(&g);
}

static int64_t iabs64(int64_t v) { return v < 0 ? -v : v; }

int orc_workload_stencil27(int32_t nx, int32_t ny, int32_t nz, double center, double neighbor, double frac,
                           double lo, double hi, uint64_t seed, int64_t *nnzOut, int32_t *rows, int32_t *cols,
                           double *vals) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !nnzOut) return -1;
    const int64_t n = (int64_t)nx * ny * nz;
    if (n > 2147483647LL) return -1;
    const int64_t stencilNnz = (3LL * nx - 2) * (3LL * ny - 2) * (3LL * nz - 2);
    const int64_t nExtra = (int64_t)floor(frac * (double)stencilNnz);
    *nnzOut = stencilNnz + nExtra;
    if (!rows) return 0;
    /* extras: rows, columns, values in draw order, outside the stencil and
     * without repeats */
    int32_t *er = NULL, *ec = NULL;
    double *ev = NULL;
    uint64_t *set = NULL;
    int64_t cap = 16;
    if (nExtra > 0) {
        er = (int32_t *)malloc((size_t)nExtra * sizeof(int32_t));
        ec = (int32_t *)malloc((size_t)nExtra * sizeof(int32_t));
        ev = (double *)malloc((size_t)nExtra * sizeof(double));
        while (cap < 2 * nExtra + 16) cap <<= 1;
        set = (uint64_t *)calloc((size_t)cap, sizeof(uint64_t));
        if (!er || !ec || !ev || !set) {
            free(er), free(ec), free(ev), free(set);
            return -1;
        }
        orc_mt64 g;
        mt64_seed(&g, seed);
        for (int64_t t = 0; t < nExtra; ++t) {
            int64_t r, c;
            for (;;) {
                r = (int64_t)mt64_bounded(&g, (uint64_t)n);
                c = (int64_t)mt64_bounded(&g, (uint64_t)n);
                const int64_t dx = iabs64(c % nx - r % nx), dy = iabs64((c / nx) % ny - (r / nx) % ny),
                              dz = iabs64(c / ((int64_t)nx * ny) - r / ((int64_t)nx * ny));
                if (dx <= 1 && dy <= 1 && dz <= 1) continue; /* inside the stencil */
                const uint64_t key = (uint64_t)r * (uint64_t)n + (uint64_t)c + 1u;
                uint64_t h = key * 0x9E3779B97F4A7C15ULL;
                int64_t slot = (int64_t)(h >> 20) & (cap - 1);
                int dup = 0;
                while (set[slot]) {
                    if (set[slot] == key) {
                        dup = 1;
                        break;
                    }
                    slot = (slot + 1) & (cap - 1);
                }
                if (dup) continue;
                set[slot] = key;
                break;
            }
            er[t] = (int32_t)r;
            ec[t] = (int32_t)c;
            ev[t] = lo + (hi - lo) * mt64_unit(&g);
        }
        free(set);
    }
    /* extras grouped by row, draw order kept */
    int64_t *xstart = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *order = nExtra > 0 ? (int64_t *)malloc((size_t)nExtra * sizeof(int64_t)) : NULL;
    if (!xstart || (nExtra > 0 && !order)) {
        free(xstart), free(order), free(er), free(ec), free(ev);
        return -1;
    }
    for (int64_t t = 0; t < nExtra; ++t) xstart[er[t] + 1]++;
    for (int64_t r = 0; r < n; ++r) xstart[r + 1] += xstart[r];
    {
        int64_t *fill = (int64_t *)malloc((size_t)n * sizeof(int64_t));
        if (!fill) {
            free(xstart), free(order), free(er), free(ec), free(ev);
            return -1;
        }
        memcpy(fill, xstart, (size_t)n * sizeof(int64_t));
        for (int64_t t = 0; t < nExtra; ++t) order[fill[er[t]]++] = t;
        free(fill);
    }
    /* rows in order: the stencil entries (z, y, x neighbours ascending), then
     * the row's extras */
    const int64_t plane = (int64_t)nx * ny;
    int64_t p = 0;
    for (int64_t r = 0; r < n; ++r) {
        const int64_t x = r % nx, y = (r / nx) % ny, z = r / plane;
        for (int dz = -1; dz <= 1; ++dz) {
            if (z + dz < 0 || z + dz >= nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                if (y + dy < 0 || y + dy >= ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    if (x + dx < 0 || x + dx >= nx) continue;
                    rows[p] = (int32_t)r;
                    cols[p] = (int32_t)(r + dz * plane + dy * nx + dx);
                    vals[p] = (dx == 0 && dy == 0 && dz == 0) ? center : neighbor;
                    ++p;
                }
            }
        }
        for (int64_t q = xstart[r]; q < xstart[r + 1]; ++q) {
            const int64_t t = order[q];
            rows[p] = er[t];
            cols[p] = ec[t];
            vals[p] = ev[t];
            ++p;
        }
    }
    free(xstart), free(order), free(er), free(ec), free(ev);
    return 0;
}
