// Matrix sources: the reference's own stencil generator and Matrix Market
// loader (drop-in, identical output), and this library's seeded synthetic
// workloads (27-point / 7-point stencils with extra entries, banded matrices).

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <numeric>
#include <random>
#include <set>
#include <sstream>
#include <unordered_set>

#include "hbdia_internal.hpp"

namespace hbdia {

// ---------------------------------------------------------------------------
// create3DStencil27Point(nx, ny, nz, noise, iteration)
// (src/Format/HBDIA.cpp:1416-1607).  For the output to be identical this
// follows the reference's visiting order, its std::mt19937 draw sequence
// (seed 42 + iteration, noise rows first, then per row column/value draws) and
// its final std::sort of an index permutation by row (not stable, so the
// same sort call is needed to get the same order of entries within a row).
// The reference loops the coordinate it multiplies by 1 up to nz and the one
// it multiplies by nx*ny up to nx, so its indices stay inside the matrix only
// when nx == nz (otherwise it writes past nnzPerRow); that case is rejected.
template <typename T>
void reference_stencil27(int nx, int ny, int nz, double noise, int iteration, Coo<T> &out) {
    if (nx != nz)
        throw Error(HBDIA_ERR_UNSUPPORTED,
                    "create3DStencil27Point indexes outside the matrix unless nx == nz");
    const int total = nx * ny * nz;
    std::vector<int> &rows = out.rows;
    std::vector<int> &cols = out.cols;
    std::vector<T> &vals = out.vals;
    rows.clear();
    cols.clear();
    vals.clear();
    out.nnzPerRow.assign(static_cast<size_t>(total), 0);
    auto index = [&](int a, int b, int c) { return c * nx * ny + b * nx + a; };

    std::mt19937 gen(42 + iteration);
    std::uniform_int_distribution<int> colDist(0, total - 1);
    std::uniform_real_distribution<double> valueDist(-1.0, 1.0);
    std::vector<int> noiseInRow(static_cast<size_t>(total), 0);
    if (noise > 0.0) {
        const long long stencilEntries = total * 27;
        const int target = static_cast<int>(static_cast<double>(stencilEntries) * noise);
        std::uniform_int_distribution<int> rowDist(0, total - 1);
        for (int t = 0; t < target; ++t) noiseInRow[rowDist(gen)]++;
    }

    for (int a = 0; a < nz; a++) {
        for (int b = 0; b < ny; b++) {
            for (int c = 0; c < nx; c++) {
                const int centre = index(a, b, c);
                for (int da = -1; da <= 1; da++)
                    for (int db = -1; db <= 1; db++)
                        for (int dc = -1; dc <= 1; dc++) {
                            const int na = a + da, nb = b + db, nc = c + dc;
                            if (na < 0 || na >= nx || nb < 0 || nb >= ny || nc < 0 || nc >= nz) continue;
                            rows.push_back(centre);
                            cols.push_back(index(na, nb, nc));
                            out.nnzPerRow[centre]++;
                            const int moved = (da != 0) + (db != 0) + (dc != 0);
                            vals.push_back(moved == 0 ? static_cast<T>(26.1)
                                           : moved == 1 ? static_cast<T>(-1.1)
                                           : moved == 2 ? static_cast<T>(-0.1)
                                                        : static_cast<T>(-0.01));
                        }
                const int want = noiseInRow[centre];
                if (want > 0) {
                    std::set<int> used;
                    for (int dc = -1; dc <= 1; dc++)
                        for (int db = -1; db <= 1; db++)
                            for (int da = -1; da <= 1; da++) {
                                const int na = a + da, nb = b + db, nc = c + dc;
                                if (na >= 0 && na < nx && nb >= 0 && nb < ny && nc >= 0 && nc < nz)
                                    used.insert(index(na, nb, nc));
                            }
                    int added = 0, attempts = 0;
                    const int maxAttempts = want * 10 + 100;
                    while (added < want && attempts < maxAttempts) {
                        attempts++;
                        const int col = colDist(gen);
                        if (used.find(col) != used.end()) continue;
                        used.insert(col);
                        rows.push_back(centre);
                        cols.push_back(col);
                        vals.push_back(static_cast<T>(valueDist(gen)));
                        added++;
                        out.nnzPerRow[centre]++;
                    }
                }
            }
        }
    }

    std::vector<size_t> perm(rows.size());
    std::iota(perm.begin(), perm.end(), 0);
    std::sort(perm.begin(), perm.end(), [&](size_t p, size_t q) { return rows[p] < rows[q]; });
    std::vector<int> r2(rows.size()), c2(cols.size());
    std::vector<T> v2(vals.size());
    for (size_t e = 0; e < perm.size(); e++) {
        r2[e] = rows[perm[e]];
        c2[e] = cols[perm[e]];
        v2[e] = vals[perm[e]];
    }
    rows.swap(r2);
    cols.swap(c2);
    vals.swap(v2);
    out.numRows = total;
    out.numCols = total;
}

// ---------------------------------------------------------------------------
// loadMTX(filename) (src/Format/HBDIA.cpp:161-263) when numRows, numCols <= 0,
// else loadMTX(filename, numRows, numCols) (src/Format/HBDIA.cpp:265-370).
// Same parsing rules: '%' lines before the size line, "symmetric" anywhere in
// them mirrors off-diagonal entries, missing values read as 1, at most the
// declared number of entries.  The first form sorts by (row, col) through the
// same std::sort call on an index permutation; the second validates indices
// against the given dimensions (std::out_of_range) and does not sort.
template <typename T>
bool load_mtx(const std::string &path, int numRowsArg, int numColsArg, Coo<T> &out) {
    const bool sized = numRowsArg > 0 || numColsArg > 0;
    if (sized && (numRowsArg <= 0 || numColsArg <= 0)) return false;
    std::ifstream file(path);
    if (!file.is_open()) return false;
    std::string line;
    bool symmetric = false;
    while (std::getline(file, line)) {
        if (!line.empty() && line[0] == '%') {
            if (line.find("symmetric") != std::string::npos) symmetric = true;
        } else {
            break;
        }
    }
    int fileRows = 0, fileCols = 0, fileNnz = 0;
    {
        std::istringstream hs(line);
        hs >> fileRows >> fileCols >> fileNnz;
    }
    out.rows.clear();
    out.cols.clear();
    out.vals.clear();
    out.nnzPerRow.clear();
    out.numRows = sized ? numRowsArg : fileRows;
    out.numCols = sized ? numColsArg : fileCols;
    int original = 0;
    while (original < fileNnz && std::getline(file, line)) {
        std::istringstream es(line);
        int r, c;
        T v;
        if (!(es >> r >> c)) continue;
        if (!(es >> v)) v = T(1);
        r -= 1;
        c -= 1;
        if (sized) {
            if (r < 0 || r >= out.numRows)
                throw Error(HBDIA_ERR_OUT_OF_RANGE, "Row index " + std::to_string(r) +
                                                         " from file is out of range [0, " +
                                                         std::to_string(out.numRows - 1) + "]");
            if (c < 0 || c >= out.numCols)
                throw Error(HBDIA_ERR_OUT_OF_RANGE, "Column index " + std::to_string(c) +
                                                         " from file is out of range [0, " +
                                                         std::to_string(out.numCols - 1) + "]");
        }
        out.rows.push_back(r);
        out.cols.push_back(c);
        out.vals.push_back(v);
        original++;
        if (symmetric && r != c) {
            out.rows.push_back(c);
            out.cols.push_back(r);
            out.vals.push_back(v);
        }
    }
    if (!sized) {
        const size_t n = out.vals.size();
        std::vector<size_t> idx(n);
        for (size_t i = 0; i < n; ++i) idx[i] = i;
        const auto &R = out.rows;
        const auto &C = out.cols;
        std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
            if (R[a] != R[b]) return R[a] < R[b];
            return C[a] < C[b];
        });
        std::vector<int> r2(n), c2(n);
        std::vector<T> v2(n);
        for (size_t i = 0; i < n; ++i) {
            r2[i] = R[idx[i]];
            c2[i] = C[idx[i]];
            v2[i] = out.vals[idx[i]];
        }
        out.rows.swap(r2);
        out.cols.swap(c2);
        out.vals.swap(v2);
    }
    return original > 0;
}

template void reference_stencil27<double>(int, int, int, double, int, Coo<double> &);
template void reference_stencil27<float>(int, int, int, double, int, Coo<float> &);
template bool load_mtx<double>(const std::string &, int, int, Coo<double> &);
template bool load_mtx<float>(const std::string &, int, int, Coo<float> &);

// ---------------------------------------------------------------------------
// Seeded synthetic workloads (this library's own definitions).
namespace {

inline uint64_t bounded(std::mt19937_64 &g, uint64_t n) {
    return static_cast<uint64_t>((static_cast<unsigned __int128>(g()) * n) >> 64);
}
inline double unit(std::mt19937_64 &g) { return static_cast<double>(g() >> 11) * 0x1.0p-53; }

struct Extra {
    int32_t row, col;
    double val;
};

// Extras drawn outside a pattern, without repeats, in draw order.
template <typename InPattern>
std::vector<Extra> draw_extras(int64_t count, int64_t n, double lo, double hi, uint64_t seed,
                               InPattern inPattern) {
    std::vector<Extra> ex;
    ex.reserve(static_cast<size_t>(count));
    std::mt19937_64 g(seed);
    std::unordered_set<uint64_t> seen;
    seen.reserve(static_cast<size_t>(count) * 2 + 16);
    for (int64_t t = 0; t < count; ++t) {
        int64_t r, c;
        for (;;) {
            r = static_cast<int64_t>(bounded(g, static_cast<uint64_t>(n)));
            c = static_cast<int64_t>(bounded(g, static_cast<uint64_t>(n)));
            if (inPattern(r, c)) continue;
            if (!seen.insert(static_cast<uint64_t>(r) * static_cast<uint64_t>(n) + c).second) continue;
            break;
        }
        ex.push_back(Extra{static_cast<int32_t>(r), static_cast<int32_t>(c), lo + (hi - lo) * unit(g)});
    }
    return ex;
}

// extras grouped by row, draw order kept: (start per row, permutation)
void group_by_row(const std::vector<Extra> &ex, int64_t n, std::vector<int64_t> &start,
                  std::vector<int32_t> &order) {
    start.assign(static_cast<size_t>(n) + 1, 0);
    for (const Extra &e : ex) start[static_cast<size_t>(e.row) + 1]++;
    for (int64_t r = 0; r < n; ++r) start[r + 1] += start[r];
    order.resize(ex.size());
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (size_t i = 0; i < ex.size(); ++i) order[fill[ex[i].row]++] = static_cast<int32_t>(i);
}

// one cached draw, so the two-call protocol draws once
std::mutex g_cache_mu;
std::string g_cache_key;
std::vector<Extra> g_cache_extras;

template <typename Draw>
std::vector<Extra> cached_extras(const std::string &key, Draw draw) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (key != g_cache_key) {
        g_cache_extras = draw();
        g_cache_key = key;
    }
    return g_cache_extras;
}

}  // namespace

int generate_stencil(int stencilPoints, int32_t nx, int32_t ny, int32_t nz, double center,
                     double neighbor, double frac, double lo, double hi, uint64_t seed,
                     int64_t *nnzOut, int32_t *rows, int32_t *cols, double *vals) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !nnzOut)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "grid dimensions must be positive");
    const int64_t n = static_cast<int64_t>(nx) * ny * nz;
    if (n > 2147483647LL) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "grid too large for int32 indices");
    const bool full = stencilPoints == 27;
    auto coords = [&](int64_t r, int64_t &x, int64_t &y, int64_t &z) {
        x = r % nx;
        y = (r / nx) % ny;
        z = r / (static_cast<int64_t>(nx) * ny);
    };
    auto inPattern = [&](int64_t r, int64_t c) {
        int64_t x0, y0, z0, x1, y1, z1;
        coords(r, x0, y0, z0);
        coords(c, x1, y1, z1);
        const int64_t dx = std::llabs(x1 - x0), dy = std::llabs(y1 - y0), dz = std::llabs(z1 - z0);
        if (full) return dx <= 1 && dy <= 1 && dz <= 1;
        return dx + dy + dz <= 1;
    };
    const int64_t stencilNnz = full ? (3LL * nx - 2) * (3LL * ny - 2) * (3LL * nz - 2)
                                    : n + 2LL * ((nx - 1LL) * ny * nz + nx * (ny - 1LL) * nz +
                                                 static_cast<int64_t>(nx) * ny * (nz - 1LL));
    const int64_t nExtra = full ? static_cast<int64_t>(std::floor(frac * static_cast<double>(stencilNnz))) : 0;
    std::vector<Extra> ex;
    if (nExtra > 0) {
        std::ostringstream key;
        key << "s27/" << nx << "/" << ny << "/" << nz << "/" << frac << "/" << lo << "/" << hi << "/" << seed;
        ex = cached_extras(key.str(), [&] { return draw_extras(nExtra, n, lo, hi, seed, inPattern); });
    }
    *nnzOut = stencilNnz + nExtra;
    if (!rows) return HBDIA_OK;
    std::vector<int64_t> xstart;
    std::vector<int32_t> xorder;
    group_by_row(ex, n, xstart, xorder);
    // row starts: stencil count per row + extras per row
    auto span = [](int64_t c, int64_t len) { return 1 + (c > 0) + (c < len - 1); };
    std::vector<int64_t> rstart(static_cast<size_t>(n) + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int64_t x, y, z;
        coords(r, x, y, z);
        const int64_t sx = span(x, nx), sy = span(y, ny), sz = span(z, nz);
        const int64_t s = full ? sx * sy * sz : 1 + (sx - 1) + (sy - 1) + (sz - 1);
        rstart[r + 1] = s + (xstart[r + 1] - xstart[r]);
    }
    for (int64_t r = 0; r < n; ++r) rstart[r + 1] += rstart[r];
    const int64_t plane = static_cast<int64_t>(nx) * ny;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int64_t x, y, z;
        coords(r, x, y, z);
        int64_t p = rstart[r];
        for (int dz = -1; dz <= 1; ++dz) {
            if (z + dz < 0 || z + dz >= nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                if (y + dy < 0 || y + dy >= ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    if (x + dx < 0 || x + dx >= nx) continue;
                    const int moved = (dx != 0) + (dy != 0) + (dz != 0);
                    if (!full && moved > 1) continue;
                    rows[p] = static_cast<int32_t>(r);
                    cols[p] = static_cast<int32_t>(r + dz * plane + dy * nx + dx);
                    vals[p] = moved == 0 ? center : neighbor;
                    ++p;
                }
            }
        }
        for (int64_t q = xstart[r]; q < xstart[r + 1]; ++q) {
            const Extra &e = ex[xorder[q]];
            rows[p] = e.row;
            cols[p] = e.col;
            vals[p] = e.val;
            ++p;
        }
    }
    return HBDIA_OK;
}

int generate_banded(int32_t n, const int32_t *offs, int32_t noffs, double lo, double hi, double drop,
                    double scatter, uint64_t seed, int64_t *nnzOut, int32_t *rows, int32_t *cols,
                    double *vals) {
    if (n <= 0 || noffs <= 0 || !offs || !nnzOut)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad banded-matrix arguments");
    std::vector<int32_t> o(offs, offs + noffs);
    std::sort(o.begin(), o.end());
    o.erase(std::unique(o.begin(), o.end()), o.end());
    const bool hasCentre = std::binary_search(o.begin(), o.end(), 0);
    // band values: one draw per (row, offset) position inside the matrix, row by
    // row, offsets ascending: keep-draw then value-draw.
    std::mt19937_64 g(seed);
    std::vector<int64_t> rstart(static_cast<size_t>(n) + 1, 0);
    std::vector<std::pair<int32_t, double>> band;  // (col, value); centre gets its value later
    band.reserve(static_cast<size_t>(n) * o.size());
    std::vector<int64_t> centrePos(static_cast<size_t>(n), -1);
    for (int64_t r = 0; r < n; ++r) {
        double absSum = 0.0;
        for (int32_t off : o) {
            const int64_t c = r + off;
            if (c < 0 || c >= n) continue;
            if (off == 0) {
                centrePos[r] = static_cast<int64_t>(band.size());
                band.emplace_back(static_cast<int32_t>(c), 0.0);
                continue;
            }
            const bool keep = unit(g) >= drop;
            const double v = lo + (hi - lo) * unit(g);
            if (!keep) continue;
            band.emplace_back(static_cast<int32_t>(c), v);
            absSum += std::fabs(v);
        }
        if (centrePos[r] >= 0) band[centrePos[r]].second = absSum + 1.0;
        rstart[r + 1] = static_cast<int64_t>(band.size());
    }
    (void)hasCentre;
    const int64_t nExtra = static_cast<int64_t>(std::floor(scatter * static_cast<double>(band.size())));
    std::ostringstream key;
    key << "band/" << n << "/" << noffs << "/" << o.front() << "/" << o.back() << "/" << lo << "/" << hi
        << "/" << drop << "/" << scatter << "/" << seed;
    auto inPattern = [&](int64_t r, int64_t c) { return std::binary_search(o.begin(), o.end(), static_cast<int32_t>(c - r)); };
    std::vector<Extra> ex = nExtra > 0 ? cached_extras(key.str(), [&] {
        return draw_extras(nExtra, n, lo, hi, seed ^ 0x9e3779b97f4a7c15ULL, inPattern);
    }) : std::vector<Extra>();
    *nnzOut = static_cast<int64_t>(band.size()) + nExtra;
    if (!rows) return HBDIA_OK;
    std::vector<int64_t> xstart;
    std::vector<int32_t> xorder;
    group_by_row(ex, n, xstart, xorder);
    int64_t p = 0;
    for (int64_t r = 0; r < n; ++r) {
        for (int64_t q = rstart[r]; q < rstart[r + 1]; ++q) {
            rows[p] = static_cast<int32_t>(r);
            cols[p] = band[q].first;
            vals[p] = band[q].second;
            ++p;
        }
        for (int64_t q = xstart[r]; q < xstart[r + 1]; ++q) {
            const Extra &e = ex[xorder[q]];
            rows[p] = e.row;
            cols[p] = e.col;
            vals[p] = e.val;
            ++p;
        }
    }
    return HBDIA_OK;
}

namespace {
inline uint64_t splitmix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
}  // namespace

int generate_stencil27_spd(int32_t nx, int32_t ny, int32_t nz, double shift, double extraFraction, uint64_t seed,
                           int64_t *nnzOut, int32_t *rows, int32_t *cols, double *vals) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !nnzOut || shift < 0 || extraFraction < 0 || extraFraction > 1)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "bad SPD stencil arguments");
    const int64_t n = static_cast<int64_t>(nx) * ny * nz;
    if (n > 2147483647LL) throw Error(HBDIA_ERR_INVALID_ARGUMENT, "grid too large for int32 indices");
    const int64_t stencilNnz = (3LL * nx - 2) * (3LL * ny - 2) * (3LL * nz - 2);
    const int64_t plane = static_cast<int64_t>(nx) * ny;
    // Symmetric off-pattern pairs (i < j, j outside i's 27-point neighbourhood,
    // no pair twice): floor(extraFraction * stencil nnz / 2) of them, each
    // stored as (i, j) and (j, i), drawn from a splitmix sequence of the seed.
    const int64_t pairs = static_cast<int64_t>(std::floor(extraFraction * static_cast<double>(stencilNnz) / 2.0));
    // unordered pairs outside the pattern: all pairs minus the stencil's off-diagonal ones
    const int64_t farPairs = n * (n - 1) / 2 - (stencilNnz - n) / 2;
    if (pairs > farPairs / 2)
        throw Error(HBDIA_ERR_INVALID_ARGUMENT, "grid too small for that many off-pattern entries");
    std::vector<std::pair<int32_t, int32_t>> extra;
    extra.reserve(static_cast<size_t>(pairs));
    {
        std::unordered_set<uint64_t> seen;
        uint64_t state = seed ^ 0x5bd1e9955bd1e995ULL;
        auto near = [&](int64_t a, int64_t b) {
            const int64_t ax = a % nx, ay = (a / nx) % ny, az = a / plane;
            const int64_t bx = b % nx, by = (b / nx) % ny, bz = b / plane;
            return std::llabs(ax - bx) <= 1 && std::llabs(ay - by) <= 1 && std::llabs(az - bz) <= 1;
        };
        while (static_cast<int64_t>(extra.size()) < pairs) {
            state = splitmix(state);
            int64_t a = static_cast<int64_t>(state % static_cast<uint64_t>(n));
            state = splitmix(state);
            int64_t b = static_cast<int64_t>(state % static_cast<uint64_t>(n));
            if (a == b || near(a, b)) continue;
            if (a > b) std::swap(a, b);
            if (!seen.insert(static_cast<uint64_t>(a) * static_cast<uint64_t>(n) + static_cast<uint64_t>(b)).second)
                continue;
            extra.emplace_back(static_cast<int32_t>(a), static_cast<int32_t>(b));
        }
    }
    *nnzOut = stencilNnz + 2 * pairs;
    if (!rows) return HBDIA_OK;
    // per-row extra columns, ascending
    std::vector<int64_t> xstart(static_cast<size_t>(n) + 1, 0);
    for (const auto &e : extra) {
        ++xstart[e.first + 1];
        ++xstart[e.second + 1];
    }
    for (int64_t r = 0; r < n; ++r) xstart[r + 1] += xstart[r];
    std::vector<int32_t> xcol(static_cast<size_t>(2 * pairs));
    {
        std::vector<int64_t> fill(xstart.begin(), xstart.end() - 1);
        for (const auto &e : extra) {
            xcol[fill[e.first]++] = e.second;
            xcol[fill[e.second]++] = e.first;
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) std::sort(xcol.begin() + xstart[r], xcol.begin() + xstart[r + 1]);
    auto span = [](int64_t c, int64_t len) { return 1 + (c > 0) + (c < len - 1); };
    std::vector<int64_t> rstart(static_cast<size_t>(n) + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r)
        rstart[r + 1] = span(r % nx, nx) * span((r / nx) % ny, ny) * span(r / plane, nz) + (xstart[r + 1] - xstart[r]);
    for (int64_t r = 0; r < n; ++r) rstart[r + 1] += rstart[r];
    // symmetric weights: -(0.5 + u), u from a hash of the unordered pair
    auto weight = [&](int64_t i, int64_t j) {
        const int64_t a = std::min(i, j), b = std::max(i, j);
        const uint64_t h = splitmix(static_cast<uint64_t>(a) * 0x100000001b3ULL ^ static_cast<uint64_t>(b) ^ seed);
        return -(0.5 + static_cast<double>(h >> 11) * 0x1.0p-53);
    };
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        const int64_t x = r % nx, y = (r / nx) % ny, z = r / plane;
        int64_t p = rstart[r], diagPos = -1;
        int64_t xe = xstart[r];
        const int64_t xend = xstart[r + 1];
        double absSum = 0.0;
        auto put = [&](int64_t c) {
            rows[p] = static_cast<int32_t>(r);
            cols[p] = static_cast<int32_t>(c);
            if (c == r) {
                diagPos = p;
                vals[p] = 0.0;
            } else {
                vals[p] = weight(r, c);
                absSum += -vals[p];
            }
            ++p;
        };
        for (int dz = -1; dz <= 1; ++dz) {
            if (z + dz < 0 || z + dz >= nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                if (y + dy < 0 || y + dy >= ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    if (x + dx < 0 || x + dx >= nx) continue;
                    const int64_t c = r + dz * plane + dy * nx + dx;
                    while (xe < xend && xcol[xe] < c) put(xcol[xe++]);  // keep columns ascending
                    put(c);
                }
            }
        }
        while (xe < xend) put(xcol[xe++]);
        vals[diagPos] = (1.0 + shift) * absSum;
    }
    return HBDIA_OK;
}

void fill_uniform(double *out, int64_t n, double lo, double hi, uint64_t seed) {
    std::mt19937_64 g(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * unit(g);
}

}  // namespace hbdia
