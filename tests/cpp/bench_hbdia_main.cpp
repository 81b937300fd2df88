// Driver for the reference's benchHBDIA() (benchmarking/benchHBDIA.cpp),
// which is compiled unchanged against include/hbdia/ by oracle/Makefile's
// `dropin` target and linked with this file and libhbdia_b200.so.
//
// It runs benchHBDIA twice on the 27-point stencil with 1 % noise (32^3,
// blockWidth 32, threshold 2, x_i = i + 1): once with device vectors and the
// GPU COO flag, once with the unified-memory flags and the CPU COO flag (both
// accepted by the drop-in).  Each y is checked bit for bit against the
// reference's arithmetic applied to the layout getters, and the first y is
// written to argv[1] (raw doubles) for the oracle comparison in Python.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/hbdia/Format/HBDIA.hpp"
#include "../../include/hbdia/Format/HBDIAVector.hpp"

using DataType = double;
void benchHBDIA(HBDIA<DataType> &matrix, const std::vector<DataType> &inputVector,
                std::vector<DataType> &outputVector, bool execCOOCPU, bool execCOOGPU,
                std::vector<double> &measurements, bool unifiedMemory, bool unifiedMemory_malloc,
                bool unifiedMemory_managedMalloc, bool unifiedMemory_NumaAllocOnNode);

// y = DIA part (ascending offsets, fma, stored zeros and outside columns
// skipped) + COO part (list order, product rounded before the add)
static std::vector<double> expected(const HBDIA<double> &m, const std::vector<double> &x) {
    const int n = m.getNumRows(), bw = m.getBlockWidth();
    const auto &opb = m.getOffsetsPerBlock();
    const auto &data = m.getHBDIAData();
    const auto &cr = m.getCpuRowIndices();
    const auto &cc = m.getCpuColIndices();
    const auto &cv = m.getCpuValues();
    std::vector<double> y(n, 0.0), coo(n, 0.0);
    for (size_t e = 0; e < cr.size(); ++e) {
        volatile double p = cv[e] * x[cc[e]];
        coo[cr[e]] = coo[cr[e]] + p;
    }
    size_t base = 0;
    for (size_t b = 0; b < opb.size(); ++b) {
        for (int lane = 0; lane < bw; ++lane) {
            const int row = static_cast<int>(b) * bw + lane;
            if (row >= n) break;
            double s = 0.0;
            for (size_t k = 0; k < opb[b].size(); ++k) {
                const double v = data[(base + k) * bw + lane];
                const long col = static_cast<long>(row) + opb[b][k];
                if (v == 0.0 || col < 0 || col >= n) continue;
                s = std::fma(v, x[col], s);
            }
            y[row] = s;
        }
        base += opb[b].size();
    }
    if (!cr.empty())
        for (int r = 0; r < n; ++r) y[r] = y[r] + coo[r];
    return y;
}

int main(int argc, char **argv) {
    HBDIA<double> m;
    m.create3DStencil27Point(32, 32, 32, 0.01, 0);
    m.convertToHBDIAFormat(32, 2);
    std::vector<double> x(m.getNumRows());
    for (int i = 0; i < m.getNumRows(); ++i) x[i] = static_cast<double>(i + 1);
    const std::vector<double> want = expected(m, x);
    int failures = 0;
    for (int pass = 0; pass < 2; ++pass) {
        std::vector<double> y, ms;
        const bool um = pass == 1;
        benchHBDIA(m, x, y, /*execCOOCPU=*/um, /*execCOOGPU=*/!um, ms, um, um, false, false);
        bool same = y.size() == want.size() && ms.size() == static_cast<size_t>(NUM_BENCH_ITER);
        for (size_t i = 0; same && i < y.size(); ++i) same = y[i] == want[i];
        double best = 1e30;
        for (double t : ms) best = t < best ? t : best;
        std::printf("%s: benchHBDIA pass %d (%s), %zu timings, best %.4f ms, y bit-exact: %s\n", same ? "ok" : "FAIL",
                    pass, um ? "unified-memory flags, CPU COO flag" : "device vectors, GPU COO flag", ms.size(), best,
                    same ? "yes" : "no");
        failures += same ? 0 : 1;
        if (pass == 0 && argc > 1) {
            FILE *f = std::fopen(argv[1], "wb");
            if (!f || std::fwrite(y.data(), sizeof(double), y.size(), f) != y.size()) ++failures;
            if (f) std::fclose(f);
        }
    }
    std::printf(failures ? "FAILED (%d)\n" : "ALL PASSED\n", failures);
    return failures ? 1 : 0;
}
