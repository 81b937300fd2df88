// C++ drop-in check: the reference's single-GPU usage
// (simple_hbdia_example.cpp:15-33) and the shape of its cuSPARSE comparison
// test (tests/run_HBDIA_cusparse_comparison.cpp:128-250), written against
// include/hbdia/, plus the GPU getters, the DIA format, duplicate removal,
// the unified-memory vector constructor, the COO result buffer and
// CHECK_CUDA.  The expected y is computed here from the layout getters with
// the reference's arithmetic (ascending-offset FMA chain for the blocked-DIA
// part, sequential multiply-then-add for the COO remainder), so the
// comparison is exact.  Exit status 0 only if every check passes.
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "hbdia/Format/HBDIA.hpp"
#include "hbdia/Format/HBDIAVector.hpp"
#include "hbdia/Operations/HBDIASpMV.hpp"

static int failures = 0;
#define CHECK(cond, what)                                   \
    do {                                                    \
        if (!(cond)) {                                      \
            std::printf("FAIL: %s\n", what);                \
            ++failures;                                     \
        } else {                                            \
            std::printf("ok:   %s\n", what);                \
        }                                                   \
    } while (0)

template <typename T>
static std::vector<T> expected(const HBDIA<T> &m, const std::vector<T> &x) {
    const int n = m.getNumRows(), bw = m.getBlockWidth();
    const auto &opb = m.getOffsetsPerBlock();
    const auto &data = m.getHBDIAData();
    std::vector<T> y(n, T(0)), coo(n, T(0));
    const auto &cr = m.getCpuRowIndices();
    const auto &cc = m.getCpuColIndices();
    const auto &cv = m.getCpuValues();
    for (size_t e = 0; e < cr.size(); ++e) {
        volatile T p = cv[e] * x[cc[e]];  // separate rounding of the product
        coo[cr[e]] = coo[cr[e]] + p;
    }
    size_t base = 0;
    for (int b = 0; b < static_cast<int>(opb.size()); ++b) {
        for (int lane = 0; lane < bw; ++lane) {
            const int row = b * bw + lane;
            if (row >= n) break;
            T sum = T(0);
            for (size_t k = 0; k < opb[b].size(); ++k) {
                const T v = data[(base + k) * bw + lane];
                const long col = static_cast<long>(row) + opb[b][k];
                if (v == T(0) || col < 0 || col >= n) continue;
                sum = std::fma(v, x[col], sum);
            }
            y[row] = sum;
        }
        base += opb[b].size();
    }
    if (!cr.empty())
        for (int r = 0; r < n; ++r) y[r] = y[r] + coo[r];
    return y;
}

template <typename T>
static void run_case(const char *name, HBDIA<T> &m, int bw, int thr, const std::vector<T> &xv) {
    m.convertToHBDIAFormat(bw, thr);
    HBDIAVector<T> x(xv);
    HBDIAVector<T> y(std::vector<T>(m.getNumRows(), T(0)));
    hbdiaSpMV(m, x, y, true, false);
    m.synchronize();
    std::vector<T> got;
    y.copyToHost(got);
    const std::vector<T> want = expected(m, xv);
    bool same = got.size() == want.size();
    for (size_t i = 0; same && i < got.size(); ++i) same = got[i] == want[i];
    CHECK(same, name);
}

int main() {
    {  // simple_hbdia_example.cpp single-GPU part
        HBDIA<double> m;
        m.create3DStencil27Point(8, 8, 8, 0.0);
        std::vector<double> x(m.getNumRows());
        for (int i = 0; i < m.getNumRows(); i++) x[i] = static_cast<double>(i + 1);
        run_case("8^3 stencil, bw 32 thr 2, x = i+1", m, 32, 2, x);
        CHECK(m.getNumBlocks() == 16, "8^3 stencil has 16 row blocks");
        CHECK(m.getCpuValues().empty(), "no COO remainder without noise");
    }
    {  // the comparison test's shape: stencil with noise, bw 32, GPU COO flag
        HBDIA<double> m;
        m.create3DStencil27Point(24, 24, 24, 0.01, 1);
        std::vector<double> x(m.getNumRows());
        for (int i = 0; i < m.getNumRows(); i++) x[i] = static_cast<double>(i);
        run_case("24^3 stencil with noise, bw 32 thr 2", m, 32, 2, x);
        CHECK(!m.getCpuValues().empty(), "noise lands in the COO remainder");
    }
    {  // float instantiation, block width 8
        HBDIA<float> m;
        m.create3DStencil27Point(12, 12, 12, 0.02, 3);
        std::vector<float> x(m.getNumRows());
        for (int i = 0; i < m.getNumRows(); i++) x[i] = 0.001f * static_cast<float>(i % 997);
        run_case("float 12^3 stencil, bw 8 thr 2", m, 8, 2, x);
    }
    {  // invalid flags throw like the reference
        std::vector<int> r = {0, 0, 1, 3}, c = {0, 3, 1, 0};
        std::vector<double> v = {1, 2, 3, 4};
        HBDIA<double> m(r, c, v, 4, 4);
        m.convertToHBDIAFormat(2, 2);
        HBDIAVector<double> x(std::vector<double>(4, 1.0)), y(std::vector<double>(4, 0.0));
        bool threw = false;
        try {
            hbdiaSpMV(m, x, y, false, false);
        } catch (const std::runtime_error &) {
            threw = true;
        }
        CHECK(threw, "both COO flags false with a COO remainder throws std::runtime_error");
        bool oor = false;
        try {
            HBDIA<double> bad(std::vector<int>{5}, std::vector<int>{0}, std::vector<double>{1.0}, 4, 4);
        } catch (const std::out_of_range &) {
            oor = true;
        }
        CHECK(oor, "out-of-range index throws std::out_of_range");
    }
    {  // GPU getters (include/Format/HBDIA.hpp:155-165) hold the host layout's contents
        HBDIA<double> m;
        m.create3DStencil27Point(16, 16, 16, 0.02, 2);
        m.convertToHBDIAFormat(32, 2);
        const auto &opb = m.getOffsetsPerBlock();
        std::vector<int> flat, start, sizes;
        for (const auto &b : opb) {
            start.push_back(static_cast<int>(flat.size()));
            sizes.push_back(static_cast<int>(b.size()));
            flat.insert(flat.end(), b.begin(), b.end());
        }
        start.push_back(static_cast<int>(flat.size()));
        auto down = [](const auto *d, size_t count) {
            using E = std::remove_cv_t<std::remove_pointer_t<decltype(d)>>;
            std::vector<E> h(count);
            if (d && count) CHECK_CUDA(cudaMemcpy(h.data(), d, count * sizeof(E), cudaMemcpyDeviceToHost));
            return h;
        };
        const auto &data = m.getHBDIAData();
        CHECK(m.getHBDIADataDevice() && down(m.getHBDIADataDevice(), data.size()) == data,
              "getHBDIADataDevice holds getHBDIAData");
        CHECK(down(m.getFlattenedOffsetsDevice(), flat.size()) == flat, "getFlattenedOffsetsDevice");
        CHECK(down(m.getBlockStartIndicesDevice(), start.size()) == start, "getBlockStartIndicesDevice");
        CHECK(down(m.getBlockSizesDevice(), sizes.size()) == sizes, "getBlockSizesDevice");
        CHECK(m.getFlattenedVectorOffsetsDevice() == nullptr, "no vector offsets for a whole matrix");
        const auto &cr = m.getCpuRowIndices();
        CHECK(!cr.empty() && down(m.getCpuRowIndicesDevice(), cr.size()) == cr, "getCpuRowIndicesDevice");
        CHECK(down(m.getCpuColIndicesDevice(), cr.size()) == m.getCpuColIndices(), "getCpuColIndicesDevice");
        CHECK(down(m.getCpuValuesDevice(), cr.size()) == m.getCpuValues(), "getCpuValuesDevice");
        CHECK(down(m.getCpuRowPtrDevice(), m.getCpuRowPtr().size()) == m.getCpuRowPtr(), "getCpuRowPtrDevice");
    }
    {  // DIA format and duplicate removal (src/Format/HBDIA.cpp:372-505)
        std::vector<int> r = {2, 0, 1, 0, 2, 1}, c = {0, 1, 1, 1, 2, 0};
        std::vector<double> v = {5, 1, 2, 3, 4, 6};
        HBDIA<double> d(r, c, v, 3, 3);
        CHECK(!d.isDIAFormat() && !d.getHasDIA(), "not DIA before convertToDIAFormat");
        d.convertToDIAFormat();
        CHECK(d.isDIAFormat(), "isDIAFormat after convertToDIAFormat");
        CHECK(d.getNumNonZeros() == 5, "duplicate (0,1) merged by convertToDIAFormat");
        CHECK((d.getOffsets() == std::vector<int>{-2, -1, 0, 1}), "DIA offsets ascending");
        const auto &dg = d.getDiagonals();
        CHECK(dg.size() == 4 && dg[3][0] == 4.0 && dg[2][1] == 2.0 && dg[2][2] == 4.0 && dg[1][1] == 6.0,
              "DIA diagonals hold the merged values");
        HBDIA<double> u(r, c, v, 3, 3);
        u.removeCOODuplicates();
        CHECK((u.getRowIndices() == std::vector<int>{0, 1, 1, 2, 2}) &&
                  (u.getColIndices() == std::vector<int>{1, 0, 1, 0, 2}) && u.getValues()[0] == 4.0,
              "removeCOODuplicates sums duplicates and sorts by (row, col)");
    }
    {  // the unified-memory constructor and the COO result buffer
        std::vector<double> xv(100, 2.0);
        HBDIAVector<double> a(xv, true, true, false, false);
        std::vector<double> back;
        a.copyToHost(back);
        CHECK(back == xv, "unified-memory ctor holds the data");
        double *coo = a.getDeviceCOOResultsPtr();
        CHECK(coo != nullptr && coo == a.getDeviceCOOResultsPtr(), "getDeviceCOOResultsPtr is one buffer");
        std::vector<double> z(100, 1.0);
        CHECK_CUDA(cudaMemcpy(z.data(), coo, 100 * sizeof(double), cudaMemcpyDeviceToHost));
        CHECK(z == std::vector<double>(100, 0.0), "COO result buffer starts zeroed");
    }
    {  // narrow value storage through the C++ API: quad-interleaved FP32 == per-block FP32
        HBDIA<double> m;
        m.create3DStencil27Point(24, 24, 24, 0.01, 1);
        m.convertToHBDIAFormat(32, 2);
        std::vector<double> xv(m.getNumRows());
        for (int i = 0; i < m.getNumRows(); i++) xv[i] = 1.0 + 0.25 * (i % 7);
        auto run = [&](hbdia_value_storage st) {
            m.prepareForGPU(st);
            HBDIAVector<double> x(xv);
            HBDIAVector<double> y(std::vector<double>(m.getNumRows(), 0.0));
            hbdiaSpMV(m, x, y, true, false);
            m.synchronize();
            std::vector<double> got;
            y.copyToHost(got);
            return got;
        };
        const std::vector<double> f32 = run(HBDIA_STORE_F32), quad = run(HBDIA_STORE_F32_QUAD);
        CHECK(!f32.empty() && f32 == quad, "prepareForGPU(HBDIA_STORE_F32_QUAD) gives the FP32 storage's y");
        CHECK(run(HBDIA_STORE_NATIVE) == expected(m, xv), "prepareForGPU(HBDIA_STORE_NATIVE) gives the FP64 y");
    }
    {  // CHECK_CUDA throws where the reference's exits
        bool threw = false;
        try {
            CHECK_CUDA(cudaSetDevice(1 << 20));
        } catch (const std::runtime_error &e) {
            threw = std::string(e.what()).find("CUDA error at") != std::string::npos;
        }
        cudaGetLastError();
        CHECK(threw, "CHECK_CUDA throws std::runtime_error");
    }
    std::printf(failures ? "FAILED (%d)\n" : "ALL PASSED\n", failures);
    return failures ? 1 : 0;
}
