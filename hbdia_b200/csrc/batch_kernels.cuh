// Many HBDIA matrices in one persistent launch (sm_100a): the "queue"
// schedule of a batch.  (The default "concurrent" schedule runs each
// matrix's own single-matrix kernel instead; see batch.cu.)
//
// The 32-row tiles of the matrices of one launch segment form one index
// space: entry m owns tiles [e[m].tileBase, e[m+1].tileBase).  Each warp takes
// `grab` consecutive tiles at a time from an atomic counter (zeroed before
// the launch) until the space is exhausted, so small and large matrices, and
// matrices with k right-hand sides next to single-vector ones, share the SMs
// without a launch per matrix and without idle tails.
//
// The entry table is the kernel's own parameter block (__grid_constant__,
// read through the constant cache) rather than a table in global memory:
// that removed the register spills of the tile loop and raised a 256^3
// stencil from 3.7 to 4.3 TB/s on B200.  The single-matrix kernels, whose
// arguments sit at fixed parameter offsets, still keep more loads in flight
// (5.4-5.6 TB/s), which is why this schedule is for batches of many tiny
// matrices.  A segment holds up to kBatchSeg matrices (about 22 KB of the
// 32 KB parameter limit); larger batches are several segments.
//
// A tile is computed by exactly the code of the single-matrix kernels
// (bw32_tile for k == 1, bw32_spmm_tile for k > 1), so every y is bit for bit
// what hbdia_spmv_device / hbdia_spmm_device give for that matrix alone.
// KT == 0 instantiates the single-vector form only (fewer registers, for
// segments whose k are all 0 or 1); KT > 0 is the RHS tile of k > 1 entries.
#pragma once

#include "spmm_kernels.cuh"

namespace hbdia {
namespace dev {

constexpr int kBatchSeg = 160;  // matrices per launch segment

// One matrix of a batch and its bound vectors.
template <typename VT, typename XT>
struct BatchEntry {
    SpmvArgs<VT, XT> a;
    const XT *X;       // x (k == 1), or the right-hand sides, row-major n x k
    XT *Y;
    int64_t ldx, ldy;  // leading dimensions of X and Y (k > 1)
    int32_t k;         // right-hand sides; 0 skips the matrix
    int32_t tileBase;  // first tile of this matrix in the segment's index space
};

template <typename VT, typename XT>
struct BatchSeg {
    BatchEntry<VT, XT> e[kBatchSeg];
    int32_t *next;       // work counter, zero when the launch starts
    int32_t count;       // entries used
    int32_t totalTiles;  // tiles of the segment
    int32_t grab;        // tiles a warp takes per atomic
};

template <typename VT, typename XT, int U, int KT>
__global__ void __launch_bounds__(512)
spmv_bw32_batch(const __grid_constant__ BatchSeg<VT, XT> s) {
    const int lane = threadIdx.x & 31;
    int32_t m = 0, mBase = 0, mEnd = 0;  // entry and tile range of the current matrix
    for (;;) {
        int32_t g0 = 0;
        if (lane == 0) g0 = atomicAdd(s.next, s.grab);
        g0 = __shfl_sync(kFull, g0, 0);
        if (g0 >= s.totalTiles) break;
        const int32_t g1 = min(g0 + s.grab, s.totalTiles);
        for (int32_t g = g0; g < g1; ++g) {
            if (g < mBase || g >= mEnd) {
                // largest m with e[m].tileBase <= g (e[0].tileBase = 0)
                int32_t lo = 0, hi = s.count;
                while (hi - lo > 1) {
                    const int32_t mid = (lo + hi) >> 1;
                    if (s.e[mid].tileBase <= g) lo = mid;
                    else hi = mid;
                }
                m = lo;
                mBase = s.e[m].tileBase;
                mEnd = m + 1 < s.count ? s.e[m + 1].tileBase : s.totalTiles;
            }
            const BatchEntry<VT, XT> &e = s.e[m];
            const int32_t tile = g - mBase;
            if (e.k == 1) {
                bw32_tile<VT, XT, U>(e.a, e.X, e.Y, tile, lane);
            } else if constexpr (KT > 0) {
                if (e.k > 1) bw32_spmm_tile<VT, XT, KT>(e.a, e.X, e.ldx, e.Y, e.ldy, e.k, tile, lane);
            }
        }
    }
}

}  // namespace dev
}  // namespace hbdia
