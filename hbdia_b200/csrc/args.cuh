// Kernel argument block of one device plan (shared by the launchers).
#pragma once

#include "hbdia_internal.hpp"
#include "spmv_kernels.cuh"

namespace hbdia {

template <typename VT, typename XT>
inline dev::SpmvArgs<VT, XT> make_args(const DevicePlan &P) {
    dev::SpmvArgs<VT, XT> a;
    a.vals = static_cast<const VT *>(P.vals);
    a.scale = P.scale;
    a.offs = P.offs;
    a.blkOff = P.blkOff;
    a.cooRow = P.cooRow;
    a.cooCol = P.cooCol;
    a.cooVal = static_cast<const XT *>(P.cooVal);
    a.cooRowPtr = P.cooRowPtr;
    a.cooTile = P.cooTile;
    a.n = P.n;
    a.xn = P.xn;
    a.bw = P.bw;
    a.numBlocks = P.numBlocks;
    a.numTiles = P.numTiles;
    a.hasCoo = P.nCoo > 0;
    a.quadLayout = P.quadLayout ? 1 : 0;
    return a;
}

}  // namespace hbdia
