// Host-side chunk schedule of the staged SpMV kernel (see chunks.hpp).
//
// For every chunk of kTilesPerChunk row tiles: one record with the chunk's
// offset / COO ranges, and the x windows its diagonals read -- the union over
// its tiles and offsets of [32 t + off, 32 t + off + 32) clipped to [0, n),
// merged into disjoint ranges.  Each window is staged from a 16-byte-aligned
// start while the stage's x capacity lasts; what is not staged is read from
// global memory by the kernel.

#include <omp.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "chunks.hpp"
#include "hbdia_internal.hpp"

namespace hbdia {

void build_chunk_schedule(int32_t n, int32_t numBlocks, int32_t numTiles, const int32_t *blkOff,
                          const int32_t *offs, const int32_t *cooTile, int vrows, int xcap,
                          int xElemBytes, std::vector<int32_t> &rec, std::vector<XWindow> &win) {
    const int T = kTilesPerChunk;
    const int64_t numChunks = (static_cast<int64_t>(numTiles) + T - 1) / T;
    rec.assign(static_cast<size_t>(numChunks) * kRecInts, 0);
    std::vector<std::vector<XWindow>> per(static_cast<size_t>(numChunks));
    // elements per 16 bytes of x
    const int32_t al = 16 / xElemBytes;
    const int32_t nStageable = n - n % al;  // staged ranges never pass this

#pragma omp parallel
    {
        std::vector<std::pair<int32_t, int32_t>> iv;
        iv.reserve(256);
#pragma omp for schedule(dynamic, 512)
        for (int64_t c = 0; c < numChunks; ++c) {
            int32_t *R = &rec[static_cast<size_t>(c) * kRecInts];
            const int32_t t0 = static_cast<int32_t>(c * T);
            const int32_t tEnd = std::min<int32_t>(t0 + T, numTiles);
            const int32_t tBlkEnd = std::max<int32_t>(t0, std::min<int32_t>(t0 + T, numBlocks));
            const int32_t k0 = t0 < numBlocks ? blkOff[t0] : blkOff[numBlocks];
            const int32_t k1 = tBlkEnd > t0 ? blkOff[tBlkEnd] : k0;
            R[kRecT0] = t0;
            R[kRecK0] = k0;
            R[kRecK1] = k1;
            R[kRecC0] = cooTile[t0];
            R[kRecC1] = cooTile[tEnd];
            for (int w = 0; w <= T; ++w) {
                const int32_t t = t0 + w;
                R[kRecTileK + w] = t < tBlkEnd ? blkOff[t] : k1;
                R[kRecTileC + w] = cooTile[std::min(t, numTiles)];
            }
            const bool staged = (k1 - k0) <= vrows;
            R[kRecFlags] = staged ? 1 : 0;
            if (!staged) continue;
            // x ranges read by the chunk's diagonals
            iv.clear();
            for (int32_t t = t0; t < tBlkEnd; ++t) {
                const int64_t row0 = static_cast<int64_t>(t) * 32;
                for (int32_t k = blkOff[t]; k < blkOff[t + 1]; ++k) {
                    const int64_t s = std::max<int64_t>(row0 + offs[k], 0);
                    const int64_t e = std::min<int64_t>(row0 + offs[k] + 32, n);
                    if (s < e) iv.emplace_back(static_cast<int32_t>(s), static_cast<int32_t>(e));
                }
            }
            std::sort(iv.begin(), iv.end());
            std::vector<XWindow> &W = per[c];
            int32_t pos = 0, bytes = 0;
            for (size_t i = 0; i < iv.size();) {
                int32_t s = iv[i].first, e = iv[i].second;
                size_t j = i + 1;
                while (j < iv.size() && iv[j].first <= e) {
                    e = std::max(e, iv[j].second);
                    ++j;
                }
                i = j;
                if (static_cast<int>(W.size()) >= kMaxWindows) break;  // later ranges: read from global
                XWindow w;
                w.alignedStart = s - s % al;
                w.end = e;
                int32_t se = (e + al - 1) / al * al;
                if (se > nStageable) se = nStageable;
                const int32_t len = se - w.alignedStart;
                if (len > 0 && pos + len <= xcap) {
                    w.pos = pos;
                    w.stagedEnd = se;
                    pos += len;
                    bytes += len * xElemBytes;
                } else {
                    w.pos = -1;
                    w.stagedEnd = w.alignedStart;
                }
                W.push_back(w);
            }
            R[kRecNWin] = static_cast<int32_t>(W.size());
            R[kRecXBytes] = bytes;
        }
    }
    // concatenate
    int64_t total = 0;
    for (int64_t c = 0; c < numChunks; ++c) {
        rec[static_cast<size_t>(c) * kRecInts + kRecWin0] = static_cast<int32_t>(total);
        total += static_cast<int64_t>(per[c].size());
    }
    if (total > 2147483647LL) throw Error(HBDIA_ERR_UNSUPPORTED, "too many x windows");
    win.resize(static_cast<size_t>(total));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < numChunks; ++c) {
        const int64_t b = rec[static_cast<size_t>(c) * kRecInts + kRecWin0];
        std::copy(per[c].begin(), per[c].end(), win.begin() + b);
    }
}

}  // namespace hbdia
