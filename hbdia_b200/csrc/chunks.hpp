// Chunk schedule of the staged (TMA) SpMV kernel: shared by the host-side
// builder (chunks.cpp) and the kernel (spmv_tma.cuh).
#pragma once

#include <stdint.h>

namespace hbdia {

// A chunk is kTilesPerChunk consecutive 32-row tiles.  The host describes
// each chunk with one fixed-size record and a list of x windows (merged
// ranges of x that the chunk's diagonals read); the kernel's producer warp
// copies the chunk's values, offsets, x windows and COO remainder into one
// shared-memory stage from that description alone.
constexpr int kTilesPerChunk = 4;
constexpr int kRecInts = 24;  // record size in int32 (96 bytes, 16-byte multiple)

// record fields
enum ChunkRec : int {
    kRecT0 = 0,        // first tile of the chunk
    kRecFlags = 1,     // bit 0: values/offsets/x staged (rows fit the stage)
    kRecK0 = 2,        // first stored-offset index of the chunk (blkOff[t0])
    kRecK1 = 3,        // one past the last (blkOff[min(t0+T, numBlocks)])
    kRecC0 = 4,        // first COO entry of the chunk
    kRecC1 = 5,        // one past the last
    kRecWin0 = 6,      // first window of the chunk in the window list
    kRecNWin = 7,      // windows of the chunk in the table (<= kMaxWindows)
    kRecXBytes = 8,    // bytes of x staged for the chunk
    kRecTileK = 9,     // kTilesPerChunk + 1 tile starts in offset units (absolute)
    kRecTileC = kRecTileK + kTilesPerChunk + 1,  // kTilesPerChunk + 1 tile starts in COO entries
};
static_assert(kRecTileC + kTilesPerChunk + 1 <= kRecInts, "record too small");

constexpr int kMaxWindows = 32;  // window table entries per chunk (one per producer lane)

// Window entry (int4): x range [start, end) needed by the chunk; staged part
// [alignedStart, stagedEnd) lives at stage position pos (elements), or
// pos = -1 when not staged (then stagedEnd == alignedStart).
struct XWindow {
    int32_t alignedStart;  // start rounded down to 16 bytes of x
    int32_t end;           // true end (exclusive)
    int32_t pos;           // element position in the stage's x buffer, or -1
    int32_t stagedEnd;     // end of the staged part (exclusive)
};

}  // namespace hbdia
