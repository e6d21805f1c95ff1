// Multi-view batch: scratch layout shared by the batched kernels.
#pragma once
#include <cstdint>
#include "../../include/stratum.h"
#include "shading.cuh"

namespace st {

constexpr int kTileW = 8, kTileH = 4;  // one warp per 8x4 pixel tile

// Scratch: 16 u32 counters, the resolve taps, then one FrameConst per view.
enum : int {
  kTraceNext = 0,   // next tile to claim (trace)
  kTraceDone = 1,   // warps that found the queue empty (trace)
  kShadeNext = 2,
  kShadeDone = 3,
  kTotalTiles = 4,  // tiles over all views (written by the prologue)
  kResolveNext = 5,
  kResolveDone = 6,
  kLightNext = 7,
  kLightDone = 8,
  kCounters = 16
};
struct BatchScratch {
  uint32_t counters[kCounters];
  ResolveTaps taps;
  FrameConst view[1];  // n entries
};
inline size_t batchScratchBytes(int views) {
  return sizeof(BatchScratch) + size_t(views > 1 ? views - 1 : 0) * sizeof(FrameConst);
}

// Tile count of a view under an order: row-major tiles, or whole 4x4-tile
// super-tiles (Morton order inside each) whose out-of-frame tiles are skipped.
SD int tileCount(int width, int height, int order) {
  int tx = (width + kTileW - 1) / kTileW, ty = (height + kTileH - 1) / kTileH;
  if (order == 1) return ((tx + 3) / 4) * ((ty + 3) / 4) * 16;
  return tx * ty;
}
SD bool tileCoord(int local, int tilesX, int tilesY, int order, int& tx, int& ty) {
  if (order == 1) {
    int st = local >> 4, w = local & 15, superX = (tilesX + 3) / 4;
    tx = (st % superX) * 4 + ((w & 1) | ((w >> 1) & 2));
    ty = (st / superX) * 4 + (((w >> 1) & 1) | ((w >> 2) & 2));
  } else {
    tx = local % tilesX;
    ty = local / tilesX;
  }
  return tx < tilesX && ty < tilesY;
}

}  // namespace st
