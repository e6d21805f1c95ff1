// tracePrimary drop-in (kernels/trace.cu:29-61 of the reference): every pixel of
// a strip of rows.
//
// A block covers 16x16 pixels with eight warps, each tracing one 8x4 tile with
// the warp-cooperative traversal of the batched renderer (traverse_coop.cuh):
// lanes walk their own rays to the hierarchy leaves, and the warp evaluates one
// (lot, group) at a time for every lane waiting on it.  The drop-in has only
// the reference's buffers, so there is no table-wide group cache; instead the
// block keeps the groups its warps build (by the random-access grammar) in a
// shared-memory table, and a warp that needs a group another warp of the block
// has built reads it from there (neighbouring tiles reach the same groups: on
// the bench poses a 16x16 block needs 6-9x fewer group builds than its warps
// would alone).  Each ray still visits its leaves in the reference's order with
// the same running best, so Hit and Surface equal the per-thread traversal
// (traverse.cuh) bit for bit; building with STRATUM_DROPIN_PER_LANE selects that
// per-thread form instead.
//
// The reference's 64-row strips leave each launch a tail of partly idle SMs:
// six 1600x900 views in 15 strips each trace in 24.4 ms, in one call per view
// (rowCount = height, which the entry point accepts) in 14.3 ms.  A
// programmatic dependent launch of each strip was tried and measured no
// faster: a dependent grid may be scheduled early, but its griddepcontrol.wait
// returns only once the preceding grid has completed, and skipping that wait is
// safe only when the preceding kernel is known to be another strip.
#include <mutex>

#include "common_api.cuh"
#include "traverse_coop.cuh"

// Block shape in 8x4-pixel warp tiles, and resident blocks per SM the register
// allocation must allow (2 blocks of 2 x 4 tiles: 512 threads, up to 128
// registers a thread).
#ifndef STRATUM_DROPIN_TILES_X
#define STRATUM_DROPIN_TILES_X 2
#endif
#ifndef STRATUM_DROPIN_TILES_Y
#define STRATUM_DROPIN_TILES_Y 4
#endif
#ifndef STRATUM_DROPIN_BLOCKS
#define STRATUM_DROPIN_BLOCKS 2
#endif

namespace st {

constexpr int kDropInTilesX = STRATUM_DROPIN_TILES_X, kDropInTilesY = STRATUM_DROPIN_TILES_Y;
constexpr int kDropInThreads = 32 * kDropInTilesX * kDropInTilesY;
constexpr int kDropInW = 8 * kDropInTilesX, kDropInH = 4 * kDropInTilesY;
struct DropInShared {
  WarpStage stage[kDropInThreads / 32];
  BlockCache cache;
};

__global__ void __launch_bounds__(kDropInThreads, STRATUM_DROPIN_BLOCKS)
    tracePrimaryK(const float* __restrict__ W, const float* __restrict__ N, const uint32_t* __restrict__ O,
                  const float* __restrict__ C, float* Hit, float* Surface, int width, int height, int rowStart,
                  int rowCount) {
  extern __shared__ __align__(16) unsigned char dropInBytes[];
  DropInShared& sh = *reinterpret_cast<DropInShared*>(dropInBytes);
  __shared__ Camera cam;
  __shared__ uint32_t org[4];
  if (threadIdx.x == 0) {
    cam = makeCamera(C);
    for (int i = 0; i < 4; i++) org[i] = O[i];
  }
  blockCacheInit(sh.cache);
  __syncthreads();
  const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
  const int x = int(blockIdx.x) * kDropInW + (warp % kDropInTilesX) * 8 + (lane & 7);
  const int y = rowStart + int(blockIdx.y) * kDropInH + (warp / kDropInTilesX) * 4 + (lane >> 3);
  const bool active = x < width && y < height && y < rowStart + rowCount;
  const f3 rd = primaryDir(cam, active ? x : 0, active ? y : 0, width, height);
#ifdef STRATUM_DROPIN_PER_LANE
  if (!active) return;
  const TraceResult r = traceRay(W, reinterpret_cast<const float4*>(N), org[0], org[2], cam.pos, rd,
                                 1.08f / float(height));
#else
  const TraceResult r = traceWarp<true>(W, reinterpret_cast<const float4*>(N), org[0], org[2], cam.pos, rd,
                                        1.08f / float(height), active, sh.stage[warp], groupCache(nullptr),
                                        &sh.cache);
  if (!active) return;
#endif
  storeTrace(Hit, Surface, size_t(y) * width + x, r);
}

}  // namespace st

using namespace st;

namespace {
constexpr int kSmemDevices = 64;
}

extern "C" int stratum_tracePrimary(const float* World, const float* Nodes, const unsigned* Origin, const float* C,
                                    float* Hit, float* Surface, int width, int height, int rowStart, int rowCount,
                                    stratum_stream_t stream) {
  if (!World || !Nodes || !Origin || !C || !Hit || !Surface || !frameOk(width, height)) return STRATUM_EINVAL;
  if (rowStart < 0 || rowCount < 0) return STRATUM_EINVAL;
  int rows = rowCount < height - rowStart ? rowCount : height - rowStart;
  if (rows <= 0) return STRATUM_OK;
  static std::once_flag once[kSmemDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kSmemDevices) return STRATUM_EINVAL;
  std::call_once(once[dev], [] {
    cudaFuncSetAttribute(tracePrimaryK, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(DropInShared)));
  });
  dim3 grid((width + kDropInW - 1) / kDropInW, (rows + kDropInH - 1) / kDropInH);
  tracePrimaryK<<<grid, kDropInThreads, sizeof(DropInShared), asStream(stream)>>>(
      World, Nodes, static_cast<const uint32_t*>(Origin), C, Hit, Surface, width, height, rowStart, rowCount);
  return launchStatus();
}
