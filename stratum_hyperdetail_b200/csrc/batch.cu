// Batched multi-view frame path: many views of any resolution, pose and world
// seed per launch.  Each kernel reads a device table of stratum_view; every
// per-ray / per-pixel / per-lot computation is the single-view code, so a
// view's results in a batch are bit-identical to rendering it alone.
//
//   stepViewsK      one thread per view: stepCamera
//   clearViewsK,
//   refreshViewsK   clearQueue + prepareLots of all views (grid: slots x views)
//   buildViewsK     all views' queued lots, one 64-thread block per lot
//   prologueK       tile bases of every view under the chosen tile order, the
//                   per-view frame constants (camera basis, sun, origin), the
//                   resolve taps and the group caches' launch epochs, computed
//                   once per frame
//   cacheResetK     clears the directory of a full group cache the prologue
//                   chose to reset (group_cache.cuh)
//   traceViewsK     persistent: each warp claims `grab` 8x4-pixel tiles at a
//                   time from a device queue over all views and traces them
//   shadeViewsK     persistent: material colour of the same tiles (albedo into
//                   Linear; sky pixels get their final colour)
//   lightViewsK     persistent: lighting of the hit pixels from that albedo
//                   (relief normal, sun shadow, ambient, GGX, reflections, fog)
//                   into Linear -- two kernels because the shading code split in
//                   two measured faster than one (instruction fetch)
//   resolveViewsK   persistent: contact occlusion, accumulation and tone map
//                   (History, Pixels); a kernel of its own because the two
//                   fused measured slower (the shading code alone fills the
//                   instruction cache)
//
// The tile queues reset themselves: the last warp to find a queue empty zeroes
// its counters, so consecutive launches (and graph replays) need no memset.
#include <mutex>

#include "batch.cuh"
#include "common_api.cuh"
#include "hierarchy.cuh"
#include "traverse_coop.cuh"
#include "traverse_pool.cuh"
#include "world.cuh"

static_assert(sizeof(stratum_view) == 128, "stratum_view layout is part of the ABI");

namespace st {

__global__ void stepViewsK(stratum_view* V, int n) {
  int v = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (v >= n) return;
  stratum_view& w = V[v];
  stepOne(w.C, w.Origin, w.I, w.dt, w.width, w.height);
}

__global__ void applyPosesK(const stratum_view* V, const stratum_pose* P, const int* flags, int n) {
  int v = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (v >= n) return;
  const stratum_view& w = V[v];
  const int f = flags[v];
  if (f & 1) {
    const stratum_pose& p = P[v];
    w.C[0] = p.pos[0]; w.C[1] = p.pos[1]; w.C[2] = p.pos[2]; w.C[3] = p.yaw; w.C[4] = p.pitch;
    for (int i = 0; i < 4; i++) w.Origin[i] = p.origin[i];
  }
  const_cast<float*>(w.I)[23] = (f & 2) ? 1.0f : 0.0f;
}

__global__ void clearViewsK(const stratum_view* V, int n) {
  int v = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (v < n) V[v].Queue[0] = 0u;
}

__global__ void refreshViewsK(const stratum_view* __restrict__ V, int n) {
  int slot = int(blockIdx.x * blockDim.x + threadIdx.x), v = int(blockIdx.y);
  if (slot >= kLots || v >= n) return;
  const stratum_view& w = V[v];
  refreshSlot(slot, w.Origin, int(w.C[14]), w.World, w.Tags, w.Queue);
}

__global__ void __launch_bounds__(64) buildViewsK(const stratum_view* __restrict__ V, int n) {
  __shared__ __align__(16) float sm[kNodes][8];
  const int v = int(blockIdx.y);
  if (v >= n) return;
  buildQueue(V[v].Queue, V[v].World, V[v].Nodes, int(blockIdx.x), int(gridDim.x), sm);
}

// The directory of a group cache whose reset the prologue just decided.
__global__ void cacheResetK(const stratum_view* __restrict__ V, int n) {
  const int v = int(blockIdx.y);
  if (v >= n || !V[v].Groups) return;
  const GroupCacheHeader* h = reinterpret_cast<const GroupCacheHeader*>(V[v].Groups);
  if (h->capacity == 0u || h->resetAt != h->launches || h->resets == 0u) return;
  uint4* d = reinterpret_cast<uint4*>(groupCache(V[v].Groups).dir(0, 0));
  for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < kCacheDirWords / 4; i += int(gridDim.x * blockDim.x))
    d[i] = make_uint4(0u, 0u, 0u, 0u);
}
__global__ void cacheInitK(uint32_t* base, uint32_t entries) {
  GroupCacheHeader* h = reinterpret_cast<GroupCacheHeader*>(base);
  h->next = 0u; h->capacity = entries; h->resets = 0u; h->fills = 0u; h->launches = 0u; h->resetAt = 0u;
}

__global__ void prologueK(stratum_view* V, int n, int order, BatchScratch* S) {
  if (threadIdx.x == 0) {
    int base = 0;
    for (int v = 0; v < n; v++) {
      V[v].tileBase = base;
      V[v].tilesX = (V[v].width + kTileW - 1) / kTileW;
      // a view with no pixels owns no tiles (and is never looked up)
      if (V[v].width > 0 && V[v].height > 0) base += tileCount(V[v].width, V[v].height, order);
    }
    S->counters[kTotalTiles] = uint32_t(base);
    S->taps = makeTaps();
  }
  for (int v = int(threadIdx.x); v < n; v += int(blockDim.x)) {
    S->view[v] = makeFrame(V[v].C, V[v].Origin);
    if (V[v].Groups) {  // this launch's epoch; a full cache starts again now and then
      GroupCacheHeader* h = reinterpret_cast<GroupCacheHeader*>(V[v].Groups);
      h->launches++;
      if (h->capacity != 0u && h->next >= h->capacity && h->launches - h->resetAt >= kCacheResetInterval) {
        h->next = 0u;
        h->resets++;
        h->resetAt = h->launches;  // cacheResetK clears the directory next
      }
    }
  }
}

// Last view whose first tile is <= tile (binary search; warp-uniform).
SD int viewOf(const stratum_view* __restrict__ V, int n, int tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (V[mid].tileBase <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Claim `grab` tiles for this warp; returns the first, or >= total when empty.
SD int claim(uint32_t* next, int grab) {
  int t0 = 0;
  if ((threadIdx.x & 31) == 0) t0 = int(atomicAdd(next, uint32_t(grab)));
  return __shfl_sync(0xffffffffu, t0, 0);
}
// The last warp to see the queue empty resets it for the next launch.
SD void retire(uint32_t* next, uint32_t* done, int threads) {
  if ((threadIdx.x & 31) == 0) {
    __threadfence();
    uint32_t warps = gridDim.x * uint32_t(threads / 32);
    if (atomicAdd(done, 1u) == warps - 1) { *next = 0u; *done = 0u; }
  }
}

// STRATUM_TRACE_OCC / THREADS resident blocks (rounded down).  512 threads per
// SM (128 registers, a few bytes of spills): the six-view 1600x900 trace 4-5 %
// faster than at 640 (96 registers, 88/136 bytes of spills), every pose faster;
// 768 (80 registers, heavy spills) is slower still.
// The warp-cooperative traversal (traverse_coop.cuh) unless built with
// STRATUM_BATCH_PER_LANE (each lane walks its own ray, as the drop-in kernel).
#ifndef STRATUM_TRACE_OCC
#define STRATUM_TRACE_OCC 512
#endif
template <int THREADS>
__global__ void __launch_bounds__(THREADS, STRATUM_TRACE_OCC / THREADS)
    traceViewsK(const stratum_view* __restrict__ V, int n, int grab, int order, BatchScratch* S) {
  extern __shared__ __align__(16) unsigned char stageBytes[];  // THREADS / 32 WarpStage
  const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
  const int total = int(S->counters[kTotalTiles]);
#pragma unroll 1
  for (;;) {
    const int t0 = claim(&S->counters[kTraceNext], grab);
    if (t0 >= total) break;
    const int t1 = min(t0 + grab, total);
#pragma unroll 1
    for (int tile = t0; tile < t1; tile++) {
      const int v = viewOf(V, n, tile);
      const int W = V[v].width, H = V[v].height;
      int tx, ty;
      if (!tileCoord(tile - V[v].tileBase, V[v].tilesX, (H + kTileH - 1) / kTileH, order, tx, ty)) continue;
      const int x = tx * kTileW + (lane & 7), y = ty * kTileH + (lane >> 3);
      const bool inFrame = x < W && y < H;
      const Camera cam = S->view[v].cam;
      const uint32_t o0 = S->view[v].o[0], o2 = S->view[v].o[2];
      f3 rd = primaryDir(cam, inFrame ? x : 0, inFrame ? y : 0, W, H);
#ifdef STRATUM_BATCH_PER_LANE
      if (!inFrame) continue;
      TraceResult r = traceRay(V[v].World, reinterpret_cast<const float4*>(V[v].Nodes), o0, o2, cam.pos, rd,
                               1.08f / float(H));
#else
      TraceResult r = traceWarp(V[v].World, reinterpret_cast<const float4*>(V[v].Nodes), o0, o2, cam.pos, rd,
                                1.08f / float(H), inFrame, reinterpret_cast<WarpStage*>(stageBytes)[warp],
                                groupCache(V[v].Groups));
      if (!inFrame) continue;
#endif
      storeTrace(V[v].Hit, V[v].Surface, size_t(y) * W + x, r);
    }
  }
  retire(&S->counters[kTraceNext], &S->counters[kTraceDone], THREADS);
}

// The block-pooled trace (traverse_pool.cuh): a block claims THREADS / 32
// tiles at once, one per warp, and its warps serve one another's groups.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, STRATUM_TRACE_OCC / THREADS)
    tracePooledK(const stratum_view* __restrict__ V, int n, int order, BatchScratch* S) {
  constexpr int P = THREADS / 32;
  extern __shared__ __align__(16) unsigned char poolBytes[];
  PoolShared<P>& sh = *reinterpret_cast<PoolShared<P>*>(poolBytes);
  __shared__ int firstTile;
  const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
  const int total = int(S->counters[kTotalTiles]);
#pragma unroll 1
  for (;;) {
    if (threadIdx.x == 0) firstTile = int(atomicAdd(&S->counters[kTraceNext], uint32_t(P)));
    __syncthreads();
    const int t0 = firstTile;
    __syncthreads();  // every thread has read it before it is written again
    if (t0 >= total) break;
    const int tile = t0 + warp;
    int v = 0, W = 1, H = 1, tx = 0, ty = 0;
    bool ok = tile < total;
    if (ok) {
      v = viewOf(V, n, tile);
      W = V[v].width;
      H = V[v].height;
      ok = tileCoord(tile - V[v].tileBase, V[v].tilesX, (H + kTileH - 1) / kTileH, order, tx, ty);
    }
    const int x = tx * kTileW + (lane & 7), y = ty * kTileH + (lane >> 3);
    const bool inFrame = ok && x < W && y < H;
    const Camera cam = S->view[v].cam;
    const uint32_t o0 = S->view[v].o[0], o2 = S->view[v].o[2];
    const f3 rd = primaryDir(cam, inFrame ? x : 0, inFrame ? y : 0, W, H);
    const TraceResult r = tracePooled<P>(sh, V, v, V[v].World, reinterpret_cast<const float4*>(V[v].Nodes), o0, o2,
                                         cam.pos, rd, 1.08f / float(H), inFrame);
    if (inFrame) storeTrace(V[v].Hit, V[v].Surface, size_t(y) * W + x, r);
  }
  retire(&S->counters[kTraceNext], &S->counters[kTraceDone], THREADS);
}

// STRATUM_SHADE_OCC / THREADS resident blocks: 1536 threads per SM (40 registers,
// some spills) measured fastest; shading is latency-bound.
#ifndef STRATUM_SHADE_OCC
#define STRATUM_SHADE_OCC 1536
#endif
template <int THREADS>
__global__ void __launch_bounds__(THREADS, STRATUM_SHADE_OCC / THREADS) shadeViewsK(const stratum_view* __restrict__ V, int n, int grab, int order,
                                                      BatchScratch* S) {
  const int lane = int(threadIdx.x & 31);
  const int total = int(S->counters[kTotalTiles]);
#pragma unroll 1
  for (;;) {
    const int t0 = claim(&S->counters[kShadeNext], grab);
    if (t0 >= total) break;
    const int t1 = min(t0 + grab, total);
#pragma unroll 1
    for (int tile = t0; tile < t1; tile++) {
      const int v = viewOf(V, n, tile);
      const int W = V[v].width, H = V[v].height;
      int tx, ty;
      if (!tileCoord(tile - V[v].tileBase, V[v].tilesX, (H + kTileH - 1) / kTileH, order, tx, ty)) continue;
      const int x = tx * kTileW + (lane & 7), y = ty * kTileH + (lane >> 3);
      if (x >= W || y >= H) continue;
      const FrameConst F = S->view[v];
      const size_t b = size_t(y) * W + x;
      const float4* hit = reinterpret_cast<const float4*>(V[v].Hit);
      const float4* surf = reinterpret_cast<const float4*>(V[v].Surface);
      const float4 h4 = hit[b];
      const f3 rd = primaryDir(F.cam, x, y, W, H);
      f3 c;
      if (int(h4.y) == kSkyId) {
        c = skyColor(rd, F.sun);
      } else {
        SurfacePoint sp;
        surfacePoint(V[v].World, F, h4, surf[b], rd, H, sp);
        c = pixelAlbedo(sp);
      }
      reinterpret_cast<float4*>(V[v].Linear)[b] = make_float4(c.x, c.y, c.z, 1.0f);
    }
  }
  retire(&S->counters[kShadeNext], &S->counters[kShadeDone], THREADS);
}

// STRATUM_RESOLVE_OCC / THREADS resident blocks (0: the compiler's choice;
// 1024, 1536 and 2048 threads per SM measured the same).
#ifndef STRATUM_RESOLVE_OCC
#define STRATUM_RESOLVE_OCC 0
#endif
template <int THREADS>
__global__ void __launch_bounds__(THREADS, STRATUM_SHADE_OCC / THREADS) lightViewsK(const stratum_view* __restrict__ V,
                                                                                int n, int grab, int order,
                                                                                BatchScratch* S) {
  const int lane = int(threadIdx.x & 31);
  const int total = int(S->counters[kTotalTiles]);
#pragma unroll 1
  for (;;) {
    const int t0 = claim(&S->counters[kLightNext], grab);
    if (t0 >= total) break;
    const int t1 = min(t0 + grab, total);
#pragma unroll 1
    for (int tile = t0; tile < t1; tile++) {
      const int v = viewOf(V, n, tile);
      const int W = V[v].width, H = V[v].height;
      int tx, ty;
      if (!tileCoord(tile - V[v].tileBase, V[v].tilesX, (H + kTileH - 1) / kTileH, order, tx, ty)) continue;
      const int x = tx * kTileW + (lane & 7), y = ty * kTileH + (lane >> 3);
      if (x >= W || y >= H) continue;
      const size_t b = size_t(y) * W + x;
      const float4 h4 = reinterpret_cast<const float4*>(V[v].Hit)[b];
      if (int(h4.y) == kSkyId) continue;
      const FrameConst F = S->view[v];
      const f3 rd = primaryDir(F.cam, x, y, W, H);
      float4* lin = reinterpret_cast<float4*>(V[v].Linear) + b;
      const float4 a = *lin;
      SurfacePoint sp;
      surfacePoint(V[v].World, F, h4, reinterpret_cast<const float4*>(V[v].Surface)[b], rd, H, sp);
      const f3 c = pixelLight(V[v].World, F, sp, rd, int(h4.y), mk(a.x, a.y, a.z));
      *lin = make_float4(c.x, c.y, c.z, 1.0f);
    }
  }
  retire(&S->counters[kLightNext], &S->counters[kLightDone], THREADS);
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, STRATUM_RESOLVE_OCC / THREADS) resolveViewsK(const stratum_view* __restrict__ V, int n, int grab, int order,
                                                        BatchScratch* S) {
  const int lane = int(threadIdx.x & 31);
  const int total = int(S->counters[kTotalTiles]);
#pragma unroll 1
  for (;;) {
    const int t0 = claim(&S->counters[kResolveNext], grab);
    if (t0 >= total) break;
    const int t1 = min(t0 + grab, total);
#pragma unroll 1
    for (int tile = t0; tile < t1; tile++) {
      const int v = viewOf(V, n, tile);
      const int W = V[v].width, H = V[v].height;
      int tx, ty;
      if (!tileCoord(tile - V[v].tileBase, V[v].tilesX, (H + kTileH - 1) / kTileH, order, tx, ty)) continue;
      const int x = tx * kTileW + (lane & 7), y = ty * kTileH + (lane >> 3);
      if (x >= W || y >= H) continue;
      const FrameConst F = S->view[v];
      const size_t b = size_t(y) * W + x;
      const float4 l = reinterpret_cast<const float4*>(V[v].Linear)[b];
      resolvePixel(mk(l.x, l.y, l.z), reinterpret_cast<float4*>(V[v].History), V[v].Pixels, F, S->taps,
                   reinterpret_cast<const float4*>(V[v].Hit), reinterpret_cast<const float4*>(V[v].Surface), W, H, x, y);
    }
  }
  retire(&S->counters[kResolveNext], &S->counters[kResolveDone], THREADS);
}

template <class K>
int residentBlocks(K kernel, int threads, size_t smem = 0) {
  int dev = 0, sms = 148, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
  return sms * (per > 0 ? per : 1);
}
// Dynamic shared memory of a trace block: one WarpStage per warp.
constexpr size_t traceSmem(int threads) { return size_t(threads / 32) * sizeof(WarpStage); }

enum Parts { kTrace = 1, kShade = 2 };

// Persistent grids of one block size on one device: the resident-block count of
// each kernel, computed once per (block size, device) and published through
// std::call_once, so concurrent first calls (the render server's scheduler and
// a direct caller) all see the four grids complete.
constexpr int kGridDevices = 64;
struct PersistentGrids { int trace, pooled, shade, light, resolve; };

template <int T>
int launchParts(const stratum_view* V, int n, const stratum_tune& t, BatchScratch* S, cudaStream_t s, int parts) {
  static std::once_flag once[kGridDevices];
  static PersistentGrids grids[kGridDevices];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -int(e);
  if (dev < 0 || dev >= kGridDevices) return STRATUM_EINVAL;
  std::call_once(once[dev], [&] {
    PersistentGrids g;
    g.trace = residentBlocks(traceViewsK<T>, T, traceSmem(T));
    g.pooled = residentBlocks(tracePooledK<T>, T, sizeof(PoolShared<T / 32>));
    g.shade = residentBlocks(shadeViewsK<T>, T);
    g.light = residentBlocks(lightViewsK<T>, T);
    g.resolve = residentBlocks(resolveViewsK<T>, T);
    grids[dev] = g;
  });
  const PersistentGrids& g = grids[dev];
  const int order = t.order & 1;  // tile order; bit 1 selects the block-pooled trace
  if ((parts & kTrace) && (t.order & 2))
    tracePooledK<T><<<g.pooled, T, sizeof(PoolShared<T / 32>), s>>>(V, n, order, S);
  else if (parts & kTrace)
    traceViewsK<T><<<g.trace, T, traceSmem(T), s>>>(V, n, t.grab, order, S);
  if (parts & kShade) shadeViewsK<T><<<g.shade, T, 0, s>>>(V, n, t.grab, order, S);
  if (parts & kShade) lightViewsK<T><<<g.light, T, 0, s>>>(V, n, t.grab, order, S);
  if (parts & kShade) resolveViewsK<T><<<g.resolve, T, 0, s>>>(V, n, t.grab, order, S);
  return launchStatus();
}

bool tuneOk(const stratum_tune& t) {
  return (t.threads == 64 || t.threads == 128 || t.threads == 256) && t.grab >= 1 && t.grab <= 16 &&
         t.order >= 0 && t.order <= 3;
}

// parts: kTrace (with the prologue), kShade (uses the prologue's scratch), or both.
int render(stratum_view* V, int n, void* scratch, unsigned long long bytes, const stratum_tune* tune, cudaStream_t s,
           int parts) {
  if (!V || !scratch || n <= 0 || n > 65535 || bytes < batchScratchBytes(n)) return STRATUM_EINVAL;
  stratum_tune t = tune ? *tune : stratum_tune{128, 1, 1};
  if (!tuneOk(t)) return STRATUM_EINVAL;
  BatchScratch* S = static_cast<BatchScratch*>(scratch);
  if (parts & kTrace) {
    prologueK<<<1, 256, 0, s>>>(V, n, t.order & 1, S);
    cacheResetK<<<dim3(64, n), 256, 0, s>>>(V, n);
  }
  if (t.threads == 64) return launchParts<64>(V, n, t, S, s, parts);
  if (t.threads == 256) return launchParts<256>(V, n, t, S, s, parts);
  return launchParts<128>(V, n, t, S, s, parts);
}

// ---- allocation-free variant -------------------------------------------------
// The renderer's scratch (queue counters, resolve taps, per-view frame
// constants) for callers that cannot give the library device memory, held in
// one static device array.  Every GPU that loads the library holds this array
// (about 6.9 KB) until the process exits.
constexpr int kNoAllocMaxViews = STRATUM_NOALLOC_MAX_VIEWS;
constexpr size_t kNoAllocBytes = sizeof(BatchScratch) + size_t(kNoAllocMaxViews - 1) * sizeof(FrameConst);
static __device__ __align__(256) unsigned char gNoAllocScratch[kNoAllocBytes];

}  // namespace st

#include <cuda.h>
#include <mutex>

namespace {
// Device address of gNoAllocScratch per device ordinal, looked up with that
// device current on the first call in each of its contexts.  Host code must
// not use the array's name as an address: on the host it is only a stand-in
// for the device symbol.  The address belongs to the context the module was
// loaded into, so it is cached with that context's unique id: after a
// cudaDeviceReset the next call finds a new context and looks it up again.
constexpr int kMaxDevices = 128;
std::mutex gNoAllocLock;
struct NoAllocSlot { unsigned long long ctx; void* addr; };
NoAllocSlot gNoAllocAddr[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 if none or unknown),
// through the driver entry points the runtime hands out.
unsigned long long currentContextId() {
  static std::once_flag once;
  static CtxGetCurrentFn getCurrent = nullptr;
  static CtxGetIdFn getId = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      getCurrent = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      getId = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!getCurrent || !getId || getCurrent(&ctx) != CUDA_SUCCESS || !ctx || getId(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

int noAllocScratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -int(e);
  if (dev < 0 || dev >= kMaxDevices) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> hold(gNoAllocLock);
  NoAllocSlot& slot = gNoAllocAddr[dev];
  const unsigned long long ctx = currentContextId();
  if (!slot.addr || ctx == 0 || slot.ctx != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, st::gNoAllocScratch);
    if (e != cudaSuccess || !p) return e != cudaSuccess ? -int(e) : STRATUM_EINVAL;
    slot.addr = p;
    slot.ctx = currentContextId();  // the lookup has made the device's context current
  }
  *out = slot.addr;
  return STRATUM_OK;
}
}  // namespace

using namespace st;
int stratumHierarchyGrid();

extern "C" {

unsigned long long stratum_batchScratchBytes(int views) { return views > 0 ? batchScratchBytes(views) : 0; }

unsigned long long stratum_groupCacheBytes(int entries) { return entries >= 0 ? groupCacheBytes(entries) : 0; }
int stratum_groupCacheInit(unsigned* Groups, int entries, stratum_stream_t stream) {
  if (!Groups || entries < 0 || uint32_t(entries) > kCacheMaxEntries) return STRATUM_EINVAL;
  cudaError_t e = cudaMemsetAsync(Groups, 0, kCacheEntryOffset, asStream(stream));
  if (e != cudaSuccess) return -int(e);
  cacheInitK<<<1, 1, 0, asStream(stream)>>>(Groups, uint32_t(entries));
  return launchStatus();
}

int stratum_applyPoses(stratum_view* views, const stratum_pose* poses, const int* flags, int n,
                       stratum_stream_t stream) {
  if (!views || !poses || !flags || n <= 0) return STRATUM_EINVAL;
  applyPosesK<<<(n + 63) / 64, 64, 0, asStream(stream)>>>(views, poses, flags, n);
  return launchStatus();
}
int stratum_stepViews(stratum_view* views, int n, stratum_stream_t stream) {
  if (!views || n <= 0) return STRATUM_EINVAL;
  stepViewsK<<<(n + 63) / 64, 64, 0, asStream(stream)>>>(views, n);
  return launchStatus();
}
int stratum_refreshViews(stratum_view* views, int n, stratum_stream_t stream) {
  if (!views || n <= 0 || n > 65535) return STRATUM_EINVAL;
  clearViewsK<<<(n + 63) / 64, 64, 0, asStream(stream)>>>(views, n);
  refreshViewsK<<<dim3(kLots / 128, n), 128, 0, asStream(stream)>>>(views, n);
  return launchStatus();
}
int stratum_buildViews(stratum_view* views, int n, stratum_stream_t stream) {
  if (!views || n <= 0 || n > 65535) return STRATUM_EINVAL;
  int per = stratumHierarchyGrid() / n;
  buildViewsK<<<dim3(per < 16 ? 16 : per, n), 64, 0, asStream(stream)>>>(views, n);
  return launchStatus();
}
int stratum_traceViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream) {
  return render(views, n, scratch, scratchBytes, tune, asStream(stream), kTrace);
}
int stratum_shadeViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream) {
  return render(views, n, scratch, scratchBytes, tune, asStream(stream), kShade);
}
int stratum_renderViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                        const stratum_tune* tune, stratum_stream_t stream) {
  return render(views, n, scratch, scratchBytes, tune, asStream(stream), kTrace | kShade);
}
// renderViews with the library's static scratch: allocates nothing, calls no
// allocating routine.  The queue counters are cleared on the stream first, so
// the call does not depend on how an earlier call ended.
int stratum_renderViewsNoAlloc(stratum_view* views, int n, const stratum_tune* tune, stratum_stream_t stream) {
  if (!views || n <= 0) return STRATUM_EINVAL;
  if (n > kNoAllocMaxViews) return STRATUM_ELIMIT;
  void* scratch = nullptr;
  int s = noAllocScratch(&scratch);
  if (s != STRATUM_OK) return s;
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * kCounters, asStream(stream));
  if (e != cudaSuccess) return -int(e);
  return render(views, n, scratch, kNoAllocBytes, tune, asStream(stream), kTrace | kShade);
}
int stratum_frameViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream) {
  int s;
  if ((s = stratum_stepViews(views, n, stream)) != STRATUM_OK) return s;
  if ((s = stratum_refreshViews(views, n, stream)) != STRATUM_OK) return s;
  if ((s = stratum_buildViews(views, n, stream)) != STRATUM_OK) return s;
  return stratum_renderViews(views, n, scratch, scratchBytes, tune, stream);
}

}  // extern "C"
