// Per-lot 64-group bounding hierarchy (kernels/accel.cu of the reference).
//
// Drop-in entry points keep the reference's two-kernel form: buildGroupBounds
// writes the 64 leaves of each queued lot, reduceGroupBounds one level.  The
// B200 form, buildLotHierarchy, does a whole lot in one 64-thread block: each
// thread runs the grammar of one group in bounds mode, the 63 internal nodes
// are reduced in shared memory, and the 127 nodes leave as one coalesced 4 KiB
// store.  Min/max and small-integer sums are exact, so every form produces the
// same bits.  Node 0 of each lot block is never written (the reference leaves
// it untouched).
#include "common_api.cuh"
#include "grammar.cuh"

namespace st {

// Queue length clamped to the table, so a stale count never reads past the queue.
__device__ __forceinline__ int queued(const uint32_t* Q) { return int(min(Q[0], uint32_t(kLots))); }

__device__ __forceinline__ void leafBounds(const LotDesc& lot, int g, float* n) {
  BoundsSink s;
  int count = runGroup(lot, g, s);
  n[0] = s.lo.x; n[1] = s.lo.y; n[2] = s.lo.z; n[3] = float(count);
  n[4] = s.hi.x; n[5] = s.hi.y; n[6] = s.hi.z; n[7] = float(g);
}

__global__ void __launch_bounds__(64) buildGroupBoundsK(const uint32_t* Q, const float* W, float* N, int queueBase) {
  int q = queueBase + int(blockIdx.x), g = int(threadIdx.x);
  if (q >= queued(Q) || g >= kGroups) return;
  int slot = int(Q[q + 1]);
  if (slot < 0 || slot >= kLots) return;
  LotDesc lot = loadLot(W, slot);
  float n[8];
  leafBounds(lot, g, n);
  float4* dst = reinterpret_cast<float4*>(N + (size_t(slot) * kNodes + kGroups + g) * 8);
  dst[0] = make_float4(n[0], n[1], n[2], n[3]);
  dst[1] = make_float4(n[4], n[5], n[6], n[7]);
}

__global__ void reduceGroupBoundsK(const uint32_t* Q, float* N, int first, int queueBase) {
  int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  int q = queueBase + i / first, j = i % first + first;
  if (q >= queued(Q) || q >= queueBase + kChunk) return;
  int slot = int(Q[q + 1]);
  if (slot < 0 || slot >= kLots) return;
  float* b = N + (size_t(slot) * kNodes + j) * 8;
  const float *a = N + (size_t(slot) * kNodes + 2 * j) * 8, *c = a + 8;
  for (int k = 0; k < 3; k++) { b[k] = fminf(a[k], c[k]); b[4 + k] = fmaxf(a[4 + k], c[4 + k]); }
  b[3] = a[3] + c[3];
  b[7] = 0.0f;
}

// One block (64 threads) per queued lot, grid-striding over the queue.
__device__ __forceinline__ void lotHierarchy(const float* W, float* N, int slot, float (*sm)[8]) {
  const int g = int(threadIdx.x);
  LotDesc lot = loadLotRW(W, slot);
  leafBounds(lot, g, sm[kGroups + g]);
  __syncthreads();
#pragma unroll 1
  for (int first = 32; first >= 1; first >>= 1) {
    if (g < first) {
      int j = first + g;
      float *b = sm[j], *a = sm[2 * j], *c = sm[2 * j + 1];
#pragma unroll
      for (int k = 0; k < 3; k++) { b[k] = fminf(a[k], c[k]); b[4 + k] = fmaxf(a[4 + k], c[4 + k]); }
      b[3] = a[3] + c[3];
      b[7] = 0.0f;
    }
    __syncthreads();
  }
  float4* dst = reinterpret_cast<float4*>(N + size_t(slot) * kNodes * 8);
  const float4* src = reinterpret_cast<const float4*>(&sm[0][0]);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int i = g + 64 * k;  // float4 index within the 4 KiB block; 0 and 1 are node 0
    if (i >= 2) dst[i] = src[i];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(64) buildLotHierarchyK(const uint32_t* Q, const float* W, float* N) {
  __shared__ __align__(16) float sm[kNodes][8];
  const int count = queued(Q);
#pragma unroll 1
  for (int q = int(blockIdx.x); q < count; q += int(gridDim.x)) {
    int slot = int(Q[q + 1]);
    if (slot >= 0 && slot < kLots) lotHierarchy(W, N, slot, sm);
  }
}

// All views' refresh queues in one launch: blockIdx.y is the view.
__global__ void __launch_bounds__(64) buildLotHierarchyBatchK(const uint32_t* Q, const float* W, float* N, int views) {
  __shared__ __align__(16) float sm[kNodes][8];
  const int v = int(blockIdx.y);
  if (v >= views) return;
  const uint32_t* q0 = Q + size_t(v) * (kLots + 1);
  const float* w0 = W + size_t(v) * kLots * kLotFloats;
  float* n0 = N + size_t(v) * kLots * kNodes * 8;
  const int count = queued(q0);
#pragma unroll 1
  for (int q = int(blockIdx.x); q < count; q += int(gridDim.x)) {
    int slot = int(q0[q + 1]);
    if (slot >= 0 && slot < kLots) lotHierarchy(w0, n0, slot, sm);
  }
}

int hierarchyGrid() {
  static int blocks = 0;
  if (!blocks) {
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, buildLotHierarchyK, 64, 0);
    blocks = sms * (per > 0 ? per : 8);
  }
  return blocks;
}

}  // namespace st

using namespace st;

extern "C" {

int stratum_buildGroupBounds(const unsigned* Queue, const float* World, float* Nodes, int queueBase,
                             stratum_stream_t stream) {
  if (!Queue || !World || !Nodes || queueBase < 0 || queueBase >= kLots) return STRATUM_EINVAL;
  buildGroupBoundsK<<<kChunk, 64, 0, asStream(stream)>>>(Queue, World, Nodes, queueBase);
  return launchStatus();
}
int stratum_reduceGroupBounds(const unsigned* Queue, float* Nodes, int first, int queueBase, stratum_stream_t stream) {
  if (!Queue || !Nodes || queueBase < 0 || queueBase >= kLots) return STRATUM_EINVAL;
  if (first != 32 && first != 16 && first != 8 && first != 4 && first != 2 && first != 1) return STRATUM_EINVAL;
  reduceGroupBoundsK<<<(kChunk * first + 63) / 64, 64, 0, asStream(stream)>>>(Queue, Nodes, first, queueBase);
  return launchStatus();
}
int stratum_buildBVH(const unsigned* Queue, const float* World, float* Nodes, stratum_stream_t stream) {
  if (!Queue || !World || !Nodes) return STRATUM_EINVAL;
  buildLotHierarchyK<<<hierarchyGrid(), 64, 0, asStream(stream)>>>(Queue, World, Nodes);
  return launchStatus();
}
int stratum_buildBVHBatch(const unsigned* Queue, const float* World, float* Nodes, int views, stratum_stream_t stream) {
  if (!Queue || !World || !Nodes || views <= 0 || views > 65535) return STRATUM_EINVAL;
  int per = hierarchyGrid() / views;
  buildLotHierarchyBatchK<<<dim3(per < 16 ? 16 : per, views), 64, 0, asStream(stream)>>>(Queue, World, Nodes, views);
  return launchStatus();
}

}  // extern "C"
