// Per-lot 64-group bounding hierarchy (kernels/accel.cu of the reference).
//
// Drop-in entry points keep the reference's two-kernel form: buildGroupBounds
// writes the 64 leaves of each queued lot, reduceGroupBounds one level.  The
// B200 form, buildBVH, refreshes every queued lot in one launch with one block
// per lot (hierarchy.cuh); it produces the same bits.
#include <mutex>

#include "common_api.cuh"
#include "hierarchy.cuh"

namespace st {

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

__global__ void __launch_bounds__(64) buildLotHierarchyK(const uint32_t* Q, const float* W, float* N) {
  __shared__ __align__(16) float sm[kNodes][8];
  buildQueue(Q, W, N, int(blockIdx.x), int(gridDim.x), sm);
}

}  // namespace st

using namespace st;

// Resident blocks of the hierarchy kernel on the current device (SMs x
// occupancy), computed once per device; std::call_once publishes it to
// concurrent first callers.
int stratumHierarchyGrid() {
  constexpr int kDevices = 64;
  static std::once_flag once[kDevices];
  static int blocks[kDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) dev = 0;
  std::call_once(once[dev], [dev] {
    int sms = 148, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, buildLotHierarchyK, 64, 0);
    blocks[dev] = sms * (per > 0 ? per : 8);
  });
  return blocks[dev];
}

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
  buildLotHierarchyK<<<stratumHierarchyGrid(), 64, 0, asStream(stream)>>>(Queue, World, Nodes);
  return launchStatus();
}

}  // extern "C"
