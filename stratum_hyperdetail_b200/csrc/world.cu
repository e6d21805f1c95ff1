// Camera state, floating origin and lot-table refresh (kernels/world.cu:57-111
// of the reference): initCamera, stepCamera, clearQueue, prepareLots and
// planBounds, one view per call.
#include "common_api.cuh"
#include "world.cuh"

namespace st {

__global__ void initCameraK(float* C, uint32_t* O, int seed) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int i = 0; i < 64; i++) C[i] = 0.0f;
  for (int i = 0; i < 4; i++) O[i] = 0u;
  C[0] = 112.0f; C[1] = 76.0f; C[2] = 155.0f; C[3] = -2.53f; C[4] = -0.30f;
  C[7] = -0.55f; C[8] = 0.45f; C[9] = 0.93f; C[10] = 0.28f; C[12] = 38.0f;
  C[14] = float(seed); C[15] = 1.0f; C[19] = 1.0f; C[30] = 1.0f;
}

__global__ void stepCameraK(float* C, uint32_t* O, const float* I, float dt, int width, int height) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  stepOne(C, O, I, dt, width, height);
}

__global__ void clearQueueK(uint32_t* Q) {
  if (blockIdx.x == 0 && threadIdx.x == 0) Q[0] = 0u;
}

// One thread per table slot.
__global__ void prepareLotsK(const uint32_t* O, const float* C, float* W, uint32_t* T, uint32_t* Q) {
  int slot = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (slot >= kLots) return;
  refreshSlot(slot, O, int(C[14]), W, T, Q);
}

// Indirect-dispatch arguments of the reference's chunked bound build
// (world.cu:106-111): 8 chunks x (1 + 6 levels) x 3 u32.
__global__ void planBoundsK(const uint32_t* Q, uint32_t* A) {
  int chunk = int(threadIdx.x);
  if (chunk >= kChunks) return;
  int count = int(Q[0]) - chunk * kChunk;
  count = count < 0 ? 0 : (count > kChunk ? kChunk : count);
  uint32_t* a = A + chunk * 21;
  a[0] = uint32_t(count); a[1] = 1u; a[2] = 1u;
  int level = 1;
  for (int first = 32; first >= 1; first /= 2, level++) {
    a[level * 3] = uint32_t((count * first + 63) / 64); a[level * 3 + 1] = 1u; a[level * 3 + 2] = 1u;
  }
}

}  // namespace st

using namespace st;

extern "C" {

int stratum_initCamera(float* C, unsigned* Origin, int seed, stratum_stream_t stream) {
  if (!C || !Origin) return STRATUM_EINVAL;
  initCameraK<<<1, 1, 0, asStream(stream)>>>(C, Origin, seed);
  return launchStatus();
}
int stratum_initWorld(float* C, unsigned* Origin, int seed, stratum_stream_t stream) {
  return stratum_initCamera(C, Origin, seed, stream);
}
int stratum_stepCamera(float* C, unsigned* Origin, const float* I, float dt, int width, int height,
                       stratum_stream_t stream) {
  if (!C || !Origin || !I || !frameOk(width, height)) return STRATUM_EINVAL;
  stepCameraK<<<1, 1, 0, asStream(stream)>>>(C, Origin, I, dt, width, height);
  return launchStatus();
}
int stratum_clearQueue(unsigned* Queue, stratum_stream_t stream) {
  if (!Queue) return STRATUM_EINVAL;
  clearQueueK<<<1, 1, 0, asStream(stream)>>>(Queue);
  return launchStatus();
}
int stratum_prepareLots(const unsigned* Origin, const float* C, float* World, unsigned* Tags, unsigned* Queue,
                        stratum_stream_t stream) {
  if (!Origin || !C || !World || !Tags || !Queue) return STRATUM_EINVAL;
  prepareLotsK<<<kLots / 64, 64, 0, asStream(stream)>>>(Origin, C, World, Tags, Queue);
  return launchStatus();
}
int stratum_schedulePages(const unsigned* Origin, const float* C, float* World, unsigned* Tags, unsigned* Queue,
                          stratum_stream_t stream) {
  int s = stratum_clearQueue(Queue, stream);
  return s != STRATUM_OK ? s : stratum_prepareLots(Origin, C, World, Tags, Queue, stream);
}
int stratum_planBounds(const unsigned* Queue, unsigned* Args, stratum_stream_t stream) {
  if (!Queue || !Args) return STRATUM_EINVAL;
  planBoundsK<<<1, kChunks, 0, asStream(stream)>>>(Queue, Args);
  return launchStatus();
}
int stratum_commitPages(const unsigned* Queue, unsigned* Args, stratum_stream_t stream) {
  return stratum_planBounds(Queue, Args, stream);
}

}  // extern "C"
