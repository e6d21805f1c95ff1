// tracePrimary drop-in (kernels/trace.cu:29-61 of the reference): one thread
// per pixel over a strip of rows, 8x8 blocks as the reference launches it.
#include "common_api.cuh"
#include "traverse.cuh"

// Minimum resident 64-thread blocks per SM the register allocation must allow.
#ifndef STRATUM_TRACE_MINB
#define STRATUM_TRACE_MINB 1
#endif

namespace st {

__global__ void __launch_bounds__(64, STRATUM_TRACE_MINB) tracePrimaryK(const float* __restrict__ W, const float* __restrict__ N,
                                                   const uint32_t* __restrict__ O, const float* __restrict__ C,
                                                   float* Hit, float* Surface, int width, int height, int rowStart,
                                                   int rowCount) {
  __shared__ Camera cam;
  __shared__ uint32_t org[4];
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    cam = makeCamera(C);
    for (int i = 0; i < 4; i++) org[i] = O[i];
  }
  __syncthreads();
  int x = int(blockIdx.x * blockDim.x + threadIdx.x), y = rowStart + int(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= width || y >= height || y >= rowStart + rowCount) return;
  f3 rd = primaryDir(cam, x, y, width, height);
  TraceResult r = traceRay(W, reinterpret_cast<const float4*>(N), org[0], org[2], cam.pos, rd, 1.08f / float(height));
  storeTrace(Hit, Surface, size_t(y) * width + x, r);
}

}  // namespace st

using namespace st;

extern "C" int stratum_tracePrimary(const float* World, const float* Nodes, const unsigned* Origin, const float* C,
                                    float* Hit, float* Surface, int width, int height, int rowStart, int rowCount,
                                    stratum_stream_t stream) {
  if (!World || !Nodes || !Origin || !C || !Hit || !Surface || !frameOk(width, height)) return STRATUM_EINVAL;
  if (rowStart < 0 || rowCount < 0) return STRATUM_EINVAL;
  int rows = rowCount < height - rowStart ? rowCount : height - rowStart;
  if (rows <= 0) return STRATUM_OK;
  dim3 grid((width + 7) / 8, (rows + 7) / 8);
  tracePrimaryK<<<grid, dim3(8, 8), 0, asStream(stream)>>>(World, Nodes, Origin, C, Hit, Surface, width, height,
                                                         rowStart, rowCount);
  return launchStatus();
}
