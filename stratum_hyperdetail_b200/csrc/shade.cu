// shadePixels and resolveFrame drop-ins (kernels/shade.cu:45-123 of the
// reference), 8x8 blocks as the reference launches them.
#include "common_api.cuh"
#include "shading.cuh"

namespace st {

__global__ void __launch_bounds__(64) shadePixelsK(const float* __restrict__ W, const uint32_t* __restrict__ O,
                                                  const float* __restrict__ C, const float* __restrict__ Hit,
                                                  const float* __restrict__ Surface, float* Linear, int width,
                                                  int height, int rowStart, int rowCount) {
  __shared__ FrameConst F;
  if (threadIdx.x == 0 && threadIdx.y == 0) F = makeFrame(C, O);
  __syncthreads();
  int x = int(blockIdx.x * blockDim.x + threadIdx.x), y = rowStart + int(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= width || y >= height || y >= rowStart + rowCount) return;
  const size_t b = size_t(y) * width + x;
  f3 rd = primaryDir(F.cam, x, y, width, height);
  float4 h = reinterpret_cast<const float4*>(Hit)[b], s = reinterpret_cast<const float4*>(Surface)[b];
  f3 c = shadePixel(W, F, h, s, rd, height);
  reinterpret_cast<float4*>(Linear)[b] = make_float4(c.x, c.y, c.z, 1.0f);
}

__global__ void __launch_bounds__(64) resolveFrameK(const float* __restrict__ Linear, float* History, uint32_t* Pixels,
                                                   const float* __restrict__ C, const float* __restrict__ Hit,
                                                   const float* __restrict__ Surface, int width, int height) {
  __shared__ FrameConst F;
  __shared__ ResolveTaps taps;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    F = makeFrame(C, nullptr);
    taps = makeTaps();
  }
  __syncthreads();
  int x = int(blockIdx.x * blockDim.x + threadIdx.x), y = int(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= width || y >= height) return;
  float4 l4 = reinterpret_cast<const float4*>(Linear)[size_t(y) * width + x];
  resolvePixel(mk(l4.x, l4.y, l4.z), reinterpret_cast<float4*>(History), Pixels, F, taps,
               reinterpret_cast<const float4*>(Hit), reinterpret_cast<const float4*>(Surface), width, height, x, y);
}

}  // namespace st

using namespace st;

extern "C" {

int stratum_shadePixels(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                        const float* Surface, float* Linear, int width, int height, int rowStart, int rowCount,
                        stratum_stream_t stream) {
  if (!World || !Origin || !C || !Hit || !Surface || !Linear || !frameOk(width, height)) return STRATUM_EINVAL;
  if (rowStart < 0 || rowCount < 0) return STRATUM_EINVAL;
  int rows = rowCount < height - rowStart ? rowCount : height - rowStart;
  if (rows <= 0) return STRATUM_OK;
  dim3 grid((width + 7) / 8, (rows + 7) / 8);
  shadePixelsK<<<grid, dim3(8, 8), 0, asStream(stream)>>>(World, Origin, C, Hit, Surface, Linear, width, height,
                                                        rowStart, rowCount);
  return launchStatus();
}

int stratum_resolveFrame(const float* Linear, float* History, unsigned* Pixels, const float* C, const float* Hit,
                         const float* Surface, int width, int height, stratum_stream_t stream) {
  if (!Linear || !History || !Pixels || !C || !Hit || !Surface || !frameOk(width, height)) return STRATUM_EINVAL;
  dim3 grid((width + 7) / 8, (height + 7) / 8);
  resolveFrameK<<<grid, dim3(8, 8), 0, asStream(stream)>>>(Linear, History, Pixels, C, Hit, Surface, width, height);
  return launchStatus();
}

}  // extern "C"
