// Shared host-side helpers of the C ABI launchers.
#pragma once
#include <cuda_runtime.h>
#include "../../include/stratum.h"

namespace st {
// Map the state after a launch to the ABI's status codes.
inline int launchStatus() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? STRATUM_OK : -int(e);
}
inline cudaStream_t asStream(stratum_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
inline bool frameOk(int width, int height) {
  return width > 0 && height > 0 && width <= STRATUM_MAX_DIM && height <= STRATUM_MAX_DIM;
}
}  // namespace st
