// Autotuner of the batched trace: block size, queue depth (tiles claimed per
// queue access) and tile order (ray-sort key).  Each candidate is timed with
// CUDA events on the caller's stream over the caller's actual batch; the
// fastest is returned.  Only the trace kernel runs (it overwrites Hit and
// Surface, which every frame rewrites before use), so view state such as the
// sample history is left untouched.
#include <cuda_runtime.h>

#include "../../include/stratum.h"

extern "C" int stratum_traceViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                                  const stratum_tune* tune, stratum_stream_t stream);

extern "C" int stratum_autotune(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                                stratum_tune* best, float* bestMs, stratum_stream_t stream) {
  if (!views || !scratch || !best || n <= 0) return STRATUM_EINVAL;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return -int(cudaGetLastError());
  if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -int(cudaGetLastError()); }
  const int threads[3] = {64, 128, 256}, grabs[3] = {1, 2, 4}, orders[2] = {0, 1};
  float bestTime = 1e30f;
  stratum_tune pick{128, 1, 1};
  int status = STRATUM_OK;
  for (int th : threads)
    for (int g : grabs)
      for (int o : orders) {
        stratum_tune t{th, g, o};
        if ((status = stratum_traceViews(views, n, scratch, scratchBytes, &t, stream)) != STRATUM_OK) goto done;
        float total = 0.0f;
        for (int rep = 0; rep < 2; rep++) {
          cudaEventRecord(a, s);
          if ((status = stratum_traceViews(views, n, scratch, scratchBytes, &t, stream)) != STRATUM_OK) goto done;
          cudaEventRecord(b, s);
          if (cudaEventSynchronize(b) != cudaSuccess) { status = -int(cudaGetLastError()); goto done; }
          float ms = 0.0f;
          cudaEventElapsedTime(&ms, a, b);
          total += ms;
        }
        if (total < bestTime) { bestTime = total; pick = t; }
      }
done:
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (status == STRATUM_OK) {
    *best = pick;
    if (bestMs) *bestMs = bestTime / 2.0f;
  }
  return status;
}
