// The per-frame sequence of the reference engine (src/engine.js:67-83) over
// the drop-in entry points: stepCamera, clearQueue, prepareLots, planBounds,
// the hierarchy refresh, then trace and shade in 64-row strips, then resolve.
// Everything is enqueued on one stream; nothing synchronises.
#include "../../include/stratum.h"

extern "C" {

int stratum_frame(float* C, unsigned* Origin, const float* I, float dt, float* World, unsigned* Tags, float* Nodes,
                  unsigned* Queue, unsigned* Args, float* Hit, float* Surface, float* Linear, float* History,
                  unsigned* Pixels, int width, int height, int draw, stratum_stream_t stream) {
  if (!C || !Origin || !I || !World || !Tags || !Nodes || !Queue) return STRATUM_EINVAL;
  if (draw && (!Hit || !Surface || !Linear || !History || !Pixels)) return STRATUM_EINVAL;
  if (width <= 0 || height <= 0 || width > STRATUM_MAX_DIM || height > STRATUM_MAX_DIM) return STRATUM_EINVAL;
  // src/engine.js:69 clamps dt to [0, 0.1].
  float step = dt < 0.0f ? 0.0f : (dt > 0.1f ? 0.1f : dt);
  int s;
  if ((s = stratum_stepCamera(C, Origin, I, step, width, height, stream)) != STRATUM_OK) return s;
  if ((s = stratum_clearQueue(Queue, stream)) != STRATUM_OK) return s;
  if ((s = stratum_prepareLots(Origin, C, World, Tags, Queue, stream)) != STRATUM_OK) return s;
  if (Args && (s = stratum_planBounds(Queue, Args, stream)) != STRATUM_OK) return s;
  if ((s = stratum_buildBVH(Queue, World, Nodes, stream)) != STRATUM_OK) return s;
  if (!draw) return STRATUM_OK;
  const int rows = 64;
  for (int y = 0; y < height; y += rows) {
    int count = height - y < rows ? height - y : rows;
    if ((s = stratum_tracePrimary(World, Nodes, Origin, C, Hit, Surface, width, height, y, count, stream)) != STRATUM_OK)
      return s;
  }
  for (int y = 0; y < height; y += rows) {
    int count = height - y < rows ? height - y : rows;
    if ((s = stratum_shadePixels(World, Origin, C, Hit, Surface, Linear, width, height, y, count, stream)) != STRATUM_OK)
      return s;
  }
  return stratum_resolveFrame(Linear, History, Pixels, C, Hit, Surface, width, height, stream);
}

const char* stratum_version(void) { return "stratum-b200 0.1.0 (sm_100a)"; }

}  // extern "C"
