// FP32 issue-rate probe: the denominator of the frame path's roofline.
//
// The trace and shade kernels are bound by FP32/ALU instruction issue, not by
// HBM or tensor cores, so their roofline is the rate at which the SMs retire
// independent FP32 lane operations.  This kernel measures it on the running
// GPU: every thread keeps 8 independent multiply-add chains (two instructions
// each, since the library is built without FMA contraction) in registers, so
// the only limit is issue.  ops = threads x iters x 8 chains x 2.
#include "common_api.cuh"

namespace st {
__global__ void __launch_bounds__(256) issueProbeK(float* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = float(threadIdx.x + k);
#pragma unroll 1
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == 123.456f) out[0] = s;  // keeps the chains live; practically never stores
}
}  // namespace st

extern "C" int stratum_issueProbe(float* out, int blocks, int iters, stratum_stream_t stream) {
  if (!out || blocks <= 0 || iters <= 0) return STRATUM_EINVAL;
  st::issueProbeK<<<blocks, 256, 0, st::asStream(stream)>>>(out, iters, 0.999999f, 0.000001f);
  return st::launchStatus();
}
