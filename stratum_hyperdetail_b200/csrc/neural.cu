// The optional material surrogate's kernels (kernels/learning.cu of the
// reference, see neural.cuh): parameter initialisation, one training step and
// the surrogate-shaded drop-in.
//
// A training step is ~64 samples x 291 parameters of work, so the reference's
// five launches (prepare, forward, score, gradient, Adam) are one block here:
// the samples' work rows and the gradient stay in shared memory and the phases
// are separated by block barriers.
#include "common_api.cuh"
#include "neural.cuh"

namespace st {

// learning.cu:5-10
__global__ void initNeuralK(float* W, float* M, float* V, float* Brain, int seed) {
  const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i < kNnParams) {
    W[i] = (hash1(i + seed) - 0.5f) * 0.08f;
    M[i] = 0.0f;
    V[i] = 0.0f;
    if (i >= kNnW2) W[i] = 0.0f;
  }
  if (i < 32) Brain[i] = 0.0f;
  if (i == kNnB2) W[i] = 0.36f;
  if (i == kNnB2 + 1) W[i] = 0.29f;
  if (i == kNnB2 + 2) W[i] = 0.20f;
}

constexpr int kStepThreads = 320;  // >= 291 parameters and >= 64 samples

// One training step (learning.cu:11-58) on a frame's Hit/Surface.
__global__ void __launch_bounds__(kStepThreads) materialStepK(const float* __restrict__ World,
                                                             const uint32_t* __restrict__ O,
                                                             const float* __restrict__ C,
                                                             const float* __restrict__ Hit,
                                                             const float* __restrict__ Surface, float* W, float* M,
                                                             float* V, float* Brain, float* WorkOut, int width,
                                                             int height) {
  __shared__ float work[kNnBatch * kNnWs];
  __shared__ float grad[kNnParams];
  __shared__ FrameConst F;
  if (!materialTrainNow(C)) return;  // uniform over the block
  const int i = int(threadIdx.x);
  if (i == 0) F = makeFrame(C, O);
  __syncthreads();
  // prepare (learning.cu:11-24): the last of six hashed pixels that hit brick or stone
  if (i < kNnBatch) {
    float* w = work + i * kNnWs;
    int chosen = -1;
    for (int trial = 0; trial < 6; trial++) {
      const int px = int(hash1(i * 1877 + trial * 331 + int(C[6]) * 59) * float(width * height));
      const int id = int(Hit[px * 4 + 1]);
      if (id >= 0) {
        const int mat = int(Hit[px * 4 + 2]);
        if (mat == 0 || mat == 1) chosen = px;
      }
    }
    for (int j = 0; j < kNnWs; j++) w[j] = 0.0f;
    if (chosen >= 0) {
      const int x = chosen % width, y = chosen / width;
      const f3 rd = primaryDir(F.cam, x, y, width, height);
      const float4 h = reinterpret_cast<const float4*>(Hit)[chosen];
      const float4 s = reinterpret_cast<const float4*>(Surface)[chosen];
      SurfacePoint sp;
      surfacePoint(World, F, h, s, rd, height, sp);
      const int mat = int(h.z);
      for (int j = 0; j < kNnInputs; j++) w[j] = nnFeature(j, sp.u, sp.v, h.w, mat);
      const f3 target = substrate(sp.u, sp.v, h.w, mat);
      w[kNnTarget] = target.x; w[kNnTarget + 1] = target.y; w[kNnTarget + 2] = target.z;
      w[kNnValid] = 1.0f;
      w[kNnMat] = float(mat);
    }
  }
  __syncthreads();
  // forward (learning.cu:25-29)
  if (i < kNnBatch) {
    float* w = work + i * kNnWs;
    for (int h = 0; h < kNnHidden; h++) {
      float z = W[kNnB1 + h];
      for (int j = 0; j < kNnInputs; j++) z += W[h * 8 + j] * w[j];
      w[kNnHid + h] = nnActivate(z);
    }
    for (int o = 0; o < 3; o++) {
      float z = W[kNnB2 + o];
      for (int h = 0; h < kNnHidden; h++) z += W[kNnW2 + o * 24 + h] * w[kNnHid + h];
      w[kNnOut + o] = z;
    }
  }
  __syncthreads();
  // score on the 8 held-out samples and the validation gate (learning.cu:30-41)
  if (i == 0) {
    float err = 0.0f, baseline = 0.0f, n = 0.0f;
    for (int k = kNnTrain; k < kNnBatch; k++) {
      const float* w = work + k * kNnWs;
      if (w[kNnValid] > 0.5f) {
        n += 1.0f;
        const f3 mean = substrateMean(int(w[kNnMat]));
        for (int o = 0; o < 3; o++) {
          const float d = w[kNnOut + o] - w[kNnTarget + o];
          err += d * d;
          const float m = o == 0 ? mean.x : (o == 1 ? mean.y : mean.z);
          const float e = m - w[kNnTarget + o];
          baseline += e * e;
        }
      }
    }
    if (n > 0.0f) {
      const float a = Brain[1] < 1.0f ? 1.0f : 0.065f;
      Brain[2] = lerp(Brain[2], err / (n * 3.0f), a);
      Brain[3] = lerp(Brain[3], baseline / (n * 3.0f), a);
      Brain[1] += n;
    }
    Brain[4] = Brain[1] >= 256.0f && Brain[2] < Brain[3] * 0.90f && Brain[2] < 0.0012f ? 1.0f : 0.0f;
  }
  // gradient over the 56 training samples (learning.cu:42-52)
  if (i < kNnParams) {
    float g = 0.0f, count = 0.0f;
    for (int k = 0; k < kNnTrain; k++) {
      const float* w = work + k * kNnWs;
      if (w[kNnValid] > 0.5f) {
        count += 1.0f;
        if (i < kNnW2) {
          const int h = i < kNnB1 ? i / 8 : i - kNnB1;
          float d = 0.0f;
          for (int o = 0; o < 3; o++) d += (w[kNnOut + o] - w[kNnTarget + o]) * W[kNnW2 + o * 24 + h];
          const float a = w[kNnHid + h];
          d *= 1.0f - a * a;
          g += i < kNnB1 ? d * w[i % 8] : d;
        } else if (i < kNnB2) {
          const int o = (i - kNnW2) / 24, h = (i - kNnW2) % 24;
          g += (w[kNnOut + o] - w[kNnTarget + o]) * w[kNnHid + h];
        } else {
          const int o = i - kNnB2;
          g += w[kNnOut + o] - w[kNnTarget + o];
        }
      }
    }
    grad[i] = clampv(g / fmaxf(1.0f, count), -0.8f, 0.8f);
    if (i == 0) {
      if (count > 0.0f) Brain[0] += 1.0f;
      Brain[5] = count;
    }
  }
  __syncthreads();
  // Adam (learning.cu:53-58)
  if (i < kNnParams && Brain[5] >= 1.0f) {
    const float g = grad[i];
    const float m = 0.9f * M[i] + 0.1f * g, v = 0.999f * V[i] + 0.001f * g * g;
    M[i] = m;
    V[i] = v;
    const float mh = m / (1.0f - powR(0.9f, Brain[0])), vh = v / (1.0f - powR(0.999f, Brain[0]));
    W[i] -= 0.002f * (mh / (sqrtf(vh) + 0.00001f) + 0.0001f * W[i]);
  }
  if (WorkOut)
    for (int k = i; k < kNnBatch * kNnWs; k += kStepThreads) WorkOut[k] = work[k];
}

// The surrogate's colour for n queries [u, v, seed, material].
__global__ void predictSubstrateK(const float* __restrict__ W, const float* __restrict__ Q, int n, float* Out) {
  const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float* q = Q + size_t(i) * 4;
  const f3 c = predictSubstrate(W, q[0], q[1], q[2], int(q[3]));
  Out[size_t(i) * 3] = c.x; Out[size_t(i) * 3 + 1] = c.y; Out[size_t(i) * 3 + 2] = c.z;
}

// shadePixels with the surrogate in place of the procedural substrate of
// brick and stone when C[16] enables it and the gate Brain[4] is open
// (Stratum.cu:854); otherwise exactly the drop-in shadePixels.
__global__ void __launch_bounds__(64) shadePixelsNeuralK(const float* __restrict__ World, const uint32_t* __restrict__ O,
                                                        const float* __restrict__ C, const float* __restrict__ Hit,
                                                        const float* __restrict__ Surface, float* Linear,
                                                        const float* __restrict__ W, const float* __restrict__ Brain,
                                                        int width, int height, int rowStart, int rowCount) {
  __shared__ FrameConst F;
  __shared__ int useNet;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    F = makeFrame(C, O);
    useNet = C[16] > 0.5f && Brain[4] > 0.5f;
  }
  __syncthreads();
  const int x = int(blockIdx.x * blockDim.x + threadIdx.x), y = rowStart + int(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= width || y >= height || y >= rowStart + rowCount) return;
  const size_t b = size_t(y) * width + x;
  const f3 rd = primaryDir(F.cam, x, y, width, height);
  const float4 h = reinterpret_cast<const float4*>(Hit)[b], s = reinterpret_cast<const float4*>(Surface)[b];
  f3 c;
  if (int(h.y) == kSkyId) {
    c = skyColor(rd, F.sun);
  } else {
    SurfacePoint sp;
    surfacePoint(World, F, h, s, rd, height, sp);
    f3 base = substrateMean(sp.mat);
    if (sp.mat == 0 || sp.mat == 1)
      base = useNet ? predictSubstrate(W, sp.u, sp.v, sp.seed, sp.mat) : substrate(sp.u, sp.v, sp.seed, sp.mat);
    const f3 albedo = surfaceColor(sp.q, sp.qn, sp.mat, sp.seed, sp.sfp, base) * paletteTint(sp.palette, sp.mat);
    c = pixelLight(World, F, sp, rd, int(h.y), albedo);
  }
  reinterpret_cast<float4*>(Linear)[b] = make_float4(c.x, c.y, c.z, 1.0f);
}

}  // namespace st

using namespace st;

extern "C" {

int stratum_initNeural(float* W, float* M, float* V, float* Brain, int seed, stratum_stream_t stream) {
  if (!W || !M || !V || !Brain) return STRATUM_EINVAL;
  initNeuralK<<<2, 256, 0, asStream(stream)>>>(W, M, V, Brain, seed);
  return launchStatus();
}

int stratum_materialStep(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                         const float* Surface, float* W, float* M, float* V, float* Brain, float* Work, int width,
                         int height, stratum_stream_t stream) {
  if (!World || !Origin || !C || !Hit || !Surface || !W || !M || !V || !Brain || !frameOk(width, height))
    return STRATUM_EINVAL;
  materialStepK<<<1, kStepThreads, 0, asStream(stream)>>>(World, Origin, C, Hit, Surface, W, M, V, Brain, Work,
                                                          width, height);
  return launchStatus();
}

int stratum_predictSubstrate(const float* W, const float* Queries, int n, float* Out, stratum_stream_t stream) {
  if (!W || !Queries || !Out || n < 0) return STRATUM_EINVAL;
  if (n == 0) return STRATUM_OK;
  predictSubstrateK<<<(n + 127) / 128, 128, 0, asStream(stream)>>>(W, Queries, n, Out);
  return launchStatus();
}

int stratum_shadePixelsNeural(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                              const float* Surface, float* Linear, const float* W, const float* Brain, int width,
                              int height, int rowStart, int rowCount, stratum_stream_t stream) {
  if (!World || !Origin || !C || !Hit || !Surface || !Linear || !W || !Brain || !frameOk(width, height))
    return STRATUM_EINVAL;
  if (rowStart < 0 || rowCount < 0) return STRATUM_EINVAL;
  const int rows = rowCount < height - rowStart ? rowCount : height - rowStart;
  if (rows <= 0) return STRATUM_OK;
  dim3 grid((width + 7) / 8, (rows + 7) / 8);
  shadePixelsNeuralK<<<grid, dim3(8, 8), 0, asStream(stream)>>>(World, Origin, C, Hit, Surface, Linear, W, Brain,
                                                              width, height, rowStart, rowCount);
  return launchStatus();
}

}  // extern "C"
