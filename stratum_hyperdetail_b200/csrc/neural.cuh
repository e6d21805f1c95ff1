// The optional online material surrogate (kernels/learning.cu of the
// reference): an 8 -> 24 tanh -> 3 linear network (291 parameters) that learns
// the substrate colour of brick and stone (materials 0 and 1) from the frame's
// own hit pixels, trained with Adam every fourth frame on 56 samples and scored
// on 8 held-out ones; shading uses it in place of the procedural substrate only
// when enabled (C[16]) and its validation gate is open (Brain[4]).  The
// reference keeps this file out of its build; it is carried here with its
// inputs taken from the current frame buffers (Hit material and seed, Surface
// normal and slot, the lot-frame masonry coordinates the shading uses).
//
// Its sines, cosines, exponentials and powers are evaluated in double
// precision and rounded once to float.
#pragma once
#include "shading.cuh"

namespace st {

constexpr int kNnInputs = 8, kNnHidden = 24, kNnParams = 291, kNnBatch = 64, kNnWs = 64, kNnTrain = 56;
// parameter layout: input weights [h*8 + j] (0..191), hidden biases (192..215),
// output weights [216 + o*24 + h] (216..287), output biases (288..290)
constexpr int kNnB1 = 192, kNnW2 = 216, kNnB2 = 288;
// a sample's row of the work area: features 0..7, target 8..10, output 11..13,
// hidden 14..37, valid flag 62, material 63
constexpr int kNnTarget = 8, kNnOut = 11, kNnHid = 14, kNnValid = 62, kNnMat = 63;

HD float expR(float x) { return float(exp(double(x))); }
HD float powR(float x, float y) { return float(pow(double(x), double(y))); }

// learning.cu:4: training runs on frames whose counter C[6] is a multiple of 4,
// unless frozen by C[21].
HD bool materialTrainNow(const float* C) { return (int(C[6]) % 4) == 0 && C[21] < 0.5f; }

// The network's inputs (the reference's feature(), Stratum.cu:648-657).
SD float nnFeature(int i, float u, float v, float seed, int mat) {
  if (i == 0) return sinR(u * 0.13f);
  if (i == 1) return cosR(u * 0.13f);
  if (i == 2) return sinR(v * 0.13f);
  if (i == 3) return cosR(v * 0.13f);
  if (i == 4) return noise2D(u * 0.31f + seed * 0.013f, v * 0.31f) * 2.0f - 1.0f;
  if (i == 5) return noise2D(u * 0.42f + seed * 0.01f, v * 0.038f + 1.7f) * 2.0f - 1.0f;
  if (i == 6) return float(mat) * 2.0f - 1.0f;
  return sinR(seed * 0.03f);
}
// tanh by its logistic form, clamped (Stratum.cu:658)
SD float nnActivate(float x) {
  x = clampv(x, -8.0f, 8.0f);
  return 2.0f / (1.0f + expR(-2.0f * x)) - 1.0f;
}
// Surrogate substrate colour (Stratum.cu:659-664).
SD f3 predictSubstrate(const float* __restrict__ W, float u, float v, float seed, int mat) {
  float in[kNnInputs];
  for (int j = 0; j < kNnInputs; j++) in[j] = nnFeature(j, u, v, seed, mat);
  f3 out = mk(W[kNnB2], W[kNnB2 + 1], W[kNnB2 + 2]);
  for (int h = 0; h < kNnHidden; h++) {
    float z = W[kNnB1 + h];
    for (int j = 0; j < kNnInputs; j++) z += W[h * 8 + j] * in[j];
    const float a = nnActivate(z);
    out.x += W[kNnW2 + h] * a;
    out.y += W[kNnW2 + 24 + h] * a;
    out.z += W[kNnW2 + 48 + h] * a;
  }
  return mk(sat(out.x), sat(out.y), sat(out.z));
}

}  // namespace st
