// Build-time generator for the grammar's trigonometric constants.
//
// The feature grammar evaluates cosf/sinf at only 40 distinct arguments:
//   j * 2.4f        for j in [0, 28)   (park tree foliage, assets.cu:25-27)
//   j * PI * 0.5f   for j in [0, 4)    (tower pinnacles, assets.cu:77)
//   k * PI * 0.25f  for k in [0, 8)    (roof antenna ring, assets.cu:247-248)
// The reference computes them with the host C library (its CPU harness), so
// this program evaluates them once with the same library and writes a header
// of exact hex-float literals.  Device code then reads the table and never
// evaluates a trigonometric function for feature placement.
#include <cmath>
#include <cstdio>

static float host_cos(float a) { volatile float v = a; return std::cos(static_cast<float>(v)); }
static float host_sin(float a) { volatile float v = a; return std::sin(static_cast<float>(v)); }

static void table(const char* name, int n, float (*arg)(int)) {
  std::printf("static __constant__ float %sCos[%d] = {", name, n);
  for (int i = 0; i < n; i++) std::printf("%s%a", i ? ", " : "", host_cos(arg(i)));
  std::printf("};\n");
  std::printf("static __constant__ float %sSin[%d] = {", name, n);
  for (int i = 0; i < n; i++) std::printf("%s%a", i ? ", " : "", host_sin(arg(i)));
  std::printf("};\n");
}

int main() {
  const float pi = 3.141592653589793f;
  std::printf("// Generated by gen_tables.cpp at build time. Do not edit.\n#pragma once\n");
  table("kTree", 28, [](int j) { return float(j) * 2.4f; });
  table("kQuarter", 4, [](int j) { return float(j) * 3.141592653589793f * 0.5f; });
  table("kEighth", 8, [](int k) { return float(k) * 3.141592653589793f * 0.25f; });
  (void)pi;
  return 0;
}
