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
#include <initializer_list>

static float host_cos(float a) { volatile float v = a; return std::cos(static_cast<float>(v)); }
static float host_sin(float a) { volatile float v = a; return std::sin(static_cast<float>(v)); }

// One table per function: a __constant__ copy for the device, a host copy for
// host builds of the same headers, and an accessor that picks the right one.
static void one(const char* name, const char* fn, int n, float (*arg)(int), float (*f)(float)) {
  for (const char* space : {"__constant__", "const"}) {
    std::printf("static %s float %s%s%s[%d] = {", space, name, fn, space[0] == '_' ? "" : "Host", n);
    for (int i = 0; i < n; i++) std::printf("%s%a", i ? ", " : "", f(arg(i)));
    std::printf("};\n");
  }
  std::printf("__host__ __device__ __forceinline__ float %s%s(int i) {\n#ifdef __CUDA_ARCH__\n  return %s%s[i];\n"
              "#else\n  return %s%sHost[i];\n#endif\n}\n", name + 1, fn, name, fn, name, fn);
}
static void table(const char* name, int n, float (*arg)(int)) {
  one(name, "Cos", n, arg, host_cos);
  one(name, "Sin", n, arg, host_sin);
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
