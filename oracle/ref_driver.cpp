// Test infrastructure only.  A ctypes-callable driver around the REFERENCE
// renderer's own kernels (kernels/*.cu of stratum-hyperdetail, regenerated into
// oracle/_ref/src/Stratum.cu by oracle/Makefile), compiled as host C++.
//
// It uses the same trick as the reference's tests/native_harness.cpp:14-26:
// the CUDA qualifiers are defined away, a minimal float2/float3 shim supplies the
// vector types, and thread indices become thread-local globals, so every
// __global__ entry point runs as an ordinary function per (block, thread).
// Nothing here re-implements reference math: each ref_* function only sets the
// launch indices and calls the reference kernel or device function.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#define __device__
#define __global__
#define __shared__
#define __syncthreads() ((void)0)

struct RefIdx { unsigned x = 0, y = 0, z = 0; };
static thread_local RefIdx threadIdx, blockIdx, blockDim, gridDim;

struct float2 { float x, y; };
struct float3 { float x, y, z; };
static inline float2 make_float2(float x, float y) { return {x, y}; }
static inline float3 make_float3(float x, float y, float z) { return {x, y, z}; }
static inline float3 operator+(float3 a, float3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline float3 operator-(float3 a, float3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline float3 operator*(float3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline float3 operator*(float s, float3 a) { return {a.x * s, a.y * s, a.z * s}; }
static inline float3 operator*(float3 a, float3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline float3 operator/(float3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline unsigned int atomicAdd(unsigned int* p, unsigned int v) {
  unsigned int old = *p; *p += v; return old;
}

#include "Stratum.cu"

namespace {
void one_thread() { threadIdx = {}; blockIdx = {}; blockDim = {1, 1, 1}; }
void set_pixel(int x, int y) {
  blockDim = {8, 8, 1};
  blockIdx = {unsigned(x / 8), unsigned(y / 8), 0};
  threadIdx = {unsigned(x % 8), unsigned(y % 8), 0};
}
void put_feature(const Feature& f, float* o) {
  o[0] = f.p.x; o[1] = f.p.y; o[2] = f.p.z; o[3] = f.h.x; o[4] = f.h.y; o[5] = f.h.z;
  o[6] = float(f.shape); o[7] = float(f.material); o[8] = float(f.turn); o[9] = f.seed;
}
Feature get_feature(const float* i) {
  Feature f;
  f.p = make_float3(i[0], i[1], i[2]); f.h = make_float3(i[3], i[4], i[5]);
  f.shape = int(i[6]); f.material = int(i[7]); f.turn = int(i[8]); f.seed = i[9];
  return f;
}
int threads(int n) { return n > 0 ? n : omp_get_max_threads(); }
}  // namespace

extern "C" {

void ref_offset_tag(const unsigned* origin, int dx, int dz, unsigned* out) {
  Tag t = offsetTag(origin, dx, dz);
  out[0] = t.xl; out[1] = t.xh; out[2] = t.zl; out[3] = t.zh;
}
unsigned ref_tag_hash(const unsigned* tag, int seed) {
  Tag t{tag[0], tag[1], tag[2], tag[3]};
  return tagHash(t, seed);
}
unsigned ref_hashU(unsigned x) { return hashU(x); }

// Lot descriptor in the World slot layout (world.cu:100-102), 16 floats.
void ref_describe_lot(const unsigned* tag, int seed, float* out) {
  Tag t{tag[0], tag[1], tag[2], tag[3]};
  Lot l = describeLot(t, seed);
  float v[16] = {l.w, l.d, l.h, float(l.type), float(l.mat), float(l.floors), l.seed, l.storey,
                 l.roofScale, float(l.turn), l.ox, l.oz, l.palette, 0.f, 0.f, 1.f};
  std::memcpy(out, v, sizeof v);
}

void ref_initCamera(float* C, unsigned* Origin, int seed) { one_thread(); initCamera(C, Origin, seed); }
void ref_stepCamera(float* C, unsigned* Origin, const float* I, float dt, int w, int h) {
  one_thread(); stepCamera(C, Origin, I, dt, w, h);
}
void ref_clearQueue(unsigned* Queue) { one_thread(); clearQueue(Queue); }
// Serial over all 16,384 slots, so the queue order is the slot order.
void ref_prepareLots(const unsigned* Origin, const float* C, float* World, unsigned* Tags, unsigned* Queue) {
  for (int i = 0; i < WORLD_LOTS; i++) {
    blockDim = {64, 1, 1}; blockIdx = {unsigned(i / 64), 0, 0}; threadIdx = {unsigned(i % 64), 0, 0};
    prepareLots(Origin, C, World, Tags, Queue);
  }
}
void ref_planBounds(const unsigned* Queue, unsigned* Args) {
  for (int c = 0; c < BUILD_CHUNKS; c++) {
    blockDim = {8, 1, 1}; blockIdx = {0, 0, 0}; threadIdx = {unsigned(c), 0, 0};
    planBounds(Queue, Args);
  }
}
// buildGroupBounds + reduceGroupBounds(first=32..1) for every queued lot, in
// the chunk order of src/engine.js:71 (lots are independent, so they run in
// parallel; within a lot the level order is kept).
void ref_buildBounds(const unsigned* Queue, const float* World, float* Nodes, int nthreads) {
  const int count = int(Queue[0]);
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads(nthreads))
  for (int q = 0; q < count; q++) {
    const int base = (q / BUILD_CHUNK) * BUILD_CHUNK, local = q - base;
    for (int g = 0; g < CLUSTERS; g++) {
      blockDim = {64, 1, 1}; blockIdx = {unsigned(local), 0, 0}; threadIdx = {unsigned(g), 0, 0};
      buildGroupBounds(Queue, World, Nodes, base);
    }
    for (int first = 32; first >= 1; first /= 2) {
      for (int j = 0; j < first; j++) {
        int i = local * first + j;
        blockDim = {64, 1, 1}; blockIdx = {unsigned(i / 64), 0, 0}; threadIdx = {unsigned(i % 64), 0, 0};
        reduceGroupBounds(Queue, Nodes, first, base);
      }
    }
  }
}
void ref_tracePrimary(const float* World, const float* Nodes, const unsigned* Origin, const float* C,
                      float* Hit, float* Surface, int width, int height, int rowStart, int rowCount,
                      int nthreads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads(nthreads))
  for (int y = rowStart; y < rowStart + rowCount; y++)
    for (int x = 0; x < width; x++) {
      set_pixel(x, y - rowStart);
      tracePrimary(World, Nodes, Origin, C, Hit, Surface, width, height, rowStart, rowCount);
    }
}
void ref_shadePixels(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                     const float* Surface, float* Linear, int width, int height, int rowStart,
                     int rowCount, int nthreads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads(nthreads))
  for (int y = rowStart; y < rowStart + rowCount; y++)
    for (int x = 0; x < width; x++) {
      set_pixel(x, y - rowStart);
      shadePixels(World, Origin, C, Hit, Surface, Linear, width, height, rowStart, rowCount);
    }
}
void ref_resolveFrame(const float* Linear, float* History, unsigned* Pixels, const float* C,
                      const float* Hit, const float* Surface, int width, int height, int nthreads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads(nthreads))
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) {
      set_pixel(x, y);
      resolveFrame(Linear, History, Pixels, C, Hit, Surface, width, height);
    }
}
// resolveFrame over rows [rowStart, rowStart+rowCount) only (timing samples).
void ref_resolveRows(const float* Linear, float* History, unsigned* Pixels, const float* C, const float* Hit,
                     const float* Surface, int width, int height, int rowStart, int rowCount, int nthreads) {
  const int yEnd = rowStart + rowCount < height ? rowStart + rowCount : height;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads(nthreads))
  for (int y = rowStart; y < yEnd; y++)
    for (int x = 0; x < width; x++) {
      set_pixel(x, y);
      resolveFrame(Linear, History, Pixels, C, Hit, Surface, width, height);
    }
}
// trace, shade and resolve of the listed rows only (timing samples spread over
// a frame): each pass runs every pixel of those rows, in parallel over pixels;
// a row is the reference's strip of one row (rowStart = y, rowCount = 1).
void ref_renderRows(const float* World, const float* Nodes, const unsigned* Origin, const float* C, float* Hit,
                    float* Surface, float* Linear, float* History, unsigned* Pixels, int width, int height,
                    const int* rows, int nrows, int nthreads) {
  const long n = long(nrows) * width;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads(nthreads))
  for (long i = 0; i < n; i++) {
    const int y = rows[i / width], x = int(i % width);
    set_pixel(x, 0);
    tracePrimary(World, Nodes, Origin, C, Hit, Surface, width, height, y, 1);
  }
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads(nthreads))
  for (long i = 0; i < n; i++) {
    const int y = rows[i / width], x = int(i % width);
    set_pixel(x, 0);
    shadePixels(World, Origin, C, Hit, Surface, Linear, width, height, y, 1);
  }
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads(nthreads))
  for (long i = 0; i < n; i++) {
    const int y = rows[i / width], x = int(i % width);
    set_pixel(x, y);
    resolveFrame(Linear, History, Pixels, C, Hit, Surface, width, height);
  }
}
void ref_probeGrammar(const float* Inputs, float* Output) { one_thread(); probeGrammar(Inputs, Output); }

// Feature records of one group: 10 floats each [p.xyz, h.xyz, shape, material,
// turn, seed], enumerated with sink modes 1 (count) and 2 (pick), as the
// reference harness's enumerate() does (tests/native_harness.cpp:48).
int ref_enumerate(const float* lot16, int group, float* out, int cap) {
  Lot l = readLot(lot16, 0);
  Sink c = newSink(1, make_float3(0, 0, 0), make_float3(0, 0, 1), FAR);
  c = authoredGroup(l, group, c);
  for (int i = 0; i < c.count && i < cap; i++) {
    Sink s = newSink(2, make_float3(0, 0, 0), make_float3(0, 0, 1), FAR);
    s.target = i;
    s = authoredGroup(l, group, s);
    put_feature(s.feature, out + 10 * i);
  }
  return c.count;
}
// Bounds-mode sink of one group: lo.xyz, count, hi.xyz.
void ref_group_bounds(const float* lot16, int group, float* out7) {
  Lot l = readLot(lot16, 0);
  Sink s = newSink(1, make_float3(0, 0, 0), make_float3(0, 0, 1), FAR);
  s = authoredGroup(l, group, s);
  out7[0] = s.lo.x; out7[1] = s.lo.y; out7[2] = s.lo.z; out7[3] = float(s.count);
  out7[4] = s.hi.x; out7[5] = s.hi.y; out7[6] = s.hi.z;
}
float ref_featureHit(const float* f10, const float* ro, const float* rd, float cone) {
  return featureHit(get_feature(f10), make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), cone);
}
void ref_featureNormal(const float* f10, const float* pt, float* n) {
  float3 r = featureNormal(get_feature(f10), make_float3(pt[0], pt[1], pt[2]));
  n[0] = r.x; n[1] = r.y; n[2] = r.z;
}
// queryLot over one lot's 128-node block (slot 0 of `nodes`): t, fid, feature.
float ref_queryLot(const float* lot16, const float* nodes, const float* ro, const float* rd, float best,
                   float cone, int* fid, float* f10) {
  Lot l = readLot(lot16, 0);
  Sink h = queryLot(l, nodes, 0, make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), best, cone);
  *fid = h.fid;
  put_feature(h.feature, f10);
  return h.t;
}
}  // extern "C"
