// Device math for the STRATUM frame path (sm_100a).
//
// Restates kernels/common.cu and kernels/world.cu of the reference
// (stratum-hyperdetail) for CUDA.  All files are compiled with --fmad=false,
// so every a*b+c below rounds twice exactly as the reference's CPU build does;
// together with IEEE division and square root (nvcc defaults) this makes the
// integer, addressing, descriptor and feature-record results bit-identical to
// the reference.  Transcendentals that feed only tolerance-checked outputs use
// CUDA's standard (non-intrinsic) functions; the camera basis uses double
// precision rounded to float, which matches a correctly rounded C library.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// HD: pure functions, also compiled for the host (tests check them against the
// oracle on the CPU).  SD: device-only helpers.
#define HD __host__ __device__ __forceinline__
#define SD __device__ __forceinline__

namespace st {

// ---- ABI constants (common.cu:2-16, src/engine.js:2) ------------------------
constexpr float kCell = 36.0f;
constexpr int kSide = 128;
constexpr int kLots = 16384;
constexpr int kLotFloats = 16;
constexpr int kGroups = 64;
constexpr int kNodes = 128;
constexpr int kMaxFeatures = 64;
constexpr int kChunk = 2048;
constexpr int kChunks = 8;
constexpr float kFar = 2000.0f;
constexpr float kTop = 100.0f;
constexpr float kPi = 3.141592653589793f;
// Hit[1] codes
constexpr int kSkyId = -10000;
constexpr int kGroundId = -1;

// ---- vector type ------------------------------------------------------------
struct f3 { float x, y, z; };
HD f3 mk(float x, float y, float z) { return {x, y, z}; }
HD f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
HD f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
HD f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
HD f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
HD f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD float len(f3 a) { return sqrtf(dot(a, a)); }
HD f3 unit(f3 a) { return a / fmaxf(0.000001f, len(a)); }
HD f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
HD f3 mix(f3 a, f3 b, float t) { return a + (b - a) * t; }
HD f3 vmin(f3 a, f3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
HD f3 vmax(f3 a, f3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }

// ---- scalar helpers (common.cu:27-31) ----------------------------------------
HD float clampv(float x, float a, float b) { return fminf(b, fmaxf(a, x)); }
HD float sat(float x) { return clampv(x, 0.0f, 1.0f); }
HD float lerp(float a, float b, float t) { return a + (b - a) * t; }
HD float fract(float x) { return x - floorf(x); }
HD float smooth(float a, float b, float x) {
  float t = sat((x - a) / (b - a));
  return t * t * (3.0f - 2.0f * t);
}
HD int imod(int x, int n) { int r = x % n; return r < 0 ? r + n : r; }

// ---- integer hashing (common.cu:42-44): bit-exact ----------------------------
HD uint32_t mixbits(uint32_t x) {
  x ^= x >> 16; x *= 2146121005u; x ^= x >> 15; x *= 2221713035u; x ^= x >> 16;
  return x;
}
HD float unit24(uint32_t h) { return float(h & 16777215u) / 16777216.0f; }
HD float hash1(int x) { return unit24(mixbits(uint32_t(x))); }
HD float hash2(int x, int y, int seed) {
  return unit24(mixbits(uint32_t(x) * 1973u + uint32_t(y) * 9277u + uint32_t(seed) * 26699u));
}

// ---- value noise (common.cu:45-53) ------------------------------------------
HD float noise2(float x, float y) {
  int ix = int(floorf(x)), iy = int(floorf(y));
  float fx = fract(x), fy = fract(y);
  fx = fx * fx * (3.0f - 2.0f * fx);
  fy = fy * fy * (3.0f - 2.0f * fy);
  float a = lerp(hash2(ix, iy, 13), hash2(ix + 1, iy, 13), fx);
  float b = lerp(hash2(ix, iy + 1, 13), hash2(ix + 1, iy + 1, 13), fx);
  return lerp(a, b, fy);
}
HD float fbm2(float x, float y) {
  float v = 0.0f, amp = 0.5f;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    v += noise2(x, y) * amp;
    x = x * 2.07f + 11.7f;
    y = y * 2.03f - 8.3f;
    amp *= 0.5f;
  }
  return v;
}
HD float freqWeight(float footprint, float freq) { return 1.0f - smooth(0.35f, 1.1f, footprint * freq); }

// ---- camera (common.cu:54-70) -----------------------------------------------
// sin/cos of the camera angles in double, rounded once to float.
HD float sinR(float a) { return float(sin(double(a))); }
HD float cosR(float a) { return float(cos(double(a))); }
struct Camera {
  f3 pos, fwd, right, up;
  float jx, jy;  // Halton jitter of this sample
};
HD float halton(int value, int base) {
  float inv = 1.0f / float(base), place = inv, r = 0.0f;
  for (int j = 0; j < 12 && value > 0; j++) {
    r += float(value % base) * place;
    value /= base;
    place *= inv;
  }
  return r;
}
HD Camera makeCamera(const float* C) {
  Camera c;
  c.pos = mk(C[0], C[1], C[2]);
  float s3 = sinR(C[3]), c3 = cosR(C[3]), s4 = sinR(C[4]), c4 = cosR(C[4]);
  c.fwd = mk(s3 * c4, s4, c3 * c4);
  c.right = mk(c3, 0.0f, -s3);
  c.up = cross(c.fwd, c.right);
  int sample = int(C[19]) - 1;
  c.jx = 0.0f; c.jy = 0.0f;
  if (sample > 0) { c.jx = halton(sample, 2) - 0.5f; c.jy = halton(sample, 3) - 0.5f; }
  return c;
}
HD f3 primaryDir(const Camera& c, int x, int y, int width, int height) {
  float sx = (float(x) + 0.5f + c.jx - float(width) * 0.5f) / float(height) * 1.08f;
  float sy = -(float(y) + 0.5f + c.jy - float(height) * 0.5f) / float(height) * 1.08f;
  return unit(c.fwd + c.right * sx + c.up * sy);
}
HD f3 sunDir(const float* C) {
  float s7 = sinR(C[7]), c7 = cosR(C[7]), s8 = sinR(C[8]), c8 = cosR(C[8]);
  return unit(mk(c7 * c8, s8, s7 * c8));
}

// ---- slab test (common.cu:71-77) --------------------------------------------
HD float guardedInv(float d) {
  return 1.0f / (fabsf(d) > 0.0000001f ? d : (d < 0.0f ? -0.0000001f : 0.0000001f));
}
struct Span { float lo, hi; };
HD Span slabInv(f3 ro, f3 inv, f3 lo, f3 hi) {
  f3 a = mk((lo.x - ro.x) * inv.x, (lo.y - ro.y) * inv.y, (lo.z - ro.z) * inv.z);
  f3 b = mk((hi.x - ro.x) * inv.x, (hi.y - ro.y) * inv.y, (hi.z - ro.z) * inv.z);
  f3 mn = vmin(a, b), mx = vmax(a, b);
  return {fmaxf(fmaxf(mn.x, mn.y), mn.z), fminf(fminf(mx.x, mx.y), mx.z)};
}
HD f3 invDir(f3 rd) { return mk(guardedInv(rd.x), guardedInv(rd.y), guardedInv(rd.z)); }
HD Span slab(f3 ro, f3 rd, f3 lo, f3 hi) { return slabInv(ro, invDir(rd), lo, hi); }

// ---- masonry relief (common.cu:78-87) ---------------------------------------
HD void masonryUV(f3 p, f3 n, float& u, float& v) {
  if (fabsf(n.y) > 0.5f) { u = p.x; v = p.z; }
  else if (fabsf(n.x) > 0.5f) { u = p.z; v = p.y; }
  else { u = p.x; v = p.y; }
}
HD float masonryHeight(float u, float v, int material) {
  float bw = material == 1 ? 0.46f : 0.92f, bh = material == 1 ? 0.215f : 0.46f;
  int row = int(floorf(v / bh));
  float x = fract(u / bw + float(imod(row, 2)) * 0.5f), y = fract(v / bh);
  float edge = fminf(fminf(x, 1.0f - x) * bw, fminf(y, 1.0f - y) * bh);
  float grain = noise2(u * 24.0f, v * 24.0f);
  float chipped = edge - 0.006f * smooth(0.34f, 0.73f, noise2(u * 117.0f, v * 117.0f));
  return -0.018f * (1.0f - smooth(0.008f, 0.023f, chipped)) + 0.0025f * grain;
}
HD uint32_t packRGBA8(f3 c) {
  uint32_t r = uint32_t(sat(c.x) * 255.0f), g = uint32_t(sat(c.y) * 255.0f), b = uint32_t(sat(c.z) * 255.0f);
  return r | (g << 8) | (b << 16) | 4278190080u;
}

// ---- world addressing (world.cu:3-56): bit-exact -----------------------------
struct Addr { uint32_t xl, xh, zl, zh; };
struct LotDesc {
  float w, d, h; int type, mat, floors; float seed, storey, roofScale; int turn; float ox, oz, palette;
};
// 64-bit lot address plus a signed cell offset, carry/borrow per axis.
HD Addr shiftAddr(uint32_t o0, uint32_t o1, uint32_t o2, uint32_t o3, int dx, int dz) {
  Addr a;
  a.xl = o0 + uint32_t(dx); a.xh = o1;
  if (dx >= 0 && a.xl < o0) a.xh++;
  if (dx < 0 && a.xl > o0) a.xh--;
  a.zl = o2 + uint32_t(dz); a.zh = o3;
  if (dz >= 0 && a.zl < o2) a.zh++;
  if (dz < 0 && a.zl > o2) a.zh--;
  return a;
}
HD uint32_t addrKey(Addr a, int seed) {
  return mixbits(a.xl * 1973u + mixbits(a.xh + 719u) + a.zl * 9277u + mixbits(a.zh + 173u) + uint32_t(seed) * 26699u);
}
HD float frac16(uint32_t h) { return float(h & 65535u) / 65536.0f; }
HD LotDesc describe(Addr a, int seed) {
  uint32_t key = addrKey(a, seed);
  Addr district{(a.xl >> 3) | (a.xh << 29), a.xh >> 3, (a.zl >> 3) | (a.zh << 29), a.zh >> 3};
  uint32_t dk = addrKey(district, seed + 47);
  float r = frac16(key), density = frac16(dk);
  LotDesc l;
  l.type = r > 0.94f ? 1 : 0;
  if (r < 0.10f + density * 0.045f) l.type = 3;
  if ((a.xl & 63u) == 28u) l.type = (a.zl & 3u) == 0u ? 4 : 5;
  if ((key & 255u) == 93u) l.type = 2;
  l.floors = 2 + int(float(mixbits(key + 11u) & 65535u) * (1.0f / 65536.0f) * 5.0f);
  if (density > 0.7f && l.floors < 4) l.floors = 4;
  l.storey = 3.2f + 1.15f * float(mixbits(key + 127u) & 65535u) / 65536.0f;
  l.w = 9.4f + 4.3f * float(mixbits(key + 31u) & 65535u) / 65536.0f;
  l.d = 9.0f + 4.7f * float(mixbits(key + 83u) & 65535u) / 65536.0f;
  l.h = 4.2f + float(l.floors) * l.storey;
  if (l.type == 2) { l.floors = 6; l.h = 4.2f + 6.0f * l.storey; }
  l.mat = int((key >> 4) & 1u);
  l.seed = float(mixbits(key + 271u) & 65535u);
  l.turn = int((key >> 6) & 3u);
  l.ox = (float(mixbits(key + 311u) & 65535u) / 65536.0f - 0.5f) * 0.48f;
  l.oz = (float(mixbits(key + 313u) & 65535u) / 65536.0f - 0.5f) * 0.48f;
  if (l.type >= 3) { l.ox = 0.0f; l.oz = 0.0f; l.turn = 0; }
  l.roofScale = 0.85f + 0.4f * float(mixbits(key + 317u) & 65535u) / 65536.0f;
  l.palette = float((dk >> 18) & 7u);
  return l;
}
// 64-byte descriptor = four 128-bit loads.
SD LotDesc loadLot(const float* __restrict__ W, int slot) {
  const float4* s = reinterpret_cast<const float4*>(W + slot * kLotFloats);
  float4 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2), d = __ldg(s + 3);
  LotDesc l;
  l.w = a.x; l.d = a.y; l.h = a.z; l.type = int(a.w);
  l.mat = int(b.x); l.floors = int(b.y); l.seed = b.z; l.storey = b.w;
  l.roofScale = c.x; l.turn = int(c.y); l.ox = c.z; l.oz = c.w;
  l.palette = d.x;
  return l;
}
// Plain loads for buffers the same kernel writes (no read-only cache).
HD LotDesc loadLotRW(const float* W, int slot) {
  const float4* s = reinterpret_cast<const float4*>(W + slot * kLotFloats);
  float4 a = s[0], b = s[1], c = s[2], d = s[3];
  LotDesc l;
  l.w = a.x; l.d = a.y; l.h = a.z; l.type = int(a.w);
  l.mat = int(b.x); l.floors = int(b.y); l.seed = b.z; l.storey = b.w;
  l.roofScale = c.x; l.turn = int(c.y); l.ox = c.z; l.oz = c.w;
  l.palette = d.x;
  return l;
}
HD int tableSlot(uint32_t o0, uint32_t o2, int dx, int dz) {
  int x = int((o0 + uint32_t(dx)) & 127u), z = int((o2 + uint32_t(dz)) & 127u);
  return z * kSide + x;
}
HD void slotCell(uint32_t o0, uint32_t o2, int slot, int& cx, int& cz) {
  cx = imod(slot % kSide - int(o0 & 127u) + kSide / 2, kSide) - kSide / 2;
  cz = imod(slot / kSide - int(o2 & 127u) + kSide / 2, kSide) - kSide / 2;
}
HD f3 toLot(f3 p, int turn) {
  if (turn == 1) return mk(p.z, p.y, -p.x);
  if (turn == 2) return mk(-p.x, p.y, -p.z);
  if (turn == 3) return mk(-p.z, p.y, p.x);
  return p;
}
HD f3 fromLot(f3 p, int turn) { return toLot(p, (4 - turn) % 4); }

}  // namespace st
