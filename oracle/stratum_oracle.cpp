// Test infrastructure only: the CPU oracle for the STRATUM frame path.
//
// A plain C++ restatement of the reference's algorithm (stratum-hyperdetail,
// kernels/*.cu), written for checking, not for speed.  Every function names the
// reference lines it restates.  Built without FMA contraction (oracle/Makefile),
// it reproduces the reference's float results bit for bit; this is pinned by
// tests/test_oracle_pin.py against the reference compiled from its own sources
// and against the reference's golden fixtures (tests/probes.json).
//
// The geometry is templated on the scalar type: Real=float is the restatement,
// Real=double is the FP64 re-intersection of a given feature used to bound the
// error of the GPU's distances and normals.
#include "stratum_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace orc {

// ---- ABI constants (common.cu:2-16) --------------------------------------
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

// ---- small vector type ----------------------------------------------------
template <class R> struct V3 { R x, y, z; };
using V3f = V3<float>;
template <class R> inline V3<R> mk(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R len(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> unit(V3<R> a) { return a / std::fmax(R(0.000001f), len(a)); }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline V3<R> mix(V3<R> a, V3<R> b, R t) { return a + (b - a) * t; }
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
template <class R> inline V3<R> cast3(V3f a) { return {R(a.x), R(a.y), R(a.z)}; }

// ---- scalar helpers (common.cu:27-44) --------------------------------------
template <class R> inline R clampv(R x, R a, R b) { return std::fmin(b, std::fmax(a, x)); }
template <class R> inline R sat(R x) { return clampv(x, R(0), R(1)); }
template <class R> inline R lerp(R a, R b, R t) { return a + (b - a) * t; }
template <class R> inline R fract(R x) { return x - std::floor(x); }
template <class R> inline R smooth(R a, R b, R x) {
  R t = sat((x - a) / (b - a));
  return t * t * (R(3) - R(2) * t);
}
inline int imod(int x, int n) { int r = x % n; return r < 0 ? r + n : r; }

inline uint32_t mixbits(uint32_t x) {  // hashU, common.cu:42
  x ^= x >> 16; x *= 2146121005u; x ^= x >> 15; x *= 2221713035u; x ^= x >> 16;
  return x;
}
inline float unit24(uint32_t h) { return float(h & 16777215u) / 16777216.0f; }
inline float hash1(int x) { return unit24(mixbits(uint32_t(x))); }  // common.cu:43
inline float hash2(int x, int y, int seed) {                             // common.cu:44
  return unit24(mixbits(uint32_t(x) * 1973u + uint32_t(y) * 9277u + uint32_t(seed) * 26699u));
}
// value noise and 5-octave fbm (common.cu:45-52)
template <class R> R noise2(R x, R y) {
  int ix = int(std::floor(x)), iy = int(std::floor(y));
  R fx = fract(x), fy = fract(y);
  fx = fx * fx * (R(3) - R(2) * fx);
  fy = fy * fy * (R(3) - R(2) * fy);
  R a = lerp(R(hash2(ix, iy, 13)), R(hash2(ix + 1, iy, 13)), fx);
  R b = lerp(R(hash2(ix, iy + 1, 13)), R(hash2(ix + 1, iy + 1, 13)), fx);
  return lerp(a, b, fy);
}
template <class R> R fbm2(R x, R y) {
  R v = 0, amp = R(0.5f);
  for (int i = 0; i < 5; i++) {
    v += noise2(x, y) * amp;
    x = x * R(2.07f) + R(11.7f);
    y = y * R(2.03f) - R(8.3f);
    amp *= R(0.5f);
  }
  return v;
}
template <class R> inline R freqWeight(R footprint, R freq) { return R(1) - smooth(R(0.35f), R(1.1f), footprint * freq); }

// Sines and cosines of the camera and sun angles and of the resolve taps.
// Mode 0 (default): the C library's float functions, as the reference's CPU
// build calls them.  Mode 1: evaluated in double precision and rounded once to
// float, as the CUDA path does; the C library's float functions are not always
// correctly rounded (about 1.3 % of angles in [0, 2pi) differ by one ulp here),
// so this mode gives the same ray basis as the device for every angle.
int gAngleMode = 0;
inline float angSin(float a) { return gAngleMode ? float(std::sin(double(a))) : std::sin(a); }
inline float angCos(float a) { return gAngleMode ? float(std::cos(double(a))) : std::cos(a); }
// The material surrogate's exponentials and powers follow the same switch.
inline float angExp(float x) { return gAngleMode ? float(std::exp(double(x))) : std::exp(x); }
inline float angPow(float x, float y) { return gAngleMode ? float(std::pow(double(x), double(y))) : std::pow(x, y); }

// camera basis and rays (common.cu:54-70)
inline V3f camForward(const float* C) {
  return mk(angSin(C[3]) * angCos(C[4]), angSin(C[4]), angCos(C[3]) * angCos(C[4]));
}
inline V3f camRight(const float* C) { return mk(angCos(C[3]), 0.0f, -angSin(C[3])); }
inline V3f camPos(const float* C) { return mk(C[0], C[1], C[2]); }
inline V3f sunDir(const float* C) {
  return unit(mk(angCos(C[7]) * angCos(C[8]), angSin(C[8]), angSin(C[7]) * angCos(C[8])));
}
inline float halton(int value, int base) {
  float inv = 1.0f / float(base), place = inv, r = 0.0f;
  for (int j = 0; j < 12 && value > 0; j++) {
    r += float(value % base) * place;
    value /= base;
    place *= inv;
  }
  return r;
}
inline V3f primaryDir(const float* C, int x, int y, int width, int height) {
  int sample = int(C[19]) - 1;
  float jx = 0.0f, jy = 0.0f;
  if (sample > 0) { jx = halton(sample, 2) - 0.5f; jy = halton(sample, 3) - 0.5f; }
  float sx = (float(x) + 0.5f + jx - float(width) * 0.5f) / float(height) * 1.08f;
  float sy = -(float(y) + 0.5f + jy - float(height) * 0.5f) / float(height) * 1.08f;
  V3f f = camForward(C), r = camRight(C), u = cross(f, r);
  return unit(f + r * sx + u * sy);
}
// guarded reciprocal and slab test (common.cu:71-77)
template <class R> inline R guardedInv(R d) {
  return R(1) / (std::fabs(d) > R(0.0000001f) ? d : (d < R(0) ? R(-0.0000001f) : R(0.0000001f)));
}
template <class R> struct Span { R lo, hi; };
template <class R> inline Span<R> slab(V3<R> ro, V3<R> rd, V3<R> lo, V3<R> hi) {
  R ix = guardedInv(rd.x), iy = guardedInv(rd.y), iz = guardedInv(rd.z);
  V3<R> a = mk((lo.x - ro.x) * ix, (lo.y - ro.y) * iy, (lo.z - ro.z) * iz);
  V3<R> b = mk((hi.x - ro.x) * ix, (hi.y - ro.y) * iy, (hi.z - ro.z) * iz);
  V3<R> mn = vmin(a, b), mx = vmax(a, b);
  return {std::fmax(std::fmax(mn.x, mn.y), mn.z), std::fmin(std::fmin(mx.x, mx.y), mx.z)};
}
// masonry relief height field (common.cu:78-87)
template <class R> inline void masonryUV(V3<R> p, V3<R> n, R& u, R& v) {
  if (std::fabs(n.y) > R(0.5f)) { u = p.x; v = p.z; }
  else if (std::fabs(n.x) > R(0.5f)) { u = p.z; v = p.y; }
  else { u = p.x; v = p.y; }
}
template <class R> R masonryHeight(R u, R v, int material) {
  R bw = material == 1 ? R(0.46f) : R(0.92f), bh = material == 1 ? R(0.215f) : R(0.46f);
  int row = int(std::floor(v / bh));
  R x = fract(u / bw + R(imod(row, 2)) * R(0.5f)), y = fract(v / bh);
  R edge = std::fmin(std::fmin(x, R(1) - x) * bw, std::fmin(y, R(1) - y) * bh);
  R grain = noise2(u * R(24), v * R(24));
  R chipped = edge - R(0.006f) * smooth(R(0.34f), R(0.73f), noise2(u * R(117), v * R(117)));
  return R(-0.018f) * (R(1) - smooth(R(0.008f), R(0.023f), chipped)) + R(0.0025f) * grain;
}
inline uint32_t packRGBA8(V3f c) {
  uint32_t r = uint32_t(sat(c.x) * 255.0f), g = uint32_t(sat(c.y) * 255.0f), b = uint32_t(sat(c.z) * 255.0f);
  return r | (g << 8) | (b << 16) | 4278190080u;
}

// ---- world addressing (world.cu:3-56) --------------------------------------
struct Addr { uint32_t xl, xh, zl, zh; };
struct LotDesc {
  float w, d, h; int type, mat, floors; float seed, storey, roofScale; int turn; float ox, oz, palette;
};
// 64-bit (two-word) lot address plus a signed offset per axis (world.cu:3-9)
inline Addr shiftAddr(const uint32_t* o, int dx, int dz) {
  Addr a;
  a.xl = o[0] + uint32_t(dx); a.xh = o[1];
  if (dx >= 0 && a.xl < o[0]) a.xh++;
  if (dx < 0 && a.xl > o[0]) a.xh--;
  a.zl = o[2] + uint32_t(dz); a.zh = o[3];
  if (dz >= 0 && a.zl < o[2]) a.zh++;
  if (dz < 0 && a.zl > o[2]) a.zh--;
  return a;
}
inline uint32_t addrKey(Addr a, int seed) {  // world.cu:10-12
  return mixbits(a.xl * 1973u + mixbits(a.xh + 719u) + a.zl * 9277u + mixbits(a.zh + 173u) + uint32_t(seed) * 26699u);
}
inline float frac16(uint32_t h) { return float(h & 65535u) / 65536.0f; }
LotDesc describe(Addr a, int seed) {  // world.cu:13-36
  uint32_t key = addrKey(a, seed);
  Addr district{(a.xl >> 3) | (a.xh << 29), a.xh >> 3, (a.zl >> 3) | (a.zh << 29), a.zh >> 3};
  uint32_t dk = addrKey(district, seed + 47);
  float r = frac16(key), density = frac16(dk);
  LotDesc l;
  l.type = r > 0.94f ? 1 : 0;
  if (r < 0.10f + density * 0.045f) l.type = 3;
  if ((a.xl & 63u) == 28u) l.type = (a.zl & 3u) == 0u ? 4 : 5;  // canal column, bridge every 4th
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
inline void storeLot(const LotDesc& l, float* o) {
  float v[16] = {l.w, l.d, l.h, float(l.type), float(l.mat), float(l.floors), l.seed, l.storey,
                 l.roofScale, float(l.turn), l.ox, l.oz, l.palette, 0.0f, 0.0f, 1.0f};
  std::memcpy(o, v, sizeof v);
}
inline LotDesc loadLot(const float* W, int slot) {  // world.cu:37-41
  const float* s = W + slot * kLotFloats;
  LotDesc l;
  l.w = s[0]; l.d = s[1]; l.h = s[2]; l.type = int(s[3]); l.mat = int(s[4]); l.floors = int(s[5]);
  l.seed = s[6]; l.storey = s[7]; l.roofScale = s[8]; l.turn = int(s[9]); l.ox = s[10]; l.oz = s[11];
  l.palette = s[12];
  return l;
}
inline int tableSlot(const uint32_t* o, int dx, int dz) {  // world.cu:42-45
  int x = int((o[0] + uint32_t(dx)) & 127u), z = int((o[2] + uint32_t(dz)) & 127u);
  return z * kSide + x;
}
inline void slotCell(const uint32_t* o, int slot, int& cx, int& cz) {  // world.cu:46-50
  cx = imod(slot % kSide - int(o[0] & 127u) + kSide / 2, kSide) - kSide / 2;
  cz = imod(slot / kSide - int(o[2] & 127u) + kSide / 2, kSide) - kSide / 2;
}
template <class R> inline V3<R> toLot(V3<R> p, int turn) {  // world.cu:51-55
  if (turn == 1) return mk(p.z, p.y, -p.x);
  if (turn == 2) return mk(-p.x, p.y, -p.z);
  if (turn == 3) return mk(-p.z, p.y, p.x);
  return p;
}
template <class R> inline V3<R> fromLot(V3<R> p, int turn) { return toLot(p, (4 - turn) % 4); }

// ---- features and emission (common.cu:24, sink.cu) -------------------------
struct Feat { V3f p, h; int shape, material, turn; float seed; };

inline void putFeat(const Feat& f, float* o) {
  o[0] = f.p.x; o[1] = f.p.y; o[2] = f.p.z; o[3] = f.h.x; o[4] = f.h.y; o[5] = f.h.z;
  o[6] = float(f.shape); o[7] = float(f.material); o[8] = float(f.turn); o[9] = f.seed;
}
inline Feat getFeat(const float* i) {
  Feat f;
  f.p = mk(i[0], i[1], i[2]); f.h = mk(i[3], i[4], i[5]);
  f.shape = int(i[6]); f.material = int(i[7]); f.turn = int(i[8]); f.seed = i[9];
  return f;
}

struct Counters { int64_t v[ORC_COUNTERS] = {}; };

// ---- analytic intersection (geometry.cu) -----------------------------------
template <class R> inline V3<R> intoFeature(V3<R> p, int turn) { return (turn % 2 == 1) ? mk(p.z, p.y, -p.x) : p; }
template <class R> inline V3<R> outOfFeature(V3<R> p, int turn) { return (turn % 2 == 1) ? mk(-p.z, p.y, p.x) : p; }

template <class R> V3<R> leafNormal(int x, int y, int z, int seed) {  // geometry.cu:6-8
  return unit(mk(R(hash2(x + y * 19, z, seed)) - R(0.5f), R(0.25f) + R(hash2(x - y, z + 91, seed)) * R(0.7f),
                 R(hash2(z + y * 31, x, seed + 17)) - R(0.5f)));
}
// leaf discs in a 0.18 m grid inside the foliage envelope (geometry.cu:9-31)
template <class R> R foliage(V3<R> ro, V3<R> rd, V3<R> centre, V3<R> radius, int seed, R begin, R end, Counters* cn) {
  const R cell = R(0.18f);
  R t = std::fmax(R(0.001f), begin) + R(0.0001f);
  V3<R> pos = ro + rd * t;
  int ix = int(std::floor(pos.x / cell)), iy = int(std::floor(pos.y / cell)), iz = int(std::floor(pos.z / cell));
  int sx = rd.x > R(0) ? 1 : -1, sy = rd.y > R(0) ? 1 : -1, sz = rd.z > R(0) ? 1 : -1;
  R tx = (R(ix + (sx > 0 ? 1 : 0)) * cell - ro.x) * guardedInv(rd.x);
  R ty = (R(iy + (sy > 0 ? 1 : 0)) * cell - ro.y) * guardedInv(rd.y);
  R tz = (R(iz + (sz > 0 ? 1 : 0)) * cell - ro.z) * guardedInv(rd.z);
  R dx = cell * std::fabs(guardedInv(rd.x)), dy = cell * std::fabs(guardedInv(rd.y)), dz = cell * std::fabs(guardedInv(rd.z));
  for (int k = 0; k < 48; k++) {
    if (t > end) break;
    if (cn) cn->v[ORC_FOLIAGE]++;
    R exitT = std::fmin(tx, std::fmin(ty, tz));
    V3<R> c = mk((R(ix) + R(0.5f)) * cell, (R(iy) + R(0.5f)) * cell, (R(iz) + R(0.5f)) * cell);
    V3<R> q = c - centre;
    R ell = q.x * q.x / (radius.x * radius.x) + q.y * q.y / (radius.y * radius.y) + q.z * q.z / (radius.z * radius.z);
    if (ell < R(1) && hash2(ix + iy * 113, iz, seed) > 0.20f) {
      V3<R> n = leafNormal<R>(ix, iy, iz, seed);
      R den = dot(rd, n);
      if (std::fabs(den) > R(0.00001f)) {
        R u = dot(c - ro, n) / den;
        if (u >= t && u <= exitT) {
          V3<R> pp = ro + rd * u - c;
          V3<R> tangent = unit(cross(n, mk(R(0), R(0), R(1))));
          V3<R> bitangent = cross(n, tangent);
          R a = dot(pp, tangent) / R(0.125f), b = dot(pp, bitangent) / R(0.062f);
          if (a * a + b * b < R(1)) return u;
        }
      }
    }
    if (tx < ty && tx < tz) { t = tx; tx += dx; ix += sx; }
    else if (ty < tz) { t = ty; ty += dy; iy += sy; }
    else { t = tz; tz += dz; iz += sz; }
  }
  return R(kFar);
}

// nearest positive hit of one feature, FAR if none (geometry.cu:33-91)
template <class R> R hitFeature(const Feat& f, V3<R> ro, V3<R> rd, R cone, Counters* cn) {
  if (cn) cn->v[ORC_FEAT]++;
  const int shape = f.shape;
  if (shape < 0) return R(kFar);
  const V3<R> cp = cast3<R>(f.p), h = cast3<R>(f.h);
  const int turn = f.turn;
  const V3<R> p = intoFeature(ro - cp, turn), d = intoFeature(rd, turn);
  Span<R> range = slab(p, d, h * R(-1), h);
  if (shape == 3 || shape == 4) range = slab(p, d, mk(-h.x, R(0), -h.z), h);
  if (range.hi < std::fmax(R(0.001f), range.lo)) return R(kFar);
  if (cn) cn->v[shape == 0 ? ORC_PASS_BOX : shape == 1 ? ORC_PASS_ELLIPSOID : shape == 2 ? ORC_PASS_CYLINDER
                : shape == 3 ? ORC_PASS_PRISM : ORC_PASS_ARCH]++;
  R t = range.lo > R(0.001f) ? range.lo : range.hi;
  if (shape == 1) {  // ellipsoid
    V3<R> a = mk(p.x / h.x, p.y / h.y, p.z / h.z), v = mk(d.x / h.x, d.y / h.y, d.z / h.z);
    R aa = dot(v, v), bb = dot(a, v), cc = dot(a, a) - R(1), disc = bb * bb - aa * cc;
    if (disc < R(0)) return R(kFar);
    t = (-bb - std::sqrt(disc)) / aa;
    if (t <= R(0.001f)) t = (-bb + std::sqrt(disc)) / aa;
  }
  if (shape == 2) {  // capped vertical cylinder
    R a = d.x * d.x / (h.x * h.x) + d.z * d.z / (h.z * h.z);
    R bb = p.x * d.x / (h.x * h.x) + p.z * d.z / (h.z * h.z);
    R cc = p.x * p.x / (h.x * h.x) + p.z * p.z / (h.z * h.z) - R(1);
    R best = R(kFar), disc = bb * bb - a * cc;
    if (disc >= R(0) && a > R(0.0000001f)) {
      R u = (-bb - std::sqrt(disc)) / a, v = (-bb + std::sqrt(disc)) / a;
      if (u > R(0.001f) && std::fabs(p.y + d.y * u) <= h.y) best = u;
      if (v > R(0.001f) && std::fabs(p.y + d.y * v) <= h.y) best = std::fmin(best, v);
    }
    for (int k = 0; k < 2; k++)
      if (std::fabs(d.y) > R(0.000001f)) {
        R cy = k == 0 ? -h.y : h.y, u = (cy - p.y) / d.y;
        R xx = (p.x + d.x * u) / h.x, zz = (p.z + d.z * u) / h.z;
        if (u > R(0.001f) && xx * xx + zz * zz <= R(1)) best = std::fmin(best, u);
      }
    t = best;
  }
  if (shape == 3) {  // triangular prism: the box interval clipped by two sloping half-spaces
    R nearT = std::fmax(R(0.001f), range.lo), farT = range.hi;
    for (int k = 0; k < 2; k++) {
      R sg = k == 0 ? R(1) : R(-1);
      R numer = h.y - (p.y + sg * p.x * h.y / h.x), denom = d.y + sg * d.x * h.y / h.x;
      if (std::fabs(denom) < R(0.000001f)) { if (numer < R(0)) return R(kFar); }
      else { R u = numer / denom; if (denom > R(0)) farT = std::fmin(farT, u); else nearT = std::fmax(nearT, u); }
    }
    if (farT < nearT) return R(kFar);
    t = nearT;
  }
  if (shape == 4 || shape == 7) {  // half arch / full ring: radii 1 and 0.77, end caps
    R best = R(kFar);
    R a = d.x * d.x / (h.x * h.x) + d.y * d.y / (h.y * h.y);
    R bb = p.x * d.x / (h.x * h.x) + p.y * d.y / (h.y * h.y);
    for (int ring = 0; ring < 2; ring++) {
      R rad = ring == 0 ? R(1) : R(0.77f);
      R cc = p.x * p.x / (h.x * h.x) + p.y * p.y / (h.y * h.y) - rad * rad, disc = bb * bb - a * cc;
      if (disc >= R(0) && a > R(0.000001f))
        for (int k = 0; k < 2; k++) {
          R u = (-bb + (k == 0 ? -std::sqrt(disc) : std::sqrt(disc))) / a;
          if (u > R(0.001f) && std::fabs(p.z + d.z * u) <= h.z && (shape == 7 || p.y + d.y * u >= R(0))) best = std::fmin(best, u);
        }
    }
    if (std::fabs(d.z) > R(0.000001f))
      for (int k = 0; k < 2; k++) {
        R u = ((k == 0 ? -h.z : h.z) - p.z) / d.z;
        R xx = (p.x + d.x * u) / h.x, yy = (p.y + d.y * u) / h.y, rr = xx * xx + yy * yy;
        if (u > R(0.001f) && rr <= R(1) && rr >= R(0.77f) * R(0.77f) && (shape == 7 || yy >= R(0))) best = std::fmin(best, u);
      }
    t = best;
  }
  if (shape == 1 && f.material == 7 && t < R(kFar)) t = foliage(ro, rd, cp, h, int(f.seed), range.lo, range.hi, cn);
  if (t <= R(0.001f)) return R(kFar);
  // masonry relief: four fixed-point steps along the ray (geometry.cu:82-89)
  if (shape == 0 && (f.material == 0 || f.material == 1) && h.y > R(1)) {
    V3<R> hp = p + d * t;
    R ex = std::fabs(std::fabs(hp.x) - h.x), ez = std::fabs(std::fabs(hp.z) - h.z);
    if (std::fabs(std::fabs(hp.y) - h.y) > R(0.01f)) {
      V3<R> n = ex < ez ? mk(hp.x < R(0) ? R(-1) : R(1), R(0), R(0)) : mk(R(0), R(0), hp.z < R(0) ? R(-1) : R(1));
      R denom = dot(n, d);
      if (denom < R(-0.08f)) {
        R initial = t;
        for (int k = 0; k < 4; k++) {
          if (cn) cn->v[ORC_MASONRY]++;
          V3<R> wp = ro + rd * t, wn = outOfFeature(n, turn);
          R u, v;
          masonryUV(wp, wn, u, v);
          R disp = masonryHeight(u, v, f.material) * freqWeight(t * cone, R(40));
          t = initial + disp / denom;
        }
      }
    }
  }
  return t;
}

// surface normal of a feature at a point (geometry.cu:92-114)
template <class R> V3<R> featNormal(const Feat& f, V3<R> point) {
  const int shape = f.shape, turn = f.turn;
  const V3<R> p = intoFeature(point - cast3<R>(f.p), turn), h = cast3<R>(f.h);
  V3<R> n = mk(R(0), R(1), R(0));
  if (shape == 1) n = unit(mk(p.x / (h.x * h.x), p.y / (h.y * h.y), p.z / (h.z * h.z)));
  else if (shape == 2) {
    if (std::fabs(std::fabs(p.y) - h.y) < R(0.01f)) n = mk(R(0), p.y < R(0) ? R(-1) : R(1), R(0));
    else n = unit(mk(p.x / (h.x * h.x), R(0), p.z / (h.z * h.z)));
  } else if (shape == 4 || shape == 7) {
    if (std::fabs(std::fabs(p.z) - h.z) < R(0.008f)) n = mk(R(0), R(0), p.z < R(0) ? R(-1) : R(1));
    else {
      R rr = p.x * p.x / (h.x * h.x) + p.y * p.y / (h.y * h.y);
      n = unit(mk(p.x / (h.x * h.x), p.y / (h.y * h.y), R(0))) * (rr < R(0.8f) ? R(-1) : R(1));
    }
  } else if (shape == 3) {
    if (std::fabs(std::fabs(p.z) - h.z) < R(0.006f)) n = mk(R(0), R(0), p.z < R(0) ? R(-1) : R(1));
    else if (p.y < R(0.003f)) n = mk(R(0), R(-1), R(0));
    else n = unit(mk(p.x < R(0) ? -h.y / h.x : h.y / h.x, R(1), R(0)));
  } else {
    V3<R> a = mk(std::fabs(std::fabs(p.x) - h.x), std::fabs(std::fabs(p.y) - h.y), std::fabs(std::fabs(p.z) - h.z));
    n = a.x < a.y && a.x < a.z ? mk(p.x < R(0) ? R(-1) : R(1), R(0), R(0))
        : (a.y < a.z ? mk(R(0), p.y < R(0) ? R(-1) : R(1), R(0)) : mk(R(0), R(0), p.z < R(0) ? R(-1) : R(1)));
    R bevel = std::fmin(R(0.035f), std::fmin(std::fmin(h.x, h.y), h.z) * R(0.18f));
    V3<R> q = mk(std::fmax(std::fabs(p.x) - h.x + bevel, R(0)) * (p.x < R(0) ? R(-1) : R(1)),
                 std::fmax(std::fabs(p.y) - h.y + bevel, R(0)) * (p.y < R(0) ? R(-1) : R(1)),
                 std::fmax(std::fabs(p.z) - h.z + bevel, R(0)) * (p.z < R(0) ? R(-1) : R(1)));
    if (dot(q, q) > R(0.000001f)) n = unit(q);
  }
  if (shape == 1 && f.material == 7)
    return leafNormal<R>(int(std::floor(point.x / R(0.18f))), int(std::floor(point.y / R(0.18f))),
                         int(std::floor(point.z / R(0.18f))), int(f.seed));
  return outOfFeature(n, turn);
}

// ---- the feature grammar (assets.cu:3-265) ---------------------------------
// `Out` receives every feature of one group in emission order.  Emission order
// defines the feature index, so every loop below keeps the reference's order.
template <class Out> struct Emitter {
  Out& out;
  float roofBase, roofScale;
  int count = 0;
  // sink.cu:10-13: features at or above the eave are rescaled vertically.
  void emit(V3f p, V3f h, int shape, int mat, int turn, float seed) {
    if (p.y >= roofBase) { p.y = roofBase + (p.y - roofBase) * roofScale; h.y *= roofScale; }
    Feat f{p, h, shape, mat, turn, seed};
    out(f, count++);
  }
  // sink.cu:27-33: a box on one facade face, offset `out` from the wall.
  void wall(int face, float cx, float cz, float w, float d, float u, float y, float o, float hw, float hy,
            float hd, int mat, float seed) {
    V3f p = mk(cx + u, y, cz + d + o), h = mk(hw, hy, hd);
    if (face == 1) { p = mk(cx + w + o, y, cz + u); h = mk(hd, hy, hw); }
    if (face == 2) p = mk(cx + u, y, cz - d - o);
    if (face == 3) { p = mk(cx - w - o, y, cz + u); h = mk(hd, hy, hw); }
    emit(p, h, 0, mat, 0, seed);
  }
};

template <class Out> void runGroup(const LotDesc& lot, int group, Emitter<Out>& e) {
  const float x = 0.0f, z = 0.0f, w = lot.w, d = lot.d, h = lot.h, seed = lot.seed, storey = lot.storey;
  const int type = lot.type, mat = lot.mat, floors = lot.floors;
  if (type == 5) return;  // open canal water: nothing
  if (type == 4) {        // canal bridge, group 0 only
    if (group == 0) {
      e.emit(mk(x, 0.25f, z), mk(18.0f, 0.5f, 5.0f), 0, 0, 0, seed);
      e.emit(mk(x, 1.25f, z - 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
      e.emit(mk(x, 1.25f, z + 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
      for (int k = 0; k < 12; k++) {
        float u = -16.5f + float(k) * 3.0f;
        e.emit(mk(x + u, 0.8f, z - 5.0f), mk(0.12f, 0.6f, 0.12f), 2, 6, 0, seed);
        e.emit(mk(x + u, 0.8f, z + 5.0f), mk(0.12f, 0.6f, 0.12f), 2, 6, 0, seed);
      }
    }
    return;
  }
  if (type == 3) {  // park: paving, 8 trees, fountain
    if (group == 0) e.emit(mk(x, -0.12f, z), mk(15.5f, 0.22f, 15.5f), 0, 11, 0, seed);
    if (group >= 1 && group <= 8) {
      int k = group - 1;
      float tx = x + (k < 4 ? -10.0f : 10.0f), tz = z + (float(k % 4) - 1.5f) * 6.7f;
      float th = 5.0f + hash1(int(seed) + k) * 3.0f;
      e.emit(mk(tx, th * 0.4f, tz), mk(0.19f, th * 0.4f, 0.19f), 2, 15, 0, seed);
      for (int j = 0; j < 28; j++) {
        float a = float(j) * 2.4f;
        float yy = hash1(int(seed) + j + 991) * 3.3f - 0.5f;
        float rr = std::sqrt(hash1(int(seed) + j + 330)) * 2.1f * (1.0f - yy * 0.12f);
        float size = 0.48f + hash1(int(seed) + j + 62) * 0.30f;
        e.emit(mk(tx + std::cos(a) * rr, th + yy, tz + std::sin(a) * rr), mk(size, size * 1.25f, size), 1, 7, 0,
               seed + float(j));
      }
    }
    if (group == 9) {
      e.emit(mk(x, 0.8f, z), mk(3.6f, 0.45f, 3.6f), 2, 0, 0, seed);
      e.emit(mk(x, 1.24f, z), mk(3.3f, 0.04f, 3.3f), 2, 9, 0, seed);
      e.emit(mk(x, 2.0f, z), mk(0.65f, 1.0f, 0.65f), 2, 0, 0, seed);
      e.emit(mk(x, 2.85f, z), mk(1.4f, 0.18f, 1.4f), 2, 13, 0, seed);
      e.emit(mk(x, 3.15f, z), mk(0.5f, 0.5f, 0.5f), 1, 3, 0, seed);
    }
    return;
  }
  // Buildings (types 0 pitched roof, 1 dome, 2 tower).
  if (group == 0) {  // plinth, mass, cornice, arcade void, 12 columns with capitals
    e.emit(mk(x, 0.15f, z), mk(w + 1.1f, 0.25f, d + 1.1f), 0, 0, 0, seed);
    e.emit(mk(x, (h + 4.0f) * 0.5f, z), mk(w, (h - 4.0f) * 0.5f, d), 0, mat, 0, seed);
    e.emit(mk(x, 4.0f, z), mk(w + 0.24f, 0.24f, d + 0.24f), 0, 13, 0, seed);
    e.emit(mk(x, 1.9f, z), mk(w - 3.5f, 1.9f, d - 3.5f), 0, 5, 0, seed);
    for (int f = 0; f < 4; f++)
      for (int k = 0; k < 3; k++) {
        float ext = (f % 2 == 0 ? w : d) - 0.65f, u = (float(k) - 1.0f) * ext;
        float px = f % 2 == 0 ? x + u : x + (f == 1 ? w - 0.5f : -w + 0.5f);
        float pz = f % 2 == 0 ? z + (f == 0 ? d - 0.5f : -d + 0.5f) : z + u;
        e.emit(mk(px, 2.0f, pz), mk(0.38f, 1.75f, 0.38f), 2, 0, 0, seed + float(k));
        e.emit(mk(px, 3.66f, pz), mk(0.64f, 0.18f, 0.64f), 0, 13, 0, seed);
      }
  }
  if (group == 1) {  // roof
    e.emit(mk(x, h + 0.25f, z), mk(w + 0.6f, 0.24f, d + 0.6f), 0, 13, 0, seed);
    if (type == 0) {
      int roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
      e.emit(mk(x, h + 0.35f, z), mk(w + 0.45f, 4.4f, d + 0.45f), 3, roofmat, 0, seed);
      e.emit(mk(x, h + 4.8f, z), mk(0.12f, 0.14f, d + 0.7f), 0, 3, 0, seed);
      for (int k = 0; k < 4; k++) {
        float xx = x + (k % 2 == 0 ? -w * 0.52f : w * 0.52f), zz = z + (float(k / 2) - 0.5f) * d;
        e.emit(mk(xx, h + storey, zz), mk(0.48f, 2.2f, 0.55f), 0, 1, 0, seed);
        e.emit(mk(xx, h + 6.0f, zz), mk(0.66f, 0.17f, 0.72f), 0, 0, 0, seed);
        e.emit(mk(xx, h + 6.32f, zz), mk(0.2f, 0.25f, 0.2f), 2, 14, 0, seed);
      }
    } else if (type == 1) {
      e.emit(mk(x, h + 2.2f, z), mk(w * 0.72f, 2.0f, w * 0.72f), 2, 0, 0, seed);
      e.emit(mk(x, h + 3.1f, z), mk(w * 0.79f, 8.4f, w * 0.79f), 1, 3, 0, seed);
      e.emit(mk(x, h + 12.2f, z), mk(0.24f, 1.45f, 0.24f), 2, 6, 0, seed);
      e.emit(mk(x, h + 13.8f, z), mk(0.6f, 0.6f, 0.6f), 1, 8, 0, seed);
    } else {
      e.emit(mk(x, h + 0.4f, z), mk(w * 0.72f, 5.2f, d + 0.2f), 3, 2, 0, seed);
      for (int k = 0; k < 2; k++) {
        float xx = x + (k == 0 ? -w * 0.75f : w * 0.75f), zz = z + d * 0.60f;
        e.emit(mk(xx, h + 3.5f, zz), mk(2.3f, 7.2f, 2.3f), 0, 0, 0, seed);
        e.emit(mk(xx, h + 10.9f, zz), mk(2.65f, 0.35f, 2.65f), 0, 13, 0, seed);
        e.emit(mk(xx, h + 11.2f, zz), mk(2.55f, 4.4f, 2.55f), 3, 3, 0, seed);
        e.emit(mk(xx, h + 16.0f, zz), mk(0.17f, 1.2f, 0.17f), 2, 8, 0, seed);
        for (int j = 0; j < 4; j++) {
          float a = float(j) * kPi * 0.5f;
          e.emit(mk(xx + std::cos(a) * 2.2f, h + 12.0f, zz + std::sin(a) * 2.2f), mk(0.17f, 1.1f, 0.17f), 2, 0, 0, seed);
        }
      }
    }
  }
  if (group >= 2 && group <= 5) {  // string courses, pilasters, dentils of one face
    int face = group - 2;
    float ext = face % 2 == 0 ? w : d;
    for (int j = 0; j <= floors; j++) {
      float y = 4.2f + float(j) * storey;
      e.wall(face, x, z, w, d, 0.0f, y, 0.17f, ext + 0.15f, 0.11f, 0.22f, 13, seed);
      e.wall(face, x, z, w, d, 0.0f, y + 0.21f, 0.1f, ext + 0.10f, 0.052f, 0.16f, 0, seed);
    }
    for (int j = 0; j < 5; j++) {
      float u = (float(j) / 4.0f * 2.0f - 1.0f) * (ext - 0.3f);
      e.wall(face, x, z, w, d, u, (h + 4.0f) * 0.5f, 0.16f, 0.19f, (h - 4.0f) * 0.5f, 0.22f, 13, seed);
    }
    for (int j = 0; j < 8; j++) {
      float u = (float(j) - 3.5f) * (ext / 4.0f);
      e.wall(face, x, z, w, d, u, h - 0.24f, 0.4f, 0.15f, 0.12f, 0.19f, 13, seed);
    }
  }
  if (group >= 6 && group < 30) {  // windows of one storey of one face
    int face = (group - 6) / 6, row = (group - 6) % 6;
    if (row >= floors) return;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f), wy = 1.2f;
      e.wall(face, x, z, w, d, u, y, 0.032f, 0.91f, wy, 0.045f, 4, seed + float(row * 17 + j * 9 + face * 59));
      e.wall(face, x, z, w, d, u, y - wy - 0.13f, 0.22f, 1.13f, 0.14f, 0.29f, 13, seed);
      e.wall(face, x, z, w, d, u, y + wy + 0.12f, 0.18f, 1.11f, 0.14f, 0.23f, 13, seed);
      e.wall(face, x, z, w, d, u - 1.02f, y, 0.12f, 0.11f, wy, 0.17f, 13, seed);
      e.wall(face, x, z, w, d, u + 1.02f, y, 0.12f, 0.11f, wy, 0.17f, 13, seed);
      e.wall(face, x, z, w, d, u, y, 0.12f, 0.044f, wy, 0.08f, 5, seed);
      e.wall(face, x, z, w, d, u, y + 0.3f, 0.12f, 0.94f, 0.035f, 0.08f, 5, seed);
      e.wall(face, x, z, w, d, u, y - wy + 0.46f, 0.56f, 1.10f, 0.035f, 0.035f, 6, seed);
    }
  }
  if (group == 30) {  // street furniture: lamps, bollards, arches
    for (int k = 0; k < 2; k++) {
      float px = x + (k == 0 ? -16.0f : 16.0f), pz = z + 15.9f;
      e.emit(mk(px, 2.0f, pz), mk(0.068f, 2.0f, 0.068f), 2, 6, 0, seed);
      e.emit(mk(px, 4.0f, pz), mk(0.29f, 0.38f, 0.29f), 0, 8, 0, seed);
      e.emit(mk(px, 4.44f, pz), mk(0.37f, 0.1f, 0.37f), 3, 6, 0, seed);
      e.emit(mk(px, 0.15f, pz), mk(0.27f, 0.18f, 0.27f), 2, 0, 0, seed);
    }
    for (int k = 0; k < 8; k++)
      e.emit(mk(x - 14.9f, 0.43f, z - 12.0f + float(k) * 3.3f), mk(0.10f, 0.43f, 0.10f), 2, 6, 0, seed);
    for (int face = 0; face < 4; face++)
      for (int k = 0; k < 2; k++) {
        float ext = (face % 2 == 0 ? w : d) - 0.65f, u = (k == 0 ? -0.5f : 0.5f) * ext;
        V3f c = mk(x + u, 3.16f, z + (face == 0 ? d - 0.5f : -d + 0.5f));
        if (face % 2 == 1) c = mk(x + (face == 1 ? w - 0.5f : -w + 0.5f), 3.16f, z + u);
        e.emit(c, mk(ext * 0.5f, 0.88f, 0.49f), 4, 13, face % 2, seed);
      }
  }
  if (group == 31) {  // dormers, arcade glazing, planters
    if (type == 0)
      for (int k = 0; k < 4; k++) {
        float xx = x + (k % 2 == 0 ? -w * 0.68f : w * 0.68f), zz = z + (float(k / 2) - 0.5f) * d * 0.96f;
        e.emit(mk(xx, h + 2.5f, zz), mk(1.35f, 1.05f, 1.05f), 0, 0, 0, seed);
        e.emit(mk(xx, h + 3.55f, zz), mk(1.45f, 1.0f, 1.2f), 3, 2, 1, seed);
        e.emit(mk(xx + (k % 2 == 0 ? -1.36f : 1.36f), h + 2.5f, zz), mk(0.035f, 0.70f, 0.65f), 0, 4, 0, seed);
      }
    for (int face = 0; face < 4; face++) {
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 1.6f, 0.045f, 1.05f, 1.4f, 0.055f, 4, seed);
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.13f, 0.09f, 1.25f, 0.15f, 0.12f, 13, seed);
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 0.18f, 0.18f, 1.25f, 0.10f, 0.35f, 0, seed);
    }
    for (int k = 0; k < 3; k++) {
      float xx = x + (float(k) - 1.0f) * 7.0f;
      e.emit(mk(xx, 0.48f, z + d + 1.5f), mk(0.52f, 0.42f, 0.52f), 2, 14, 0, seed);
      e.emit(mk(xx, 1.13f, z + d + 1.5f), mk(0.7f, 0.8f, 0.7f), 1, 7, 0, seed + float(k));
    }
  }
  if (group >= 32 && group < 56) {  // balconies of one storey of one face
    int face = (group - 32) / 6, row = (group - 32) % 6;
    if (row >= floors) return;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, y - 1.18f, 0.56f, 1.16f, 0.085f, 0.65f, 13, seed);
      e.wall(face, x, z, w, d, u, y - 0.28f, 1.12f, 1.15f, 0.035f, 0.035f, 6, seed);
      e.wall(face, x, z, w, d, u, y - 1.00f, 1.12f, 1.15f, 0.026f, 0.026f, 6, seed);
      for (int k = 0; k < 5; k++)
        e.wall(face, x, z, w, d, u + (float(k) - 2.0f) * 0.53f, y - 0.64f, 1.12f, 0.025f, 0.37f, 0.026f, 6, seed);
    }
  }
  if (group >= 56 && group < 60) {  // quoins (and rose windows on towers)
    int face = group - 56;
    float ext = face % 2 == 0 ? w : d;
    for (int k = 0; k < 14; k++) {
      float yy = 4.45f + float(k) * (h - 4.0f) / 14.0f, width = k % 2 == 0 ? 0.52f : 0.30f;
      e.wall(face, x, z, w, d, -ext + width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
      e.wall(face, x, z, w, d, ext - width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
    }
    if (type == 2) {
      V3f c = mk(x, h - 2.3f, z + (face == 0 ? d + 0.21f : -d - 0.21f));
      if (face % 2 == 1) c = mk(x + (face == 1 ? w + 0.21f : -w - 0.21f), h - 2.3f, z);
      e.emit(c, mk(2.35f, 2.35f, 0.26f), 7, 13, face % 2, seed);
      e.emit(c, mk(1.85f, 1.85f, 0.032f), 1, 17, face % 2, seed);
    }
  }
  if ((group == 60 || group == 61) && type == 0) {  // 32 roof slats per side
    int side = group - 60, roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
    for (int j = 0; j < 32; j++) {
      float zz = z - d + (float(j + side * 32) + 0.5f) * d / 32.0f;
      e.emit(mk(x, h + 0.395f, zz), mk(w + 0.46f, 4.42f, 0.023f), 3, roofmat, 0, seed);
    }
  }
  if (group == 62)  // curbs
    for (int side = 0; side < 2; side++)
      for (int k = 0; k < 16; k++) {
        float u = -15.5f + float(k) * 2.0f;
        e.emit(mk(x + u, 0.16f, z + (side == 0 ? -16.3f : 16.3f)), mk(0.98f, 0.19f, 0.19f), 0, 0, 0, seed);
      }
  if (group == 63)  // roofline brackets
    for (int face = 0; face < 4; face++)
      for (int k = 0; k < 8; k++) {
        float ext = face % 2 == 0 ? w : d, u = (float(k) - 3.5f) * ext * 0.25f;
        e.wall(face, x, z, w, d, u, h - 0.36f, 0.48f, 0.12f, 0.24f, 0.24f, 13, seed);
      }
  // Hyperdetail bands (assets.cu:199-249); the reference's lod is fixed at 5.
  if (group >= 2 && group <= 5) {
    int face = group - 2;
    float ext = face % 2 == 0 ? w : d;
    for (int k = 0; k < 4; k++) {
      float yy = 5.05f + float(k) * std::fmax(1.0f, (h - 6.0f) / 4.0f);
      e.wall(face, x, z, w, d, 0.0f, yy, 0.205f, ext + 0.08f, 0.035f, 0.055f, 13, seed + 410.0f + float(k));
    }
    for (int k = 0; k < 4; k++) {
      float u = (float(k) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, h - 0.72f, 0.255f, 0.055f, 0.34f, 0.07f, 0, seed + 450.0f + float(k));
    }
  }
  if (group >= 6 && group < 30) {
    int face = (group - 6) / 6, row = (group - 6) % 6;
    if (row < floors) {
      float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
      for (int j = 0; j < 4; j++) {
        float u = (float(j) - 1.5f) * (ext * 0.48f);
        e.wall(face, x, z, w, d, u - 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 500.0f + float(j));
        e.wall(face, x, z, w, d, u + 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 520.0f + float(j));
      }
      for (int j = 0; j < 4; j++) {
        float u = (float(j) - 1.5f) * (ext * 0.48f);
        e.wall(face, x, z, w, d, u, y - 1.31f, 0.30f, 1.18f, 0.045f, 0.07f, 13, seed + 540.0f + float(j));
        e.wall(face, x, z, w, d, u, y + 1.31f, 0.18f, 1.08f, 0.038f, 0.055f, 13, seed + 560.0f + float(j));
      }
    }
  }
  if (group >= 32 && group < 56) {
    int face = (group - 32) / 6, row = (group - 32) % 6;
    if (row < floors) {
      float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
      for (int j = 0; j < 4; j++) {
        float u = (float(j) - 1.5f) * (ext * 0.48f);
        e.wall(face, x, z, w, d, u, y - 0.22f, 1.17f, 1.20f, 0.028f, 0.035f, 6, seed + 600.0f + float(j));
        e.wall(face, x, z, w, d, u, y - 1.23f, 0.62f, 1.19f, 0.038f, 0.038f, 6, seed + 620.0f + float(j));
      }
      for (int j = 0; j < 4; j++) {
        float u = (float(j) - 1.5f) * (ext * 0.48f);
        e.wall(face, x, z, w, d, u - 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 640.0f + float(j));
        e.wall(face, x, z, w, d, u + 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 660.0f + float(j));
      }
    }
  }
  if (group == 30) {
    for (int k = 0; k < 4; k++) {
      float side = k < 2 ? -1.0f : 1.0f, along = (k % 2 == 0 ? -0.58f : 0.58f);
      e.emit(mk(x + side * (w + 0.34f), h * 0.38f, z + along * d), mk(0.075f, h * 0.38f, 0.075f), 2, 6, 0,
             seed + 700.0f + float(k));
    }
    for (int k = 0; k < 4; k++)
      e.emit(mk(x - 12.0f + float(k) * 8.0f, 0.48f, z + d + 2.0f), mk(0.12f, 0.48f, 0.12f), 2, 6, 0, seed + 720.0f + float(k));
    for (int k = 0; k < 8; k++)
      e.emit(mk(x - 14.0f + float(k) * 4.0f, 0.055f, z - d - 2.2f), mk(1.75f, 0.035f, 0.045f), 0, 13, 0,
             seed + 740.0f + float(k));
  }
  if (group == 31) {
    for (int k = 0; k < 4; k++) {
      float xx = x + (float(k % 2) - 0.5f) * w, zz = z + (float(k / 2) - 0.5f) * d;
      e.emit(mk(xx, h + 0.72f, zz), mk(0.34f, 0.48f, 0.34f), 2, 6, 0, seed + 800.0f + float(k));
      e.emit(mk(xx, h + 1.18f, zz), mk(0.46f, 0.055f, 0.46f), 0, 13, 0, seed + 820.0f + float(k));
    }
    for (int k = 0; k < 8; k++) {
      float a = float(k) * kPi * 0.25f;
      e.emit(mk(x + std::cos(a) * w * 0.44f, h + 0.42f, z + std::sin(a) * d * 0.44f), mk(0.055f, 0.42f, 0.055f), 2, 6,
             0, seed + 840.0f + float(k));
    }
  }
  // Street benches and the final awnings (assets.cu:252-263).
  if (group == 30)
    for (int bench = 0; bench < 2; bench++) {
      float bx = bench == 0 ? -7.0f : 7.0f, bz = d + 1.8f;
      for (int slat = 0; slat < 4; slat++)
        e.emit(mk(bx, 0.59f, bz + (float(slat) - 1.5f) * 0.13f), mk(1.3f, 0.045f, 0.053f), 0, 5, 0, seed + 900.0f + float(slat));
      for (int leg = 0; leg < 2; leg++)
        e.emit(mk(bx + (leg == 0 ? -0.95f : 0.95f), 0.3f, bz), mk(0.065f, 0.3f, 0.27f), 0, 6, 0, seed);
      for (int rail = 0; rail < 2; rail++)
        e.emit(mk(bx, 0.88f + float(rail) * 0.19f, bz + 0.23f), mk(1.3f, 0.075f, 0.045f), 0, 5, 0, seed);
    }
  if (group == 31)
    for (int face = 0; face < 4; face++)
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.1f, 0.6f, 1.38f, 0.10f, 0.7f, (int(seed)) % 2 == 0 ? 14 : 2,
             seed + 940.0f + float(face));
}

template <class F> int forEachFeature(const LotDesc& lot, int group, F&& fn) {
  Emitter<F> e{fn, lot.h, lot.roofScale};
  runGroup(lot, group, e);
  return e.count;
}

// conservative group AABB (sink.cu:15-20): [lo.xyz, count, hi.xyz]
void groupBounds(const LotDesc& lot, int group, float* o7) {
  V3f lo = mk(1000000.0f, 1000000.0f, 1000000.0f), hi = mk(-1000000.0f, -1000000.0f, -1000000.0f);
  int n = forEachFeature(lot, group, [&](const Feat& f, int) {
    V3f ext = f.h;
    if (f.turn % 2 == 1) ext = mk(f.h.z, f.h.y, f.h.x);
    V3f a = f.p - ext, b = f.p + ext;
    if (f.shape == 3 || f.shape == 4) a.y = f.p.y;
    const V3f pad = mk(0.025f, 0.025f, 0.025f);
    lo = vmin(lo, a - pad);
    hi = vmax(hi, b + pad);
  });
  o7[0] = lo.x; o7[1] = lo.y; o7[2] = lo.z; o7[3] = float(n); o7[4] = hi.x; o7[5] = hi.y; o7[6] = hi.z;
}

// the 127-node hierarchy of one lot (accel.cu:2-15) into a 128x8 block
void lotHierarchy(const LotDesc& lot, float* blk) {
  for (int g = 0; g < kGroups; g++) {
    float* n = blk + (kGroups + g) * 8;
    groupBounds(lot, g, n);
    n[7] = float(g);
  }
  for (int first = 32; first >= 1; first /= 2)
    for (int j = first; j < 2 * first; j++) {
      float *b = blk + j * 8, *a = blk + 2 * j * 8, *c = a + 8;
      for (int k = 0; k < 3; k++) { b[k] = std::fmin(a[k], c[k]); b[4 + k] = std::fmax(a[4 + k], c[4 + k]); }
      b[3] = a[3] + c[3];
      b[7] = 0.0f;
    }
}

// ---- nearest-hit query of one lot (trace.cu:2-28) --------------------------
// The two smallest candidate distances a ray has computed (tie rule): a ray
// whose nearest and second-nearest candidates are within the distance
// tolerance may legitimately resolve to either.  Candidates in culled groups
// are never computed, so `b` is an upper bound on the true second distance.
struct TwoMin {
  float a = kFar, b = kFar;
  void offer(float t) {
    if (!(t > 0.001f && t < kFar)) return;
    if (t < a) { b = a; a = t; } else if (t < b) b = t;
  }
};
struct Nearest { float t; int fid; Feat f; };
// All features of one group against the ray; t starts at the caller's bound.
inline void groupNearest(const LotDesc& lot, int group, V3f ro, V3f rd, float cone, float bound, float& t, int& fid,
                         Feat& f, TwoMin* track, Counters* cn) {
  if (cn) cn->v[ORC_GROUP]++;
  t = bound; fid = -1;
  forEachFeature(lot, group, [&](const Feat& ft, int id) {
    float th = hitFeature<float>(ft, ro, rd, cone, cn);
    if (track) track->offer(th);
    if (th > 0.001f && th < t) { t = th; f = ft; fid = id; }
  });
}
inline float nodeEntry(const float* N, int node, V3f ro, V3f rd, float best, Counters* cn) {
  if (cn) cn->v[ORC_NODE]++;
  const float* b = N + node * 8;
  if (b[3] < 0.5f) return kFar;
  Span<float> r = slab(ro, rd, mk(b[0], b[1], b[2]), mk(b[4], b[5], b[6]));
  if (r.hi < std::fmax(0.001f, r.lo) || r.lo > best) return kFar;
  return std::fmax(0.001f, r.lo);
}
// near-first descent of the 127-node tree with an 8-entry stack
Nearest queryLotNearest(const LotDesc& lot, const float* N, int slot, V3f ro, V3f rd, float best, float cone,
                        Counters* cn, TwoMin* track) {
  Nearest hit{best, -1, Feat{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f}};
  int stack[8], top = 0, node = 1, steps = 0;
  const int base = slot * kNodes;
  while (node > 0 && steps < kNodes) {
    steps++;
    float nearT = nodeEntry(N, base + node, ro, rd, hit.t, cn);
    if (nearT < hit.t && node < kGroups) {
      int left = node * 2, right = left + 1;
      float ln = nodeEntry(N, base + left, ro, rd, hit.t, cn), rn = nodeEntry(N, base + right, ro, rd, hit.t, cn);
      bool lh = ln < hit.t, rh = rn < hit.t;
      if (lh && rh) {
        int next = ln < rn ? left : right, other = ln < rn ? right : left;
        stack[top++] = other;  // at most one push per level of a 6-level tree
        node = next;
      } else if (lh) node = left;
      else if (rh) node = right;
      else { node = 0; if (top > 0) node = stack[--top]; }
    } else {
      if (nearT < hit.t && node >= kGroups) {
        float t; int fid; Feat f;
        groupNearest(lot, node - kGroups, ro, rd, cone, hit.t, t, fid, f, track, cn);
        if (fid >= 0 && t < hit.t) { hit.t = t; hit.fid = (node - kGroups) * kMaxFeatures + fid; hit.f = f; }
      }
      node = 0;
      if (top > 0) node = stack[--top];
    }
  }
  return hit;
}

// ---- primary visibility (trace.cu:29-61) -----------------------------------
void tracePixel(const float* W, const float* N, const uint32_t* O, const float* C, float* Hit, float* Surf, int width,
                int height, int x, int y, Counters* cn, float* second) {
  const int b = (y * width + x) * 4;
  V3f ro = camPos(C), rd = primaryDir(C, x, y, width, height);
  float best = kFar, seed = 0.0f;
  int fid = -10000, material = 10, found = -1;
  V3f normal = mk(0.0f, 1.0f, 0.0f);
  TwoMin cand;
  if (cn) cn->v[ORC_RAYS]++;
  if (rd.y < -0.000001f) {
    float ground = -ro.y / rd.y;
    cand.offer(ground);
    if (ground > 0.001f && ground < best) { best = ground; fid = -1; }
  }
  float nearT = 0.001f, farT = best;
  if (std::fabs(rd.y) > 0.0000001f) {
    float a = (-0.5f - ro.y) / rd.y, c = (kTop - ro.y) / rd.y;
    nearT = std::fmax(nearT, std::fmin(a, c));
    farT = std::fmin(farT, std::fmax(a, c));
  } else if (ro.y > kTop || ro.y < -0.5f) farT = -1.0f;
  if (nearT <= farT) {  // 2-D DDA over 36 m lot cells
    float t = nearT + 0.0002f;
    V3f start = ro + rd * t;
    int cx = int(std::floor((start.x + 18.0f) / kCell)), cz = int(std::floor((start.z + 18.0f) / kCell));
    int sx = rd.x > 0.0f ? 1 : -1, sz = rd.z > 0.0f ? 1 : -1;
    float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * guardedInv(rd.x);
    float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * guardedInv(rd.z);
    float dx = kCell * std::fabs(guardedInv(rd.x)), dz = kCell * std::fabs(guardedInv(rd.z));
    for (int step = 0; step < 160; step++) {
      if (t > best || t > farT || t > kFar) break;
      if (cn) cn->v[ORC_DDA]++;
      int slot = tableSlot(O, cx, cz);
      LotDesc lot = loadLot(W, slot);
      V3f cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
      V3f lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
      if (nodeEntry(N, slot * kNodes + 1, lr, ld, best, cn) < best) {
        Nearest hit = queryLotNearest(lot, N, slot, lr, ld, best, 1.08f / float(height), cn, &cand);
        if (hit.fid >= 0 && hit.t < best) {
          best = hit.t; fid = hit.fid; material = hit.f.material; seed = hit.f.seed;
          normal = fromLot(featNormal<float>(hit.f, lr + ld * best), lot.turn);
          found = slot;
        }
      }
      if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
    }
  }
  Hit[b] = best; Hit[b + 1] = float(fid); Hit[b + 2] = float(material); Hit[b + 3] = seed;
  Surf[b] = normal.x; Surf[b + 1] = normal.y; Surf[b + 2] = normal.z; Surf[b + 3] = float(found);
  if (second) second[y * width + x] = (cand.a == best) ? cand.b : cand.a;
}

// An arbitrary ray through the table (trace.cu:33-61); with `exhaustive` every
// group of each visited lot is evaluated in index order instead of walking the
// hierarchy.  out8 = [t, fid, material, seed, n.xyz, slot].
void traceRayOrc(const float* W, const float* N, const uint32_t* O, V3f ro, V3f rd, float cone, bool exhaustive,
                 float* out8) {
  float best = kFar, seed = 0.0f;
  int fid = -10000, material = 10, found = -1;
  V3f normal = mk(0.0f, 1.0f, 0.0f);
  if (rd.y < -0.000001f) {
    float ground = -ro.y / rd.y;
    if (ground > 0.001f && ground < best) { best = ground; fid = -1; }
  }
  float nearT = 0.001f, farT = best;
  if (std::fabs(rd.y) > 0.0000001f) {
    float a = (-0.5f - ro.y) / rd.y, c = (kTop - ro.y) / rd.y;
    nearT = std::fmax(nearT, std::fmin(a, c));
    farT = std::fmin(farT, std::fmax(a, c));
  } else if (ro.y > kTop || ro.y < -0.5f) farT = -1.0f;
  if (nearT <= farT) {
    float t = nearT + 0.0002f;
    V3f start = ro + rd * t;
    int cx = int(std::floor((start.x + 18.0f) / kCell)), cz = int(std::floor((start.z + 18.0f) / kCell));
    int sx = rd.x > 0.0f ? 1 : -1, sz = rd.z > 0.0f ? 1 : -1;
    float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * guardedInv(rd.x);
    float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * guardedInv(rd.z);
    float dx = kCell * std::fabs(guardedInv(rd.x)), dz = kCell * std::fabs(guardedInv(rd.z));
    for (int step = 0; step < 160; step++) {
      if (t > best || t > farT || t > kFar) break;
      int slot = tableSlot(O, cx, cz);
      LotDesc lot = loadLot(W, slot);
      V3f cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
      V3f lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
      if (exhaustive) {
        for (int g = 0; g < kGroups; g++) {
          float th; int id; Feat f;
          groupNearest(lot, g, lr, ld, cone, best, th, id, f, nullptr, nullptr);
          if (id >= 0 && th < best) {
            best = th; fid = g * kMaxFeatures + id; material = f.material; seed = f.seed;
            normal = fromLot(featNormal<float>(f, lr + ld * best), lot.turn);
            found = slot;
          }
        }
      } else if (nodeEntry(N, slot * kNodes + 1, lr, ld, best, nullptr) < best) {
        Nearest hit = queryLotNearest(lot, N, slot, lr, ld, best, cone, nullptr, nullptr);
        if (hit.fid >= 0 && hit.t < best) {
          best = hit.t; fid = hit.fid; material = hit.f.material; seed = hit.f.seed;
          normal = fromLot(featNormal<float>(hit.f, lr + ld * best), lot.turn);
          found = slot;
        }
      }
      if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
    }
  }
  out8[0] = best; out8[1] = float(fid); out8[2] = float(material); out8[3] = seed;
  out8[4] = normal.x; out8[5] = normal.y; out8[6] = normal.z; out8[7] = float(found);
}

// ---- materials (materials.cu) ----------------------------------------------
inline V3f substrateMean(int m) { return m == 1 ? mk(0.37f, 0.185f, 0.105f) : mk(0.55f, 0.485f, 0.365f); }
V3f substrate(float u, float v, float seed, int m) {
  float large = fbm2(u * 0.31f + seed * 0.013f, v * 0.31f);
  float run = fbm2(u * 0.42f + seed * 0.01f, v * 0.038f + 1.7f);
  V3f base = substrateMean(m);
  float age = 0.61f + 0.52f * large, damp = smooth(0.49f, 0.76f, run) * 0.31f;
  return base * (age - damp) + mk(0.017f, 0.024f, 0.014f) * damp;
}
// ---- optional material surrogate (learning.cu; Stratum.cu:648-664) ---------
// An 8 -> 24 tanh -> 3 network for the substrate colour of brick and stone.
constexpr int kNnInputs = 8, kNnHidden = 24, kNnParams = 291, kNnBatch = 64, kNnWs = 64, kNnTrain = 56;
constexpr int kNnB1 = 192, kNnW2 = 216, kNnB2 = 288;
constexpr int kNnTarget = 8, kNnOut = 11, kNnHid = 14, kNnValid = 62, kNnMat = 63;
inline bool materialTrainNow(const float* C) { return (int(C[6]) % 4) == 0 && C[21] < 0.5f; }  // learning.cu:4
float nnFeature(int i, float u, float v, float seed, int mat) {  // Stratum.cu:648-657
  if (i == 0) return angSin(u * 0.13f);
  if (i == 1) return angCos(u * 0.13f);
  if (i == 2) return angSin(v * 0.13f);
  if (i == 3) return angCos(v * 0.13f);
  if (i == 4) return noise2(u * 0.31f + seed * 0.013f, v * 0.31f) * 2.0f - 1.0f;
  if (i == 5) return noise2(u * 0.42f + seed * 0.01f, v * 0.038f + 1.7f) * 2.0f - 1.0f;
  if (i == 6) return float(mat) * 2.0f - 1.0f;
  return angSin(seed * 0.03f);
}
inline float nnActivate(float x) {  // Stratum.cu:658
  x = clampv(x, -8.0f, 8.0f);
  return 2.0f / (1.0f + angExp(-2.0f * x)) - 1.0f;
}
V3f predictSubstrateNet(const float* W, float u, float v, float seed, int mat) {  // Stratum.cu:659-664
  float hidden[kNnHidden];
  for (int h = 0; h < kNnHidden; h++) {
    float z = W[kNnB1 + h];
    for (int j = 0; j < kNnInputs; j++) z += W[h * 8 + j] * nnFeature(j, u, v, seed, mat);
    hidden[h] = nnActivate(z);
  }
  V3f out = mk(W[kNnB2], W[kNnB2 + 1], W[kNnB2 + 2]);
  for (int h = 0; h < kNnHidden; h++) {
    out.x += W[kNnW2 + h] * hidden[h];
    out.y += W[kNnW2 + 24 + h] * hidden[h];
    out.z += W[kNnW2 + 48 + h] * hidden[h];
  }
  return mk(sat(out.x), sat(out.y), sat(out.z));
}
// The surrogate's parameters while orc_shadePixelsNeural shades with it.
const float* gNeuralW = nullptr;

V3f skyColor(V3f rd, V3f sun) {
  float elev = sat(rd.y);
  V3f c = mix(mk(0.62f, 0.69f, 0.72f), mk(0.13f, 0.30f, 0.52f), std::pow(elev, 0.45f));
  float sd = std::fmax(0.0f, dot(rd, sun));
  c = c + mk(1.1f, 0.62f, 0.22f) * std::pow(sd, 18.0f) + mk(9.0f, 6.0f, 3.2f) * std::pow(sd, 2600.0f);
  if (rd.y > 0.025f) {
    float cloud = fbm2(rd.x / (rd.y + 0.20f) * 1.8f + 16.0f, rd.z / (rd.y + 0.20f) * 1.8f);
    float veil = smooth(0.46f, 0.70f, cloud) * smooth(0.02f, 0.2f, rd.y) * 0.55f;
    c = mix(c, mk(0.86f, 0.85f, 0.80f), veil);
  }
  return c;
}
V3f mineralCell(float u, float v, int seed) {
  int ix = int(std::floor(u)), iy = int(std::floor(v));
  float x = fract(u), y = fract(v), nearest = 10.0f, second = 10.0f, value = 0.0f;
  for (int j = -1; j <= 1; j++)
    for (int i = -1; i <= 1; i++) {
      float dx = float(i) + 0.18f + 0.64f * hash2(ix + i, iy + j, seed) - x;
      float dy = float(j) + 0.18f + 0.64f * hash2(ix + i, iy + j, seed + 47) - y;
      float dd = dx * dx + dy * dy;
      if (dd < nearest) { second = nearest; nearest = dd; value = hash2(ix + i, iy + j, seed + 83); }
      else second = std::fmin(second, dd);
    }
  return mk(std::sqrt(nearest), value, std::sqrt(second) - std::sqrt(nearest));
}
float microRelief(float u, float v, float fp) {
  float value = (noise2(u * 83.0f, v * 83.0f) - 0.5f) * 0.0016f * freqWeight(fp, 83.0f);
  value += (noise2(u * 277.0f + 8.7f, v * 277.0f) - 0.5f) * 0.00048f * freqWeight(fp, 277.0f);
  value += (noise2(u * 911.0f, v * 911.0f - 13.9f) - 0.5f) * 0.00013f * freqWeight(fp, 911.0f);
  return value;
}
V3f surfaceColor(V3f p, V3f n, int mat, float seed, float fp, V3f foundation) {
  float u, v;
  masonryUV(p, n, u, v);
  float fine = freqWeight(fp, 34.0f);
  V3f c = foundation;
  if (mat == 0 || mat == 1) {
    float bw = mat == 1 ? 0.46f : 0.92f, bh = mat == 1 ? 0.215f : 0.46f;
    int row = int(std::floor(v / bh)), brick = int(std::floor(u / bw + float(imod(row, 2)) * 0.5f));
    float xx = fract(u / bw + float(imod(row, 2)) * 0.5f), yy = fract(v / bh);
    float edge = std::fmin(std::fmin(xx, 1.0f - xx) * bw, std::fmin(yy, 1.0f - yy) * bh);
    float joint = (1.0f - smooth(0.005f, 0.021f + fp * 0.4f, edge)) * freqWeight(fp, 1.0f / bh);
    float variation = (hash2(brick, row, int(seed)) - 0.5f) * 0.19f * freqWeight(fp, 1.0f / bh);
    c = c * (1.0f + variation);
    c = mix(c, mk(0.25f, 0.245f, 0.21f), joint * 0.84f);
    float pores = fine > 0.0f ? fbm2(u * 52.0f + seed, v * 52.0f) : 0.5f;
    c = c * (1.0f + (pores - 0.5f) * 0.38f * fine);
    float deposits = smooth(0.45f, 0.76f, fbm2(u * 5.1f + seed * 0.3f, v * 6.2f));
    c = mix(c, mk(0.52f, 0.49f, 0.39f), deposits * 0.23f * (1.0f - joint));
    if (fp < 0.007f) {
      V3f mineral = mineralCell(u * 190.0f, v * 190.0f, int(seed));
      float detail = freqWeight(fp, 190.0f);
      float pit = (1.0f - smooth(0.075f, 0.23f, mineral.x)) * smooth(0.52f, 0.76f, mineral.y) * detail;
      float grit = (1.0f - smooth(0.018f, 0.072f, mineral.z)) * detail;
      c = c * (1.0f - pit * 0.66f - grit * 0.075f);
      float fleck = (1.0f - smooth(0.04f, 0.17f, mineral.x)) * (1.0f - smooth(0.07f, 0.18f, mineral.y)) * detail;
      c = mix(c, mk(0.62f, 0.56f, 0.44f), fleck * 0.78f);
      float powder = (noise2(u * 740.0f, v * 740.0f) - 0.5f) * freqWeight(fp, 740.0f);
      c = c * (1.0f + powder * (joint > 0.5f ? 0.50f : 0.24f));
    }
    float crack = std::fabs(std::sin(u * 8.4f + fbm2(u * 2.4f, v * 2.4f) * 5.0f + v * 1.3f));
    float fracture = (1.0f - smooth(0.012f, 0.042f + fp * 4.0f, crack)) * smooth(0.48f, 0.72f, noise2(u * 1.4f, v * 1.4f));
    c = c * (1.0f - fracture * 0.45f * freqWeight(fp, 15.0f));
    float moss = (1.0f - smooth(0.1f, 3.1f, p.y)) * smooth(0.44f, 0.69f, noise2(u * 1.3f, v * 0.3f));
    c = mix(c, mk(0.095f, 0.125f, 0.046f), moss * 0.7f);
  } else if (mat == 2 || mat == 14) {
    c = mat == 2 ? mk(0.14f, 0.19f, 0.22f) : mk(0.38f, 0.125f, 0.048f);
    float tile = fract(u * 3.7f), row = fract(v * 4.4f);
    float seam = (1.0f - smooth(0.01f, 0.07f, tile)) + (1.0f - smooth(0.02f, 0.11f, row));
    c = c * (0.78f + 0.26f * lerp(0.5f, noise2(u * 7.2f, v * 7.2f), freqWeight(fp, 7.2f)) -
             sat(seam) * 0.25f * freqWeight(fp, 4.4f));
  } else if (mat == 3) {
    float patina = smooth(0.28f, 0.64f, fbm2(u * 2.1f, v * 2.1f));
    c = mix(mk(0.27f, 0.145f, 0.072f), mk(0.085f, 0.24f, 0.18f), patina);
    float seam = 1.0f - smooth(0.015f, 0.07f, fract(u * 1.8f));
    c = c * (1.0f - seam * 0.4f * freqWeight(fp, 1.8f));
  } else if (mat == 4) c = mk(0.045f, 0.084f, 0.093f);
  else if (mat == 5) {
    float grain = std::sin(u * 49.0f + fbm2(u * 2.0f, v * 0.5f) * 8.0f);
    c = mk(0.12f, 0.07f, 0.039f) * (1.0f + grain * 0.12f * fine);
  } else if (mat == 6) c = mk(0.075f, 0.091f, 0.087f) * (0.8f + noise2(u * 30.0f, v * 30.0f) * 0.3f);
  else if (mat == 7) {
    float leaves = fbm2(p.x * 8.0f + p.y * 6.0f, p.z * 8.0f);
    c = mix(mk(0.055f, 0.095f, 0.020f), mk(0.18f, 0.25f, 0.055f), leaves);
  } else if (mat == 8) c = mk(0.70f, 0.43f, 0.13f);
  else if (mat == 9) c = mk(0.035f, 0.115f, 0.12f);
  else if (mat == 10) {
    float grit = lerp(0.5f, fbm2(u * 45.0f, v * 45.0f), freqWeight(fp, 45.0f));
    c = mk(0.16f, 0.17f, 0.16f) * (0.72f + grit * 0.4f);
  } else if (mat == 11) {
    int row = int(std::floor(v / 0.45f));
    float a = fract(u / 0.9f + float(imod(row, 2)) * 0.5f), b = fract(v / 0.45f);
    float joint = (1.0f - smooth(0.02f, 0.07f + fp, std::fmin(std::fmin(a, 1.0f - a), std::fmin(b, 1.0f - b))));
    c = mk(0.43f, 0.415f, 0.36f) * (0.78f + fbm2(u * 18.0f, v * 18.0f) * 0.3f);
    c = c * (1.0f - joint * 0.30f * freqWeight(fp, 2.0f));
  } else if (mat == 13) c = mk(0.54f, 0.475f, 0.35f) * (0.82f + fbm2(u * 1.6f, v * 1.6f) * 0.24f);
  else if (mat == 15) c = mk(0.17f, 0.12f, 0.065f) * (0.65f + 0.6f * fbm2(u * 31.0f, v * 3.0f));
  if (mat == 18) {
    float panel = fract(u / 1.6f);
    float frame = (1.0f - smooth(0.02f, 0.06f, panel)) + (1.0f - smooth(0.02f, 0.06f, 1.0f - panel));
    float band = 1.0f - smooth(0.03f, 0.07f, std::fabs(v - 2.65f));
    c = mix(mk(0.058f, 0.092f, 0.105f), mk(0.10f, 0.059f, 0.027f), sat(frame + band));
  }
  if (mat == 17) {
    float a = std::atan2(v - std::floor(v / 30.0f) * 30.0f - 28.5f, u);
    float glass = 0.5f + 0.5f * std::sin(a * 12.0f + seed);
    c = mix(mk(0.08f, 0.18f, 0.32f), mk(0.50f, 0.12f, 0.04f), glass);
  }
  return c;
}

// ---- lighting (shade.cu) ---------------------------------------------------
float buildingShadow(const float* W, const uint32_t* O, V3f p, V3f light, int worldSeed, Counters* cn) {
  if (light.y < 0.005f) return 0.05f;
  float limit = std::fmin(1500.0f, std::fmax(0.0f, (kTop - p.y) / light.y));
  V3f ro = p + light * 0.08f;
  int cx = int(std::floor((ro.x + 18.0f) / kCell)), cz = int(std::floor((ro.z + 18.0f) / kCell));
  int sx = light.x > 0.0f ? 1 : -1, sz = light.z > 0.0f ? 1 : -1;
  float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * guardedInv(light.x);
  float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * guardedInv(light.z);
  float dx = kCell * std::fabs(guardedInv(light.x)), dz = kCell * std::fabs(guardedInv(light.z)), t = 0.0f;
  for (int step = 0; step < 64; step++) {
    if (t > limit) break;
    if (cn) cn->v[ORC_SDDA]++;
    LotDesc l;
    if (cx >= -64 && cx < 64 && cz >= -64 && cz < 64) l = loadLot(W, tableSlot(O, cx, cz));
    else l = describe(shiftAddr(O, cx, cz), worldSeed);
    V3f cp = mk(float(cx) * kCell + l.ox, 0.0f, float(cz) * kCell + l.oz);
    if (l.type < 3) {
      V3f lr = toLot(ro - cp, l.turn), ld = toLot(light, l.turn);
      Span<float> s = slab(lr, ld, mk(-l.w + 0.05f, 4.1f, -l.d + 0.05f), mk(l.w - 0.05f, l.h, l.d - 0.05f));
      if (s.hi > std::fmax(0.06f, s.lo) && s.lo < limit) return 0.06f;
    }
    if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
  }
  return 1.0f;
}
float ambientVisibility(const float* W, const uint32_t* O, V3f p) {
  int cx = int(std::floor((p.x + 18.0f) / kCell)), cz = int(std::floor((p.z + 18.0f) / kCell));
  float occ = 0.0f;
  for (int z = -1; z <= 1; z++)
    for (int x = -1; x <= 1; x++) {
      LotDesc l = loadLot(W, tableSlot(O, cx + x, cz + z));
      if (l.type >= 3) continue;
      V3f q = toLot(p - mk(float(cx + x) * kCell + l.ox, 0.0f, float(cz + z) * kCell + l.oz), l.turn);
      float xx = std::fmax(0.0f, std::fabs(q.x) - l.w), zz = std::fmax(0.0f, std::fabs(q.z) - l.d);
      float dist = std::sqrt(xx * xx + zz * zz);
      if (dist > 0.06f) occ += sat((l.h - p.y) / (dist + l.h + 1.0f)) * std::exp(-dist * 0.12f) * 0.48f;
    }
  return clampv(1.0f - occ, 0.35f, 1.0f);
}
V3f paletteTint(float palette, int mat) {
  if (mat != 0 && mat != 1 && mat != 13) return mk(1.0f, 1.0f, 1.0f);
  static const float tint[8][3] = {{1.04f, 0.95f, 0.85f}, {0.80f, 0.89f, 1.02f}, {1.12f, 0.89f, 0.83f},
                                   {1.13f, 1.12f, 1.04f}, {0.83f, 0.84f, 0.79f}, {0.91f, 1.02f, 0.91f},
                                   {1.03f, 0.95f, 1.02f}, {1.0f, 1.0f, 1.0f}};
  int p = int(palette);
  if (p < 0 || p > 7) p = 7;
  return mk(tint[p][0], tint[p][1], tint[p][2]);
}

void shadePixel(const float* W, const uint32_t* O, const float* C, const float* Hit, const float* Surf, float* Lin,
                int width, int height, int x, int y, Counters* cn) {
  const int b = (y * width + x) * 4;
  V3f rd = primaryDir(C, x, y, width, height), ro = camPos(C), sun = sunDir(C);
  float t = Hit[b];
  int id = int(Hit[b + 1]);
  V3f result = skyColor(rd, sun);
  if (id != -10000) {
    if (cn) cn->v[ORC_SHADED]++;
    V3f p = ro + rd * t, n = mk(Surf[b], Surf[b + 1], Surf[b + 2]);
    int mat = int(Hit[b + 2]), slot = int(Surf[b + 3]);
    float seed = Hit[b + 3];
    LotDesc lot;
    V3f q = p, qn = n;
    float palette = 0.0f;
    if (slot >= 0) {
      lot = loadLot(W, slot);
      int cx, cz;
      slotCell(O, slot, cx, cz);
      V3f cp = mk(float(cx) * kCell, 0.0f, float(cz) * kCell) + mk(lot.ox, 0.0f, lot.oz);
      q = toLot(p - cp, lot.turn);
      qn = toLot(n, lot.turn);
      palette = lot.palette;
    } else {  // ground: paving inside the lot, asphalt outside, water on canals
      int cx = int(std::floor((p.x + 18.0f) / kCell)), cz = int(std::floor((p.z + 18.0f) / kCell));
      slot = tableSlot(O, cx, cz);
      lot = loadLot(W, slot);
      q = p - mk(float(cx) * kCell, 0.0f, float(cz) * kCell);
      seed = lot.seed;
      mat = std::fabs(q.x) < 16.5f && std::fabs(q.z) < 16.5f ? 11 : 10;
      if (lot.type == 5) mat = 9;
    }
    if (cn && (mat == 0 || mat == 1)) cn->v[ORC_SHADED_MASONRY]++;
    if (mat == 7 && dot(n, rd) > 0.0f) { n = n * -1.0f; qn = qn * -1.0f; }
    float footprint = std::fmax(0.00005f, t * 1.08f / float(height));
    float sfp = footprint / std::fmax(0.18f, std::fabs(dot(n, rd)));
    float u, v;
    masonryUV(q, qn, u, v);
    V3f base = substrateMean(mat);
    if (mat == 0 || mat == 1) base = gNeuralW ? predictSubstrateNet(gNeuralW, u, v, seed, mat) : substrate(u, v, seed, mat);
    V3f albedo = surfaceColor(q, qn, mat, seed, sfp, base) * paletteTint(palette, mat);
    V3f originalN = n;
    if ((mat == 0 || mat == 1) && std::fabs(qn.y) < 0.5f) {
      float eps = std::fmax(0.002f, sfp * 0.6f);
      float du = (masonryHeight(u + eps, v, mat) - masonryHeight(u - eps, v, mat)) / (2.0f * eps);
      float dv = (masonryHeight(u, v + eps, mat) - masonryHeight(u, v - eps, mat)) / (2.0f * eps);
      if (sfp < 0.005f) {
        float me = std::fmax(0.00016f, sfp * 0.8f);
        du += (microRelief(u + me, v, sfp) - microRelief(u - me, v, sfp)) / (2.0f * me);
        dv += (microRelief(u, v + me, sfp) - microRelief(u, v - me, sfp)) / (2.0f * me);
      }
      V3f tangent = std::fabs(qn.x) > 0.5f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
      float fade = freqWeight(sfp, 5.0f);
      V3f localN = unit(qn - tangent * (du * fade) - mk(0.0f, dv * fade, 0.0f));
      n = fromLot(localN, lot.turn);
    }
    if (mat == 9)
      n = unit(n + mk(std::cos(q.x * 3.7f + q.z * 1.1f) * 0.06f, 0.0f, std::sin(q.z * 4.4f - q.x * 0.9f) * 0.08f));
    float nl = std::fmax(0.0f, dot(n, sun)), nv = std::fmax(0.03f, -dot(n, rd));
    float shadow = C[18] > 0.5f ? 1.0f : buildingShadow(W, O, p + originalN * 0.035f, sun, int(C[14]), cn);
    float ao = ambientVisibility(W, O, p), rough = 0.75f;
    if (mat == 3 || mat == 6) rough = 0.38f;
    if (mat == 4) rough = 0.18f;
    if (mat == 9) rough = 0.12f;
    if (mat == 8) rough = 0.3f;
    V3f halfv = unit(sun - rd);
    float nh = std::fmax(0.0f, dot(n, halfv)), vh = std::fmax(0.0f, -dot(rd, halfv));
    float a = rough * rough, denom = nh * nh * (a * a - 1.0f) + 1.0f;
    float distribution = a * a / (kPi * denom * denom + 0.000001f);
    float k = (rough + 1.0f) * (rough + 1.0f) / 8.0f;
    float geometry = nv / (nv * (1.0f - k) + k) * nl / (nl * (1.0f - k) + k + 0.00001f);
    float f0 = mat == 3 || mat == 6 || mat == 8 ? 0.35f : 0.045f;
    float fresnel = f0 + (1.0f - f0) * std::pow(1.0f - vh, 5.0f);
    float spec = distribution * geometry * fresnel / (4.0f * nv * nl + 0.0001f);
    V3f direct = mk(2.25f, 1.72f, 1.18f) * (nl * shadow);
    float skyWeight = 0.22f + 0.29f * sat(n.y * 0.5f + 0.5f);
    V3f ambient = mk(0.25f, 0.34f, 0.44f) * (skyWeight * ao);
    ambient = ambient + mk(0.65f, 0.43f, 0.25f) * ((1.0f - sat(n.y)) * 0.10f * ao);
    result = albedo * (direct + ambient) + mk(1.0f, 0.87f, 0.63f) * (spec * nl * shadow * 2.1f);
    if (mat == 4 || mat == 9) {
      V3f reflection = rd - n * (2.0f * dot(rd, n));
      float fr = 0.10f + 0.72f * std::pow(1.0f - nv, 4.0f);
      result = mix(result, skyColor(reflection, sun) * 0.60f, fr);
      if (mat == 4) {
        float room = hash1(int(seed));
        result = result * 0.73f + mk(0.13f, 0.075f, 0.028f) * (room > 0.78f ? 0.3f : 0.03f);
      }
    }
    if (mat == 8) result = result + mk(1.1f, 0.62f, 0.19f) * 0.8f;
    if (mat == 7) result = result + albedo * (std::pow(std::fmax(0.0f, dot(rd, sun)), 4.0f) * 0.35f);
    float fog = 1.0f - std::exp(-t * 0.00068f);
    fog = lerp(fog, 1.0f, smooth(kFar * 0.68f, kFar, t));
    V3f haze = skyColor(unit(mk(rd.x, 0.004f, rd.z)), sun);
    result = mix(result, haze, fog);
    if (C[11] == 1.0f) result = paletteTint(lot.palette, 0) * mk(0.4f, 0.55f, 0.6f);
    if (C[11] == 2.0f) {
      int g = id >= 0 ? id / kMaxFeatures : 0;
      result = mk(0.15f + 0.75f * hash1(g), 0.15f + 0.75f * hash1(g + 31), 0.15f + 0.75f * hash1(g + 98));
    }
    if (C[11] == 3.0f) result = (n + mk(1.0f, 1.0f, 1.0f)) * 0.5f;
  }
  Lin[b] = result.x; Lin[b + 1] = result.y; Lin[b + 2] = result.z; Lin[b + 3] = 1.0f;
}

inline float aces(float x) { return sat(x * (2.51f * x + 0.03f) / (x * (2.43f * x + 0.59f) + 0.14f)); }
void resolvePixel(const float* Lin, float* Hist, uint32_t* Px, const float* C, const float* Hit, const float* Surf,
                  int width, int height, int x, int y) {  // shade.cu:104-123
  const int b = (y * width + x) * 4;
  V3f c = mk(Lin[b], Lin[b + 1], Lin[b + 2]);
  if (C[11] < 0.5f && int(Hit[b + 1]) != -10000 && Hit[b] < 250.0f) {
    V3f ro = camPos(C), point = ro + primaryDir(C, x, y, width, height) * Hit[b];
    V3f n = mk(Surf[b], Surf[b + 1], Surf[b + 2]);
    float occ = 0.0f;
    float radius = clampv(float(height) / (std::fmax(Hit[b], 0.5f) * 1.08f) * 0.8f, 3.0f, 28.0f);
    for (int k = 0; k < 8; k++) {
      float a = float(k) * kPi * 0.25f + 0.2f;
      int xx = int(clampv(float(x) + angCos(a) * radius, 0.0f, float(width - 1)));
      int yy = int(clampv(float(y) + angSin(a) * radius, 0.0f, float(height - 1)));
      int j = (yy * width + xx) * 4;
      if (int(Hit[j + 1]) != -10000) {
        V3f other = ro + primaryDir(C, xx, yy, width, height) * Hit[j], delta = other - point;
        float l = len(delta);
        if (l > 0.04f && l < 2.0f) occ += std::fmax(0.0f, dot(n, delta / l) - 0.12f) * std::exp(-l * 1.4f) * 0.28f;
      }
    }
    c = c * clampv(1.0f - occ, 0.55f, 1.0f);
  }
  float oldCount = Hist[b + 3], count = C[19] <= 1.0f ? 1.0f : std::fmin(64.0f, oldCount + 1.0f);
  V3f old = mk(Hist[b], Hist[b + 1], Hist[b + 2]);
  if (C[19] >= 64.0f && oldCount >= 64.0f) c = old;
  else c = mix(old, c, 1.0f / count);
  Hist[b] = c.x; Hist[b + 1] = c.y; Hist[b + 2] = c.z; Hist[b + 3] = count;
  float sx = (float(x) / float(width) - 0.5f) * 1.3f, sy = (float(y) / float(height) - 0.5f) * 1.3f;
  c = c * (C[9] * (1.0f - (sx * sx + sy * sy) * 0.12f));
  c = mk(std::pow(aces(c.x), 1.0f / 2.2f), std::pow(aces(c.y), 1.0f / 2.2f), std::pow(aces(c.z), 1.0f / 2.2f));
  Px[y * width + x] = packRGBA8(c);
}

int useThreads(int n) { return n > 0 ? n : omp_get_max_threads(); }

// ---- FP64 re-intersection of a pixel's winning feature ----------------------
// The error bound of a traced frame: the feature a pixel's Hit names is
// regenerated from its lot descriptor (group fid/64, record fid%64, the
// emission of assets.cu:3-265), the pixel's float primary ray (common.cu:63-70)
// is moved into that lot's frame in double precision (trace.cu:49-50), and the
// feature is intersected again by hitFeature<double> (geometry.cu:33-91), its
// normal taken by featNormal<double> (geometry.cu:92-114) at the FP64 hit and,
// to check the normal function apart from the distance, at the float path's
// own hit point.
//
// Foliage (material 7 ellipsoids) is a DDA over leaf discs whose cell sequence
// can differ at a cell boundary in FP64, so the "same feature" there is the
// leaf disc: the 3x3x3 cells around the float hit point are searched for a
// disc of the envelope (geometry.cu:17-26) that the ray crosses in FP64, the
// one nearest the float distance is taken, and its FP64 plane intersection
// and normal are returned.
// Ground hits (fid -1) re-intersect the plane y = 0 (trace.cu:34).
// status = kind | shape << 3 | material << 8 (shape and material of a feature).
enum { RX_SKY = 0, RX_GROUND = 1, RX_FEATURE = 2, RX_LEAF = 3, RX_MISSED = 4 };

static int leafReintersect(const Feat& f, V3<double> ro, V3<double> rd, V3f hitPoint, double tFloat, double& t64,
                           V3<double>& n64) {
  const double cell = double(0.18f);
  const V3<double> centre = cast3<double>(f.p), radius = cast3<double>(f.h);
  const int bx = int(std::floor(hitPoint.x / 0.18f)), by = int(std::floor(hitPoint.y / 0.18f)),
            bz = int(std::floor(hitPoint.z / 0.18f));
  const int seed = int(f.seed);
  double bestGap = 1e30;
  int found = 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int ix = bx + dx, iy = by + dy, iz = bz + dz;
        V3<double> c = mk((double(ix) + 0.5) * cell, (double(iy) + 0.5) * cell, (double(iz) + 0.5) * cell);
        V3<double> q = c - centre;
        double ell = q.x * q.x / (radius.x * radius.x) + q.y * q.y / (radius.y * radius.y) +
                     q.z * q.z / (radius.z * radius.z);
        if (!(ell < 1.0 && hash2(ix + iy * 113, iz, seed) > 0.20f)) continue;
        V3<double> n = leafNormal<double>(ix, iy, iz, seed);
        double den = dot(rd, n);
        if (std::fabs(den) <= 1e-5) continue;
        double u = dot(c - ro, n) / den;
        V3<double> pp = ro + rd * u - c;
        V3<double> tangent = unit(cross(n, mk(0.0, 0.0, 1.0)));
        V3<double> bitangent = cross(n, tangent);
        double a = dot(pp, tangent) / double(0.125f), b = dot(pp, bitangent) / double(0.062f);
        if (!(a * a + b * b < 1.0)) continue;
        double gap = std::fabs(u - tFloat);
        if (gap < bestGap) { bestGap = gap; t64 = u; n64 = n; found = 1; }
      }
  return found;
}

static void reintersectPixel(const float* W, const uint32_t* O, const float* C, const float* Hit, const float* Surf,
                             int width, int height, int x, int y, double* t64, double* n64, int32_t* status) {
  const size_t p = size_t(y) * width + x, b = p * 4;
  const int fid = int(Hit[b + 1]), slot = int(Surf[b + 3]);
  V3f rof = camPos(C), rdf = primaryDir(C, x, y, width, height);
  V3<double> ro = cast3<double>(rof), rd = cast3<double>(rdf);
  t64[p] = double(kFar);
  for (int k = 0; k < 6; k++) n64[p * 6 + k] = k % 3 == 1 ? 1.0 : 0.0;
  if (fid == -1) {
    t64[p] = -ro.y / rd.y;
    status[p] = RX_GROUND;
    return;
  }
  if (fid < 0 || slot < 0 || slot >= kLots) { status[p] = RX_SKY; return; }
  const LotDesc lot = loadLot(W, slot);
  const int group = fid / kMaxFeatures, index = fid % kMaxFeatures;
  Feat f{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f};
  forEachFeature(lot, group, [&](const Feat& ft, int id) { if (id == index) f = ft; });
  const int32_t kind = ((f.shape & 15) << 3) | (f.material << 8);
  int cx, cz;
  slotCell(O, slot, cx, cz);
  const V3<double> cp = mk(double(cx) * double(kCell) + double(lot.ox), 0.0, double(cz) * double(kCell) + double(lot.oz));
  const V3<double> lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
  // the float path's lot-frame ray, exactly as the trace forms it
  const V3f cpf = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
  const V3f lrf = toLot(rof - cpf, lot.turn), ldf = toLot(rdf, lot.turn);
  if (f.shape == 1 && f.material == 7) {
    const float tf = Hit[b];
    V3<double> n;
    double t;
    if (leafReintersect(f, lr, ld, lrf + ldf * tf, double(tf), t, n)) {
      t64[p] = t;
      n = fromLot(n, lot.turn);
      n64[p * 6] = n.x; n64[p * 6 + 1] = n.y; n64[p * 6 + 2] = n.z;
      n64[p * 6 + 3] = n.x; n64[p * 6 + 4] = n.y; n64[p * 6 + 5] = n.z;
      status[p] = RX_LEAF | kind;
    } else {
      status[p] = RX_MISSED | kind;
    }
    return;
  }
  const double cone = double(1.08f / float(height));
  const double t = hitFeature<double>(f, lr, ld, cone, nullptr);
  if (!(t < double(kFar))) { status[p] = RX_MISSED | kind; return; }
  const V3<double> n = fromLot(featNormal<double>(f, lr + ld * t), lot.turn);
  t64[p] = t;
  n64[p * 6] = n.x; n64[p * 6 + 1] = n.y; n64[p * 6 + 2] = n.z;
  // the normal function alone: featNormal in FP64 at the float path's own hit point
  const V3<double> nf = fromLot(featNormal<double>(f, cast3<double>(lrf + ldf * Hit[b])), lot.turn);
  n64[p * 6 + 3] = nf.x; n64[p * 6 + 4] = nf.y; n64[p * 6 + 5] = nf.z;
  status[p] = RX_FEATURE | kind;
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_setAngleRounding(int mode) { gAngleMode = mode ? 1 : 0; }
void orc_cameraBasis(const float* C, float* out6) {
  V3f f = camForward(C), r = camRight(C);
  out6[0] = f.x; out6[1] = f.y; out6[2] = f.z; out6[3] = r.x; out6[4] = r.y; out6[5] = r.z;
}
int orc_angleRounding(void) { return gAngleMode; }
void orc_offset_tag(const uint32_t* origin, int dx, int dz, uint32_t* out) {
  Addr a = shiftAddr(origin, dx, dz);
  out[0] = a.xl; out[1] = a.xh; out[2] = a.zl; out[3] = a.zh;
}
uint32_t orc_tag_hash(const uint32_t* t, int seed) { return addrKey(Addr{t[0], t[1], t[2], t[3]}, seed); }
uint32_t orc_hashU(uint32_t x) { return mixbits(x); }
void orc_describe_lot(const uint32_t* t, int seed, float* out) { storeLot(describe(Addr{t[0], t[1], t[2], t[3]}, seed), out); }

// world.cu:57-63
void orc_initCamera(float* C, uint32_t* O, int seed) {
  for (int i = 0; i < 64; i++) C[i] = 0.0f;
  for (int i = 0; i < 4; i++) O[i] = 0u;
  C[0] = 112.0f; C[1] = 76.0f; C[2] = 155.0f; C[3] = -2.53f; C[4] = -0.30f;
  C[7] = -0.55f; C[8] = 0.45f; C[9] = 0.93f; C[10] = 0.28f; C[12] = 38.0f;
  C[14] = float(seed); C[15] = 1.0f; C[19] = 1.0f; C[30] = 1.0f;
}
// world.cu:64-92
void orc_stepCamera(float* C, uint32_t* O, const float* I, float dt, int width, int height) {
  C[5] += dt; C[6] += 1.0f; C[13] = float(height); C[20] = float(width) / float(height);
  C[15] = I[23] > 0.5f ? 1.0f : 0.0f;
  int bm = int(I[8]);
  if (bm > 0) {
    for (int i = 0; i < 4; i++) O[i] = 0u;
    if (bm == 1) { C[0] = 112.0f; C[1] = 76.0f; C[2] = 155.0f; C[3] = -2.53f; C[4] = -0.30f; C[12] = 38.0f; }
    if (bm == 2) { C[0] = 18.0f; C[1] = 1.75f; C[2] = 49.0f; C[3] = -2.80f; C[4] = 0.17f; C[12] = 6.0f; }
    if (bm == 3 || bm == 6) { C[0] = 17.0f; C[1] = 6.9f; C[2] = 0.0f; C[3] = -kPi * 0.5f; C[4] = 0.015f; C[12] = 0.8f; }
    if (bm == 4) { C[0] = 400.0f; C[1] = 650.0f; C[2] = 750.0f; C[3] = -2.61f; C[4] = -0.66f; C[12] = 180.0f; }
    if (bm == 5) { C[0] = 28.0f * kCell + 20.0f; C[1] = 8.0f; C[2] = 75.0f; C[3] = -2.65f; C[4] = -0.04f; C[12] = 12.0f; }
    C[15] = 1.0f;
  }
  if (I[3] != 0.0f || I[4] != 0.0f) {
    C[3] += I[3] * 0.0022f;
    C[4] = clampv(C[4] - I[4] * 0.0022f, -1.53f, 1.53f);
    C[15] = 1.0f;
  }
  if (I[7] != 0.0f) C[12] = clampv(C[12] * std::exp(-I[7] * 0.0015f), 0.03f, 800.0f);
  float speed = C[12] * (I[5] > 0.5f ? 3.0f : 1.0f) * (I[6] > 0.5f ? 0.15f : 1.0f);
  V3f move = camForward(C) * I[0] + camRight(C) * I[1] + mk(0.0f, I[2], 0.0f);
  if (dot(move, move) > 0.0f) {
    move = unit(move) * speed * dt;
    C[0] += move.x; C[1] = clampv(C[1] + move.y, 0.08f, 1500.0f); C[2] += move.z; C[15] = 1.0f;
  }
  if (I[9] != 0.0f) { C[7] += I[9] * dt * 0.35f; C[15] = 1.0f; }
  if (I[10] > 0.0f) { C[11] = float((int(C[11]) + 1) % 4); C[15] = 1.0f; }
  if (I[13] != 0.0f) { C[9] = clampv(C[9] + I[13] * dt, 0.25f, 3.0f); C[15] = 1.0f; }
  if (I[14] > 0.0f) { C[18] = 1.0f - C[18]; C[15] = 1.0f; }
  if (I[16] > 0.0f) C[22] = 1.0f - C[22];
  if (C[22] > 0.5f) {
    C[3] += dt * 0.032f;
    V3f f = camForward(C);
    C[0] += f.x * dt * 14.0f; C[2] += f.z * dt * 14.0f; C[15] = 1.0f;
  }
  int dx = int(std::floor((C[0] + 18.0f) / kCell)), dz = int(std::floor((C[2] + 18.0f) / kCell));
  if (dx != 0 || dz != 0) {
    Addr a = shiftAddr(O, dx, dz);
    O[0] = a.xl; O[1] = a.xh; O[2] = a.zl; O[3] = a.zh;
    C[0] -= float(dx) * kCell; C[2] -= float(dz) * kCell;
  }
  C[19] = C[15] > 0.5f ? 1.0f : std::fmin(64.0f, C[19] + 1.0f);
}
void orc_clearQueue(uint32_t* Q) { Q[0] = 0u; }
// world.cu:94-105, serial in slot order
void orc_prepareLots(const uint32_t* O, const float* C, float* W, uint32_t* T, uint32_t* Q) {
  for (int slot = 0; slot < kLots; slot++) {
    int cx, cz;
    slotCell(O, slot, cx, cz);
    Addr a = shiftAddr(O, cx, cz);
    float* w = W + slot * kLotFloats;
    uint32_t* t = T + slot * 4;
    if (w[15] > 0.5f && t[0] == a.xl && t[1] == a.xh && t[2] == a.zl && t[3] == a.zh) continue;
    LotDesc l = describe(a, int(C[14]));
    float keep13 = w[13], keep14 = w[14];
    storeLot(l, w);
    w[13] = keep13; w[14] = keep14;  // the reference leaves these two words untouched
    t[0] = a.xl; t[1] = a.xh; t[2] = a.zl; t[3] = a.zh;
    uint32_t i = Q[0]++;
    Q[i + 1] = uint32_t(slot);
  }
}
// world.cu:106-111
void orc_planBounds(const uint32_t* Q, uint32_t* A) {
  for (int chunk = 0; chunk < kChunks; chunk++) {
    int count = int(Q[0]) - chunk * kChunk;
    count = count < 0 ? 0 : (count > kChunk ? kChunk : count);
    uint32_t* a = A + chunk * 21;
    a[0] = uint32_t(count); a[1] = 1u; a[2] = 1u;
    int level = 1;
    for (int first = 32; first >= 1; first /= 2, level++) {
      a[level * 3] = uint32_t((count * first + 63) / 64); a[level * 3 + 1] = 1u; a[level * 3 + 2] = 1u;
    }
  }
}
void orc_buildBounds(const uint32_t* Q, const float* W, float* N, int nthreads) {
  const int count = int(Q[0]);
#pragma omp parallel for schedule(dynamic, 8) num_threads(useThreads(nthreads))
  for (int q = 0; q < count; q++) {
    int slot = int(Q[q + 1]);
    lotHierarchy(loadLot(W, slot), N + size_t(slot) * kNodes * 8);
  }
}

int orc_enumerate(const float* lot16, int group, float* out, int cap) {
  LotDesc l = loadLot(lot16, 0);
  return forEachFeature(l, group, [&](const Feat& f, int id) { if (id < cap) putFeat(f, out + 10 * id); });
}
void orc_group_bounds(const float* lot16, int group, float* o7) { groupBounds(loadLot(lot16, 0), group, o7); }
float orc_featureHit(const float* f10, const float* ro, const float* rd, float cone) {
  return hitFeature<float>(getFeat(f10), mk(ro[0], ro[1], ro[2]), mk(rd[0], rd[1], rd[2]), cone, nullptr);
}
void orc_featureNormal(const float* f10, const float* pt, float* n) {
  V3f r = featNormal<float>(getFeat(f10), mk(pt[0], pt[1], pt[2]));
  n[0] = r.x; n[1] = r.y; n[2] = r.z;
}
double orc_featureHit_f64(const float* f10, const double* ro, const double* rd, double cone) {
  return hitFeature<double>(getFeat(f10), mk(ro[0], ro[1], ro[2]), mk(rd[0], rd[1], rd[2]), cone, nullptr);
}
void orc_featureNormal_f64(const float* f10, const double* pt, double* n) {
  V3<double> r = featNormal<double>(getFeat(f10), mk(pt[0], pt[1], pt[2]));
  n[0] = r.x; n[1] = r.y; n[2] = r.z;
}
float orc_queryLot(const float* lot16, const float* nodes, const float* ro, const float* rd, float best, float cone,
                   int* fid, float* f10) {
  Nearest h = queryLotNearest(loadLot(lot16, 0), nodes, 0, mk(ro[0], ro[1], ro[2]), mk(rd[0], rd[1], rd[2]), best,
                              cone, nullptr, nullptr);
  *fid = h.fid;
  putFeat(h.f, f10);
  return h.t;
}
// Every group of the lot, no node culling: the "exhaustive" side of the
// hierarchy-vs-exhaustive check.  Groups in index order, first wins on ties.
float orc_queryLot_exhaustive(const float* lot16, const float* ro, const float* rd, float best, float cone, int* fid,
                              float* f10) {
  LotDesc l = loadLot(lot16, 0);
  V3f o = mk(ro[0], ro[1], ro[2]), d = mk(rd[0], rd[1], rd[2]);
  float bt = best;
  int bf = -1;
  Feat bfeat{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f};
  for (int g = 0; g < kGroups; g++) {
    float t; int id; Feat f;
    groupNearest(l, g, o, d, cone, bt, t, id, f, nullptr, nullptr);
    if (id >= 0 && t < bt) { bt = t; bf = g * kMaxFeatures + id; bfeat = f; }
  }
  *fid = bf;
  putFeat(bfeat, f10);
  return bt;
}

void orc_tracePrimary(const float* W, const float* N, const uint32_t* O, const float* C, float* Hit, float* Surf,
                      int width, int height, int rowStart, int rowCount, int nthreads, int64_t* counters,
                      float* second) {
  Counters total;
  const int yEnd = std::min(height, rowStart + rowCount);
#pragma omp parallel num_threads(useThreads(nthreads))
  {
    Counters local;
#pragma omp for schedule(dynamic, 2)
    for (int y = rowStart; y < yEnd; y++)
      for (int x = 0; x < width; x++) tracePixel(W, N, O, C, Hit, Surf, width, height, x, y, counters ? &local : nullptr, second);
#pragma omp critical
    for (int i = 0; i < ORC_COUNTERS; i++) total.v[i] += local.v[i];
  }
  if (counters)
    for (int i = 0; i < ORC_COUNTERS; i++) counters[i] += total.v[i];
}
void orc_shadePixels(const float* W, const uint32_t* O, const float* C, const float* Hit, const float* Surf, float* Lin,
                     int width, int height, int rowStart, int rowCount, int nthreads, int64_t* counters) {
  Counters total;
  const int yEnd = std::min(height, rowStart + rowCount);
#pragma omp parallel num_threads(useThreads(nthreads))
  {
    Counters local;
#pragma omp for schedule(dynamic, 2)
    for (int y = rowStart; y < yEnd; y++)
      for (int x = 0; x < width; x++) shadePixel(W, O, C, Hit, Surf, Lin, width, height, x, y, counters ? &local : nullptr);
#pragma omp critical
    for (int i = 0; i < ORC_COUNTERS; i++) total.v[i] += local.v[i];
  }
  if (counters)
    for (int i = 0; i < ORC_COUNTERS; i++) counters[i] += total.v[i];
}
void orc_resolveFrame(const float* Lin, float* Hist, uint32_t* Px, const float* C, const float* Hit, const float* Surf,
                      int width, int height, int nthreads) {
#pragma omp parallel for schedule(dynamic, 2) num_threads(useThreads(nthreads))
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) resolvePixel(Lin, Hist, Px, C, Hit, Surf, width, height, x, y);
}
void orc_traceRays(const float* W, const float* N, const uint32_t* O, const float* rays, int n, int exhaustive,
                   float* out, int nthreads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(useThreads(nthreads))
  for (int i = 0; i < n; i++) {
    const float* q = rays + size_t(i) * 7;
    traceRayOrc(W, N, O, mk(q[0], q[1], q[2]), mk(q[3], q[4], q[5]), q[6], exhaustive != 0, out + size_t(i) * 8);
  }
}
// learning.cu:5-10
void orc_initNeural(float* W, float* M, float* V, float* Brain, int seed) {
  for (int i = 0; i < kNnParams; i++) {
    W[i] = (hash1(i + seed) - 0.5f) * 0.08f;
    M[i] = 0.0f;
    V[i] = 0.0f;
    if (i >= kNnW2) W[i] = 0.0f;
  }
  for (int i = 0; i < 32; i++) Brain[i] = 0.0f;
  W[kNnB2] = 0.36f; W[kNnB2 + 1] = 0.29f; W[kNnB2 + 2] = 0.20f;
}
// learning.cu:11-58, the five kernels in order; the sample's inputs come from
// the current buffers (Hit material and seed, the lot-frame masonry
// coordinates of shade.cu:54-65).
void orc_materialStep(const float* Wd, const uint32_t* O, const float* C, const float* Hit, const float* Surf,
                      float* W, float* M, float* V, float* Brain, float* WorkOut, int width, int height) {
  if (!materialTrainNow(C)) return;
  std::vector<float> work(kNnBatch * kNnWs, 0.0f);
  const V3f ro = camPos(C);
  for (int i = 0; i < kNnBatch; i++) {  // prepareMaterialBatch
    float* w = work.data() + i * kNnWs;
    int chosen = -1;
    for (int trial = 0; trial < 6; trial++) {
      const int px = int(hash1(i * 1877 + trial * 331 + int(C[6]) * 59) * float(width * height));
      const int id = int(Hit[px * 4 + 1]);
      if (id >= 0) {
        const int mat = int(Hit[px * 4 + 2]);
        if (mat == 0 || mat == 1) chosen = px;
      }
    }
    if (chosen < 0) continue;
    const int b = chosen * 4, x = chosen % width, y = chosen / width;
    const V3f rd = primaryDir(C, x, y, width, height);
    const V3f pt = ro + rd * Hit[b], n = mk(Surf[b], Surf[b + 1], Surf[b + 2]);
    const int mat = int(Hit[b + 2]), slot = int(Surf[b + 3]);
    const float seed = Hit[b + 3];
    const LotDesc lot = loadLot(Wd, slot);
    int cx, cz;
    slotCell(O, slot, cx, cz);
    const V3f cp = mk(float(cx) * kCell, 0.0f, float(cz) * kCell) + mk(lot.ox, 0.0f, lot.oz);
    V3f q = toLot(pt - cp, lot.turn), qn = toLot(n, lot.turn);
    float u, v;
    masonryUV(q, qn, u, v);
    for (int j = 0; j < kNnInputs; j++) w[j] = nnFeature(j, u, v, seed, mat);
    const V3f target = substrate(u, v, seed, mat);
    w[kNnTarget] = target.x; w[kNnTarget + 1] = target.y; w[kNnTarget + 2] = target.z;
    w[kNnValid] = 1.0f;
    w[kNnMat] = float(mat);
  }
  for (int i = 0; i < kNnBatch; i++) {  // materialForward
    float* w = work.data() + i * kNnWs;
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
  {  // scoreMaterial
    float err = 0.0f, baseline = 0.0f, n = 0.0f;
    for (int k = kNnTrain; k < kNnBatch; k++) {
      const float* w = work.data() + k * kNnWs;
      if (w[kNnValid] > 0.5f) {
        n += 1.0f;
        const V3f mean = substrateMean(int(w[kNnMat]));
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
  float grad[kNnParams];
  float count = 0.0f;
  for (int i = 0; i < kNnParams; i++) {  // materialGradient
    float g = 0.0f;
    count = 0.0f;
    for (int k = 0; k < kNnTrain; k++) {
      const float* w = work.data() + k * kNnWs;
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
    grad[i] = clampv(g / std::fmax(1.0f, count), -0.8f, 0.8f);
  }
  if (count > 0.0f) Brain[0] += 1.0f;
  Brain[5] = count;
  if (Brain[5] >= 1.0f)  // materialAdam
    for (int i = 0; i < kNnParams; i++) {
      const float g = grad[i];
      const float m = 0.9f * M[i] + 0.1f * g, v = 0.999f * V[i] + 0.001f * g * g;
      M[i] = m;
      V[i] = v;
      const float mh = m / (1.0f - angPow(0.9f, Brain[0])), vh = v / (1.0f - angPow(0.999f, Brain[0]));
      W[i] -= 0.002f * (mh / (std::sqrt(vh) + 0.00001f) + 0.0001f * W[i]);
    }
  if (WorkOut) std::memcpy(WorkOut, work.data(), sizeof(float) * work.size());
}
void orc_predictSubstrate(const float* W, const float* Q, int n, float* out) {
  for (int i = 0; i < n; i++) {
    const V3f c = predictSubstrateNet(W, Q[i * 4], Q[i * 4 + 1], Q[i * 4 + 2], int(Q[i * 4 + 3]));
    out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z;
  }
}
// shadePixels with the surrogate when C[16] > 0.5 and Brain[4] > 0.5 (Stratum.cu:854).
void orc_shadePixelsNeural(const float* Wd, const uint32_t* O, const float* C, const float* Hit, const float* Surf,
                           float* Lin, const float* W, const float* Brain, int width, int height, int rowStart,
                           int rowCount, int nthreads) {
  gNeuralW = C[16] > 0.5f && Brain[4] > 0.5f ? W : nullptr;
  orc_shadePixels(Wd, O, C, Hit, Surf, Lin, width, height, rowStart, rowCount, nthreads, nullptr);
  gNeuralW = nullptr;
}
// trace, shade and resolve of the listed rows only, in parallel over pixels.
void orc_renderRows(const float* W, const float* N, const uint32_t* O, const float* C, float* Hit, float* Surf,
                    float* Lin, float* Hist, uint32_t* Px, int width, int height, const int32_t* rows, int nrows,
                    int nthreads) {
  const long n = long(nrows) * width;
#pragma omp parallel for schedule(dynamic, 64) num_threads(useThreads(nthreads))
  for (long i = 0; i < n; i++) tracePixel(W, N, O, C, Hit, Surf, width, height, int(i % width), rows[i / width], nullptr, nullptr);
#pragma omp parallel for schedule(dynamic, 64) num_threads(useThreads(nthreads))
  for (long i = 0; i < n; i++) shadePixel(W, O, C, Hit, Surf, Lin, width, height, int(i % width), rows[i / width], nullptr);
#pragma omp parallel for schedule(dynamic, 64) num_threads(useThreads(nthreads))
  for (long i = 0; i < n; i++) resolvePixel(Lin, Hist, Px, C, Hit, Surf, width, height, int(i % width), rows[i / width]);
}
// One named (slot, fid) feature per ray, intersected in its lot frame as the
// trace forms it (world.cu:37-56, sink.cu:21, geometry.cu:33-114).
void orc_retestFeatures(const float* W, const uint32_t* O, const float* rays, const int32_t* ids, int n, float* out,
                        int nthreads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(useThreads(nthreads))
  for (int i = 0; i < n; i++) {
    const float* q = rays + size_t(i) * 7;
    const int slot = ids[2 * i], fid = ids[2 * i + 1];
    float* o = out + size_t(i) * 4;
    o[0] = kFar; o[1] = o[2] = o[3] = 0.0f;
    if (slot < 0 || slot >= kLots || fid < 0 || fid >= kGroups * kMaxFeatures) continue;
    const LotDesc lot = loadLot(W, slot);
    int cx, cz;
    slotCell(O, slot, cx, cz);
    const V3f ro = mk(q[0], q[1], q[2]), rd = mk(q[3], q[4], q[5]);
    const V3f cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
    const V3f lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
    Feat f{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f};
    forEachFeature(lot, fid / kMaxFeatures, [&](const Feat& ft, int id) { if (id == fid % kMaxFeatures) f = ft; });
    if (f.shape < 0) continue;
    const float t = hitFeature<float>(f, lr, ld, q[6], nullptr);
    if (!(t > 0.001f && t < kFar)) continue;
    const V3f nn = fromLot(featNormal<float>(f, lr + ld * t), lot.turn);
    o[0] = t; o[1] = nn.x; o[2] = nn.y; o[3] = nn.z;
  }
}
void orc_reintersectF64(const float* W, const uint32_t* O, const float* C, const float* Hit, const float* Surf,
                        int width, int height, double* t64, double* n64, int32_t* status, int nthreads) {
#pragma omp parallel for schedule(dynamic, 2) num_threads(useThreads(nthreads))
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) reintersectPixel(W, O, C, Hit, Surf, width, height, x, y, t64, n64, status);
}
void orc_resolveRows(const float* Lin, float* Hist, uint32_t* Px, const float* C, const float* Hit, const float* Surf,
                     int width, int height, int rowStart, int rowCount, int nthreads) {
  const int yEnd = std::min(height, rowStart + rowCount);
#pragma omp parallel for schedule(dynamic, 2) num_threads(useThreads(nthreads))
  for (int y = rowStart; y < yEnd; y++)
    for (int x = 0; x < width; x++) resolvePixel(Lin, Hist, Px, C, Hit, Surf, width, height, x, y);
}
// probe.cu:2-14
void orc_probeGrammar(const float* in, float* out) {
  LotDesc l;
  int g = int(in[0]), index = int(in[1]);
  l.w = in[2]; l.d = in[3]; l.h = in[4]; l.type = int(in[5]); l.mat = int(in[6]); l.floors = int(in[7]);
  l.seed = in[8]; l.storey = in[9]; l.roofScale = in[10]; l.turn = 0; l.ox = 0.0f; l.oz = 0.0f; l.palette = 0.0f;
  Feat pick{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f};
  int count = forEachFeature(l, g, [&](const Feat& f, int id) { if (id == index) pick = f; });
  out[0] = float(count); out[1] = float(pick.shape); out[2] = float(pick.material); out[3] = pick.seed;
  out[4] = pick.p.x; out[5] = pick.p.y; out[6] = pick.p.z; out[7] = pick.h.x; out[8] = pick.h.y; out[9] = pick.h.z;
  out[10] = float(pick.turn);
  V3f ro = mk(in[11], in[12], in[13]), rd = mk(in[14], in[15], in[16]);
  float t; int fid; Feat f;
  groupNearest(l, g, ro, rd, 0.0f, kFar, t, fid, f, nullptr, nullptr);
  out[11] = t; out[12] = float(fid);
  V3f n = mk(0.0f, 0.0f, 0.0f);
  if (fid >= 0) n = featNormal<float>(f, ro + rd * t);
  out[13] = n.x; out[14] = n.y; out[15] = n.z;
}

}  // extern "C"
