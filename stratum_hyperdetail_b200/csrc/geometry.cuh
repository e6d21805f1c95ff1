// Analytic ray-feature intersection and normals (kernels/geometry.cu of the
// reference): box, ellipsoid, capped cylinder, triangular prism, half arch and
// full ring, leaf discs inside foliage envelopes, and the bounded masonry
// relief correction.  Shape branches are written so a warp whose lanes test
// the same feature takes one path.
#pragma once
#include "grammar.cuh"

namespace st {

SD f3 intoFeature(f3 p, int turn) { return (turn % 2 == 1) ? mk(p.z, p.y, -p.x) : p; }
SD f3 outOfFeature(f3 p, int turn) { return (turn % 2 == 1) ? mk(-p.z, p.y, p.x) : p; }

SD f3 leafNormal(int x, int y, int z, int seed) {  // geometry.cu:6-8
  return unit(mk(hash2(x + y * 19, z, seed) - 0.5f, 0.25f + hash2(x - y, z + 91, seed) * 0.7f,
                 hash2(z + y * 31, x, seed + 17) - 0.5f));
}

// Leaf discs on a 0.18 m grid inside the envelope, <= 48 cells (geometry.cu:9-31).
static __device__ __noinline__ float foliageHit(f3 ro, f3 rd, f3 centre, f3 radius, int seed, float begin, float end) {
  const float cell = 0.18f;
  float t = fmaxf(0.001f, begin) + 0.0001f;
  f3 pos = ro + rd * t;
  int ix = int(floorf(pos.x / cell)), iy = int(floorf(pos.y / cell)), iz = int(floorf(pos.z / cell));
  int sx = rd.x > 0.0f ? 1 : -1, sy = rd.y > 0.0f ? 1 : -1, sz = rd.z > 0.0f ? 1 : -1;
  f3 inv = invDir(rd);
  float tx = (float(ix + (sx > 0 ? 1 : 0)) * cell - ro.x) * inv.x;
  float ty = (float(iy + (sy > 0 ? 1 : 0)) * cell - ro.y) * inv.y;
  float tz = (float(iz + (sz > 0 ? 1 : 0)) * cell - ro.z) * inv.z;
  float dx = cell * fabsf(inv.x), dy = cell * fabsf(inv.y), dz = cell * fabsf(inv.z);
  const float rx2 = radius.x * radius.x, ry2 = radius.y * radius.y, rz2 = radius.z * radius.z;
#pragma unroll 1
  for (int k = 0; k < 48; k++) {
    if (t > end) break;
    float exitT = fminf(tx, fminf(ty, tz));
    f3 c = mk((float(ix) + 0.5f) * cell, (float(iy) + 0.5f) * cell, (float(iz) + 0.5f) * cell);
    f3 q = c - centre;
    float ell = q.x * q.x / rx2 + q.y * q.y / ry2 + q.z * q.z / rz2;
    if (ell < 1.0f && hash2(ix + iy * 113, iz, seed) > 0.20f) {
      f3 n = leafNormal(ix, iy, iz, seed);
      float den = dot(rd, n);
      if (fabsf(den) > 0.00001f) {
        float u = dot(c - ro, n) / den;
        if (u >= t && u <= exitT) {
          f3 pp = ro + rd * u - c;
          f3 tangent = unit(cross(n, mk(0.0f, 0.0f, 1.0f)));
          f3 bitangent = cross(n, tangent);
          float a = dot(pp, tangent) / 0.125f, b = dot(pp, bitangent) / 0.062f;
          if (a * a + b * b < 1.0f) return u;
        }
      }
    }
    if (tx < ty && tx < tz) { t = tx; tx += dx; ix += sx; }
    else if (ty < tz) { t = ty; ty += dy; iy += sy; }
    else { t = tz; tz += dz; iz += sz; }
  }
  return kFar;
}

// Four fixed-point steps of the ray against the mortar height field
// (geometry.cu:82-89).  Called only for tall stone/brick boxes.
static __device__ __noinline__ float masonryRelief(Feat f, f3 ro, f3 rd, f3 p, f3 d, float t, float cone) {
  const f3 h = f.h;
  f3 hp = p + d * t;
  float ex = fabsf(fabsf(hp.x) - h.x), ez = fabsf(fabsf(hp.z) - h.z);
  if (fabsf(fabsf(hp.y) - h.y) > 0.01f) {
    f3 n = ex < ez ? mk(hp.x < 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f) : mk(0.0f, 0.0f, hp.z < 0.0f ? -1.0f : 1.0f);
    float denom = dot(n, d);
    if (denom < -0.08f) {
      float initial = t;
      f3 wn = outOfFeature(n, f.turn);
#pragma unroll 1
      for (int k = 0; k < 4; k++) {
        f3 wp = ro + rd * t;
        float u, v;
        masonryUV(wp, wn, u, v);
        float disp = masonryHeight(u, v, f.material) * freqWeight(t * cone, 40.0f);
        t = initial + disp / denom;
      }
    }
  }
  return t;
}

// Nearest positive hit of one feature, kFar if none (geometry.cu:33-91).
// `p`, `d` are the ray in the feature's frame and `inv` = invDir(d); callers
// that test many features against one ray pass them precomputed.
SD float featureHitCore(const Feat& f, f3 ro, f3 rd, f3 p, f3 d, f3 inv, float cone) {
  const int shape = f.shape;
  if (shape < 0) return kFar;
  const f3 h = f.h;
  Span range = (shape == 3 || shape == 4) ? slabInv(p, inv, mk(-h.x, 0.0f, -h.z), h) : slabInv(p, inv, h * -1.0f, h);
  if (range.hi < fmaxf(0.001f, range.lo)) return kFar;
  float t = range.lo > 0.001f ? range.lo : range.hi;
  if (shape == 1) {  // ellipsoid
    f3 a = mk(p.x / h.x, p.y / h.y, p.z / h.z), v = mk(d.x / h.x, d.y / h.y, d.z / h.z);
    float aa = dot(v, v), bb = dot(a, v), cc = dot(a, a) - 1.0f, disc = bb * bb - aa * cc;
    if (disc < 0.0f) return kFar;
    float sq = sqrtf(disc);
    t = (-bb - sq) / aa;
    if (t <= 0.001f) t = (-bb + sq) / aa;
    if (f.material == 7 && t < kFar) t = foliageHit(ro, rd, f.p, h, int(f.seed), range.lo, range.hi);
  } else if (shape == 2) {  // capped vertical cylinder
    const float hx2 = h.x * h.x, hz2 = h.z * h.z;
    float a = d.x * d.x / hx2 + d.z * d.z / hz2;
    float bb = p.x * d.x / hx2 + p.z * d.z / hz2;
    float cc = p.x * p.x / hx2 + p.z * p.z / hz2 - 1.0f;
    float best = kFar, disc = bb * bb - a * cc;
    if (disc >= 0.0f && a > 0.0000001f) {
      float sq = sqrtf(disc);
      float u = (-bb - sq) / a, v = (-bb + sq) / a;
      if (u > 0.001f && fabsf(p.y + d.y * u) <= h.y) best = u;
      if (v > 0.001f && fabsf(p.y + d.y * v) <= h.y) best = fminf(best, v);
    }
    if (fabsf(d.y) > 0.000001f) {
#pragma unroll
      for (int k = 0; k < 2; k++) {
        float cy = k == 0 ? -h.y : h.y, u = (cy - p.y) / d.y;
        float xx = (p.x + d.x * u) / h.x, zz = (p.z + d.z * u) / h.z;
        if (u > 0.001f && xx * xx + zz * zz <= 1.0f) best = fminf(best, u);
      }
    }
    t = best;
  } else if (shape == 3) {  // triangular prism: box interval clipped by two roof planes
    float nearT = fmaxf(0.001f, range.lo), farT = range.hi;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      float sg = k == 0 ? 1.0f : -1.0f;
      float numer = h.y - (p.y + sg * p.x * h.y / h.x), denom = d.y + sg * d.x * h.y / h.x;
      if (fabsf(denom) < 0.000001f) { if (numer < 0.0f) return kFar; }
      else { float u = numer / denom; if (denom > 0.0f) farT = fminf(farT, u); else nearT = fmaxf(nearT, u); }
    }
    if (farT < nearT) return kFar;
    t = nearT;
  } else if (shape == 4 || shape == 7) {  // half arch / full ring, radii 1 and 0.77
    const float hx2 = h.x * h.x, hy2 = h.y * h.y;
    float best = kFar;
    float a = d.x * d.x / hx2 + d.y * d.y / hy2;
    float bb = p.x * d.x / hx2 + p.y * d.y / hy2;
    float pq = p.x * p.x / hx2 + p.y * p.y / hy2;
#pragma unroll
    for (int ring = 0; ring < 2; ring++) {
      float rad = ring == 0 ? 1.0f : 0.77f;
      float cc = pq - rad * rad, disc = bb * bb - a * cc;
      if (disc >= 0.0f && a > 0.000001f) {
        float sq = sqrtf(disc);
#pragma unroll
        for (int k = 0; k < 2; k++) {
          float u = (-bb + (k == 0 ? -sq : sq)) / a;
          if (u > 0.001f && fabsf(p.z + d.z * u) <= h.z && (shape == 7 || p.y + d.y * u >= 0.0f)) best = fminf(best, u);
        }
      }
    }
    if (fabsf(d.z) > 0.000001f) {
#pragma unroll
      for (int k = 0; k < 2; k++) {
        float u = ((k == 0 ? -h.z : h.z) - p.z) / d.z;
        float xx = (p.x + d.x * u) / h.x, yy = (p.y + d.y * u) / h.y, rr = xx * xx + yy * yy;
        if (u > 0.001f && rr <= 1.0f && rr >= 0.77f * 0.77f && (shape == 7 || yy >= 0.0f)) best = fminf(best, u);
      }
    }
    t = best;
  }
  if (t <= 0.001f) return kFar;
  if (shape == 0 && (f.material == 0 || f.material == 1) && h.y > 1.0f) t = masonryRelief(f, ro, rd, p, d, t, cone);
  return t;
}
SD float featureHit(const Feat& f, f3 ro, f3 rd, float cone) {
  const f3 d = intoFeature(rd, f.turn);
  return featureHitCore(f, ro, rd, intoFeature(ro - f.p, f.turn), d, invDir(d), cone);
}

// featureHitCore split for hot loops: the slab test every feature starts with
// (geometry.cu:37-38) stays inline; what follows a passed slab test is out of
// line except for plain boxes, so the loop over features stays small in the
// instruction cache.  featureSlabMiss + featureAfterSlab == featureHitCore.
SD Span featureSlab(const Feat& f, f3 p, f3 inv) {
  const f3 h = f.h;
  return (f.shape == 3 || f.shape == 4) ? slabInv(p, inv, mk(-h.x, 0.0f, -h.z), h) : slabInv(p, inv, h * -1.0f, h);
}
SD bool featureSlabMiss(const Feat& f, Span range) { return f.shape < 0 || range.hi < fmaxf(0.001f, range.lo); }
static __device__ __noinline__ float featureAfterSlabOOL(Feat f, f3 ro, f3 rd, f3 p, f3 d, f3 inv, float cone) {
  return featureHitCore(f, ro, rd, p, d, inv, cone);
}
SD float featureAfterSlab(const Feat& f, f3 ro, f3 rd, f3 p, f3 d, f3 inv, Span range, float cone) {
  if (f.shape == 0 && !((f.material == 0 || f.material == 1) && f.h.y > 1.0f)) {  // plain box
    float t = range.lo > 0.001f ? range.lo : range.hi;
    return t <= 0.001f ? kFar : t;
  }
  return featureAfterSlabOOL(f, ro, rd, p, d, inv, cone);
}

// Surface normal of a feature at a point (geometry.cu:92-114).
static __device__ __noinline__ f3 featureNormal(Feat f, f3 point) {
  const int shape = f.shape, turn = f.turn;
  const f3 p = intoFeature(point - f.p, turn), h = f.h;
  f3 n = mk(0.0f, 1.0f, 0.0f);
  if (shape == 1 && f.material == 7)
    return leafNormal(int(floorf(point.x / 0.18f)), int(floorf(point.y / 0.18f)), int(floorf(point.z / 0.18f)), int(f.seed));
  if (shape == 1) n = unit(mk(p.x / (h.x * h.x), p.y / (h.y * h.y), p.z / (h.z * h.z)));
  else if (shape == 2) {
    if (fabsf(fabsf(p.y) - h.y) < 0.01f) n = mk(0.0f, p.y < 0.0f ? -1.0f : 1.0f, 0.0f);
    else n = unit(mk(p.x / (h.x * h.x), 0.0f, p.z / (h.z * h.z)));
  } else if (shape == 4 || shape == 7) {
    if (fabsf(fabsf(p.z) - h.z) < 0.008f) n = mk(0.0f, 0.0f, p.z < 0.0f ? -1.0f : 1.0f);
    else {
      float rr = p.x * p.x / (h.x * h.x) + p.y * p.y / (h.y * h.y);
      n = unit(mk(p.x / (h.x * h.x), p.y / (h.y * h.y), 0.0f)) * (rr < 0.8f ? -1.0f : 1.0f);
    }
  } else if (shape == 3) {
    if (fabsf(fabsf(p.z) - h.z) < 0.006f) n = mk(0.0f, 0.0f, p.z < 0.0f ? -1.0f : 1.0f);
    else if (p.y < 0.003f) n = mk(0.0f, -1.0f, 0.0f);
    else n = unit(mk(p.x < 0.0f ? -h.y / h.x : h.y / h.x, 1.0f, 0.0f));
  } else {
    f3 a = mk(fabsf(fabsf(p.x) - h.x), fabsf(fabsf(p.y) - h.y), fabsf(fabsf(p.z) - h.z));
    n = a.x < a.y && a.x < a.z ? mk(p.x < 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f)
        : (a.y < a.z ? mk(0.0f, p.y < 0.0f ? -1.0f : 1.0f, 0.0f) : mk(0.0f, 0.0f, p.z < 0.0f ? -1.0f : 1.0f));
    float bevel = fminf(0.035f, fminf(fminf(h.x, h.y), h.z) * 0.18f);
    f3 q = mk(fmaxf(fabsf(p.x) - h.x + bevel, 0.0f) * (p.x < 0.0f ? -1.0f : 1.0f),
              fmaxf(fabsf(p.y) - h.y + bevel, 0.0f) * (p.y < 0.0f ? -1.0f : 1.0f),
              fmaxf(fabsf(p.z) - h.z + bevel, 0.0f) * (p.z < 0.0f ? -1.0f : 1.0f));
    if (dot(q, q) > 0.000001f) n = unit(q);
  }
  return outOfFeature(n, turn);
}

// One out-of-line copy of the intersection test, so the ~110 emission sites
// of the grammar each compile to a call instead of a full inlined test.
#ifdef STRATUM_INLINE_HIT
SD float featureHitCall(Feat f, f3 ro, f3 rd, float cone) { return featureHit(f, ro, rd, cone); }
#else
static __device__ __noinline__ float featureHitCall(Feat f, f3 ro, f3 rd, float cone) { return featureHit(f, ro, rd, cone); }
#endif

// Nearest-hit sink of one group (kernels/sink.cu:22-25): first wins on ties.
struct HitSink {
  f3 ro, rd;
  float cone, t;
  int fid;
  Feat f;
  SD void take(const Feat& ft, int id) {
    float th = featureHitCall(ft, ro, rd, cone);
    if (th > 0.001f && th < t) { t = th; f = ft; fid = id; }
  }
};

}  // namespace st
