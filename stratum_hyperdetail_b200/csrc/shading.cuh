// Procedural materials and lighting (kernels/materials.cu and kernels/shade.cu
// of the reference): substrate and sky, Worley mineral cells, micro relief,
// per-material albedo, building-mass sun shadows, 3x3-lot ambient visibility,
// GGX specular, reflections, fog, and the resolve's contact occlusion,
// 64-sample running mean and ACES tone map.
#pragma once
#include "stratum_math.cuh"

namespace st {

// One out-of-line copy each of the value noise, the 5-octave fbm, the masonry
// height field and powf for all shading call sites: inlined at every use they
// multiply the kernel's code and it stalls on instruction fetch.  Same
// arithmetic, same bits.
static __device__ __noinline__ float noise2D(float x, float y) { return noise2(x, y); }
static __device__ __noinline__ float fbm2D(float x, float y) { return fbm2(x, y); }
static __device__ __noinline__ float masonryHeightD(float u, float v, int material) { return masonryHeight(u, v, material); }
static __device__ __noinline__ float powD(float x, float y) { return powf(x, y); }

SD f3 substrateMean(int m) { return m == 1 ? mk(0.37f, 0.185f, 0.105f) : mk(0.55f, 0.485f, 0.365f); }
SD f3 substrate(float u, float v, float seed, int m) {
  float large = fbm2D(u * 0.31f + seed * 0.013f, v * 0.31f);
  float run = fbm2D(u * 0.42f + seed * 0.01f, v * 0.038f + 1.7f);
  f3 base = substrateMean(m);
  float age = 0.61f + 0.52f * large, damp = smooth(0.49f, 0.76f, run) * 0.31f;
  return base * (age - damp) + mk(0.017f, 0.024f, 0.014f) * damp;
}
static __device__ __noinline__ f3 skyColor(f3 rd, f3 sun) {
  float elev = sat(rd.y);
  f3 c = mix(mk(0.62f, 0.69f, 0.72f), mk(0.13f, 0.30f, 0.52f), powD(elev, 0.45f));
  float sd = fmaxf(0.0f, dot(rd, sun));
  c = c + mk(1.1f, 0.62f, 0.22f) * powD(sd, 18.0f) + mk(9.0f, 6.0f, 3.2f) * powD(sd, 2600.0f);
  if (rd.y > 0.025f) {
    float cloud = fbm2D(rd.x / (rd.y + 0.20f) * 1.8f + 16.0f, rd.z / (rd.y + 0.20f) * 1.8f);
    float veil = smooth(0.46f, 0.70f, cloud) * smooth(0.02f, 0.2f, rd.y) * 0.55f;
    c = mix(c, mk(0.86f, 0.85f, 0.80f), veil);
  }
  return c;
}
SD f3 mineralCell(float u, float v, int seed) {
  int ix = int(floorf(u)), iy = int(floorf(v));
  float x = fract(u), y = fract(v), nearest = 10.0f, second = 10.0f, value = 0.0f;
#pragma unroll 1
  for (int j = -1; j <= 1; j++)
#pragma unroll
    for (int i = -1; i <= 1; i++) {
      float dx = float(i) + 0.18f + 0.64f * hash2(ix + i, iy + j, seed) - x;
      float dy = float(j) + 0.18f + 0.64f * hash2(ix + i, iy + j, seed + 47) - y;
      float dd = dx * dx + dy * dy;
      if (dd < nearest) { second = nearest; nearest = dd; value = hash2(ix + i, iy + j, seed + 83); }
      else second = fminf(second, dd);
    }
  return mk(sqrtf(nearest), value, sqrtf(second) - sqrtf(nearest));
}
SD float microRelief(float u, float v, float fp) {
  float value = (noise2D(u * 83.0f, v * 83.0f) - 0.5f) * 0.0016f * freqWeight(fp, 83.0f);
  value += (noise2D(u * 277.0f + 8.7f, v * 277.0f) - 0.5f) * 0.00048f * freqWeight(fp, 277.0f);
  value += (noise2D(u * 911.0f, v * 911.0f - 13.9f) - 0.5f) * 0.00013f * freqWeight(fp, 911.0f);
  return value;
}
static __device__ __noinline__ f3 surfaceColor(f3 p, f3 n, int mat, float seed, float fp, f3 foundation) {
  float u, v;
  masonryUV(p, n, u, v);
  float fine = freqWeight(fp, 34.0f);
  f3 c = foundation;
  if (mat == 0 || mat == 1) {  // brick / stone with joints, pores, minerals, cracks, moss
    float bw = mat == 1 ? 0.46f : 0.92f, bh = mat == 1 ? 0.215f : 0.46f;
    int row = int(floorf(v / bh)), brick = int(floorf(u / bw + float(imod(row, 2)) * 0.5f));
    float xx = fract(u / bw + float(imod(row, 2)) * 0.5f), yy = fract(v / bh);
    float edge = fminf(fminf(xx, 1.0f - xx) * bw, fminf(yy, 1.0f - yy) * bh);
    float joint = (1.0f - smooth(0.005f, 0.021f + fp * 0.4f, edge)) * freqWeight(fp, 1.0f / bh);
    float variation = (hash2(brick, row, int(seed)) - 0.5f) * 0.19f * freqWeight(fp, 1.0f / bh);
    c = c * (1.0f + variation);
    c = mix(c, mk(0.25f, 0.245f, 0.21f), joint * 0.84f);
    float pores = fine > 0.0f ? fbm2D(u * 52.0f + seed, v * 52.0f) : 0.5f;
    c = c * (1.0f + (pores - 0.5f) * 0.38f * fine);
    float deposits = smooth(0.45f, 0.76f, fbm2D(u * 5.1f + seed * 0.3f, v * 6.2f));
    c = mix(c, mk(0.52f, 0.49f, 0.39f), deposits * 0.23f * (1.0f - joint));
    if (fp < 0.007f) {
      f3 mineral = mineralCell(u * 190.0f, v * 190.0f, int(seed));
      float detail = freqWeight(fp, 190.0f);
      float pit = (1.0f - smooth(0.075f, 0.23f, mineral.x)) * smooth(0.52f, 0.76f, mineral.y) * detail;
      float grit = (1.0f - smooth(0.018f, 0.072f, mineral.z)) * detail;
      c = c * (1.0f - pit * 0.66f - grit * 0.075f);
      float fleck = (1.0f - smooth(0.04f, 0.17f, mineral.x)) * (1.0f - smooth(0.07f, 0.18f, mineral.y)) * detail;
      c = mix(c, mk(0.62f, 0.56f, 0.44f), fleck * 0.78f);
      float powder = (noise2D(u * 740.0f, v * 740.0f) - 0.5f) * freqWeight(fp, 740.0f);
      c = c * (1.0f + powder * (joint > 0.5f ? 0.50f : 0.24f));
    }
    float crack = fabsf(sinf(u * 8.4f + fbm2D(u * 2.4f, v * 2.4f) * 5.0f + v * 1.3f));
    float fracture = (1.0f - smooth(0.012f, 0.042f + fp * 4.0f, crack)) * smooth(0.48f, 0.72f, noise2D(u * 1.4f, v * 1.4f));
    c = c * (1.0f - fracture * 0.45f * freqWeight(fp, 15.0f));
    float moss = (1.0f - smooth(0.1f, 3.1f, p.y)) * smooth(0.44f, 0.69f, noise2D(u * 1.3f, v * 0.3f));
    c = mix(c, mk(0.095f, 0.125f, 0.046f), moss * 0.7f);
  } else if (mat == 2 || mat == 14) {  // slate / terracotta tiles
    c = mat == 2 ? mk(0.14f, 0.19f, 0.22f) : mk(0.38f, 0.125f, 0.048f);
    float tile = fract(u * 3.7f), row = fract(v * 4.4f);
    float seam = (1.0f - smooth(0.01f, 0.07f, tile)) + (1.0f - smooth(0.02f, 0.11f, row));
    c = c * (0.78f + 0.26f * lerp(0.5f, noise2D(u * 7.2f, v * 7.2f), freqWeight(fp, 7.2f)) -
             sat(seam) * 0.25f * freqWeight(fp, 4.4f));
  } else if (mat == 3) {  // copper patina
    float patina = smooth(0.28f, 0.64f, fbm2D(u * 2.1f, v * 2.1f));
    c = mix(mk(0.27f, 0.145f, 0.072f), mk(0.085f, 0.24f, 0.18f), patina);
    float seam = 1.0f - smooth(0.015f, 0.07f, fract(u * 1.8f));
    c = c * (1.0f - seam * 0.4f * freqWeight(fp, 1.8f));
  } else if (mat == 4) c = mk(0.045f, 0.084f, 0.093f);
  else if (mat == 5) {
    float grain = sinf(u * 49.0f + fbm2D(u * 2.0f, v * 0.5f) * 8.0f);
    c = mk(0.12f, 0.07f, 0.039f) * (1.0f + grain * 0.12f * fine);
  } else if (mat == 6) c = mk(0.075f, 0.091f, 0.087f) * (0.8f + noise2D(u * 30.0f, v * 30.0f) * 0.3f);
  else if (mat == 7) {
    float leaves = fbm2D(p.x * 8.0f + p.y * 6.0f, p.z * 8.0f);
    c = mix(mk(0.055f, 0.095f, 0.020f), mk(0.18f, 0.25f, 0.055f), leaves);
  } else if (mat == 8) c = mk(0.70f, 0.43f, 0.13f);
  else if (mat == 9) c = mk(0.035f, 0.115f, 0.12f);
  else if (mat == 10) {
    float grit = lerp(0.5f, fbm2D(u * 45.0f, v * 45.0f), freqWeight(fp, 45.0f));
    c = mk(0.16f, 0.17f, 0.16f) * (0.72f + grit * 0.4f);
  } else if (mat == 11) {
    int row = int(floorf(v / 0.45f));
    float a = fract(u / 0.9f + float(imod(row, 2)) * 0.5f), b = fract(v / 0.45f);
    float joint = (1.0f - smooth(0.02f, 0.07f + fp, fminf(fminf(a, 1.0f - a), fminf(b, 1.0f - b))));
    c = mk(0.43f, 0.415f, 0.36f) * (0.78f + fbm2D(u * 18.0f, v * 18.0f) * 0.3f);
    c = c * (1.0f - joint * 0.30f * freqWeight(fp, 2.0f));
  } else if (mat == 13) c = mk(0.54f, 0.475f, 0.35f) * (0.82f + fbm2D(u * 1.6f, v * 1.6f) * 0.24f);
  else if (mat == 15) c = mk(0.17f, 0.12f, 0.065f) * (0.65f + 0.6f * fbm2D(u * 31.0f, v * 3.0f));
  if (mat == 18) {
    float panel = fract(u / 1.6f);
    float frame = (1.0f - smooth(0.02f, 0.06f, panel)) + (1.0f - smooth(0.02f, 0.06f, 1.0f - panel));
    float band = 1.0f - smooth(0.03f, 0.07f, fabsf(v - 2.65f));
    c = mix(mk(0.058f, 0.092f, 0.105f), mk(0.10f, 0.059f, 0.027f), sat(frame + band));
  }
  if (mat == 17) {
    float a = atan2f(v - floorf(v / 30.0f) * 30.0f - 28.5f, u);
    float glass = 0.5f + 0.5f * sinf(a * 12.0f + seed);
    c = mix(mk(0.08f, 0.18f, 0.32f), mk(0.50f, 0.12f, 0.04f), glass);
  }
  return c;
}

// Sun visibility against building masses along a lot DDA of <= 64 cells;
// cells outside the resident table are described on the fly (shade.cu:3-22).
static __device__ __noinline__ float buildingShadow(const float* __restrict__ W, uint32_t o0, uint32_t o1, uint32_t o2,
                                             uint32_t o3, f3 p, f3 light, int worldSeed) {
  if (light.y < 0.005f) return 0.05f;
  float limit = fminf(1500.0f, fmaxf(0.0f, (kTop - p.y) / light.y));
  f3 ro = p + light * 0.08f;
  int cx = int(floorf((ro.x + 18.0f) / kCell)), cz = int(floorf((ro.z + 18.0f) / kCell));
  int sx = light.x > 0.0f ? 1 : -1, sz = light.z > 0.0f ? 1 : -1;
  float ix = guardedInv(light.x), iz = guardedInv(light.z);
  float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * ix;
  float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * iz;
  float dx = kCell * fabsf(ix), dz = kCell * fabsf(iz), t = 0.0f;
#pragma unroll 1
  for (int step = 0; step < 64; step++) {
    if (t > limit) break;
    LotDesc l = (cx >= -64 && cx < 64 && cz >= -64 && cz < 64) ? loadLot(W, tableSlot(o0, o2, cx, cz))
                                                              : describe(shiftAddr(o0, o1, o2, o3, cx, cz), worldSeed);
    if (l.type < 3) {
      f3 cp = mk(float(cx) * kCell + l.ox, 0.0f, float(cz) * kCell + l.oz);
      f3 lr = toLot(ro - cp, l.turn), ld = toLot(light, l.turn);
      Span s = slab(lr, ld, mk(-l.w + 0.05f, 4.1f, -l.d + 0.05f), mk(l.w - 0.05f, l.h, l.d - 0.05f));
      if (s.hi > fmaxf(0.06f, s.lo) && s.lo < limit) return 0.06f;
    }
    if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
  }
  return 1.0f;
}
SD float ambientVisibility(const float* __restrict__ W, uint32_t o0, uint32_t o2, f3 p) {
  int cx = int(floorf((p.x + 18.0f) / kCell)), cz = int(floorf((p.z + 18.0f) / kCell));
  float occ = 0.0f;
#pragma unroll 1
  for (int z = -1; z <= 1; z++)
#pragma unroll 1
    for (int x = -1; x <= 1; x++) {
      LotDesc l = loadLot(W, tableSlot(o0, o2, cx + x, cz + z));
      if (l.type >= 3) continue;
      f3 q = toLot(p - mk(float(cx + x) * kCell + l.ox, 0.0f, float(cz + z) * kCell + l.oz), l.turn);
      float xx = fmaxf(0.0f, fabsf(q.x) - l.w), zz = fmaxf(0.0f, fabsf(q.z) - l.d);
      float dist = sqrtf(xx * xx + zz * zz);
      if (dist > 0.06f) occ += sat((l.h - p.y) / (dist + l.h + 1.0f)) * expf(-dist * 0.12f) * 0.48f;
    }
  return clampv(1.0f - occ, 0.35f, 1.0f);
}
SD f3 paletteTint(float palette, int mat) {
  if (mat != 0 && mat != 1 && mat != 13) return mk(1.0f, 1.0f, 1.0f);
  switch (int(palette)) {
    case 0: return mk(1.04f, 0.95f, 0.85f);
    case 1: return mk(0.80f, 0.89f, 1.02f);
    case 2: return mk(1.12f, 0.89f, 0.83f);
    case 3: return mk(1.13f, 1.12f, 1.04f);
    case 4: return mk(0.83f, 0.84f, 0.79f);
    case 5: return mk(0.91f, 1.02f, 0.91f);
    case 6: return mk(1.03f, 0.95f, 1.02f);
    default: return mk(1.0f, 1.0f, 1.0f);
  }
}

struct FrameConst {
  Camera cam;
  f3 sun;
  uint32_t o[4];
  float exposure, view, shadowsOff, sample;
  int seed;
};
SD FrameConst makeFrame(const float* C, const uint32_t* O) {
  FrameConst f;
  f.cam = makeCamera(C);
  f.sun = sunDir(C);
  for (int i = 0; i < 4; i++) f.o[i] = O ? O[i] : 0u;
  f.exposure = C[9]; f.view = C[11]; f.shadowsOff = C[18]; f.sample = C[19];
  f.seed = int(C[14]);
  return f;
}

// Shading of one pixel (shade.cu:45-102) in three parts, so the batched path
// can run the material and the lighting as two kernels (each a smaller body of
// code for the instruction cache): the surface point, its albedo, its light.
// shadePixel composes them; every path computes the same values in the same
// order.

// A hit pixel's surface as shading sees it (shade.cu:45-70): the hit point in
// the world and lot frames, the normal (flipped for foliage seen from inside),
// material and seed (ground: paving, asphalt or water from the lot), the
// footprint and the masonry coordinates.
struct SurfacePoint {
  f3 p, n, q, qn;
  LotDesc lot;
  int mat;
  float seed, palette, t, sfp, u, v;
};
SD void surfacePoint(const float* __restrict__ W, const FrameConst& F, float4 hit, float4 surf, f3 rd, int height,
                     SurfacePoint& s) {
  s.t = hit.x;
  s.p = F.cam.pos + rd * s.t;
  s.n = mk(surf.x, surf.y, surf.z);
  s.mat = int(hit.z);
  int slot = int(surf.w);
  if (slot >= kLots) slot = -1;  // never index past the table on a malformed Surface
  s.seed = hit.w;
  s.q = s.p; s.qn = s.n;
  s.palette = 0.0f;
  if (slot >= 0) {
    s.lot = loadLot(W, slot);
    int cx, cz;
    slotCell(F.o[0], F.o[2], slot, cx, cz);
    f3 cp = mk(float(cx) * kCell, 0.0f, float(cz) * kCell) + mk(s.lot.ox, 0.0f, s.lot.oz);
    s.q = toLot(s.p - cp, s.lot.turn);
    s.qn = toLot(s.n, s.lot.turn);
    s.palette = s.lot.palette;
  } else {  // ground: paving inside the lot, asphalt outside, water on canals
    int cx = int(floorf((s.p.x + 18.0f) / kCell)), cz = int(floorf((s.p.z + 18.0f) / kCell));
    slot = tableSlot(F.o[0], F.o[2], cx, cz);
    s.lot = loadLot(W, slot);
    s.q = s.p - mk(float(cx) * kCell, 0.0f, float(cz) * kCell);
    s.seed = s.lot.seed;
    s.mat = fabsf(s.q.x) < 16.5f && fabsf(s.q.z) < 16.5f ? 11 : 10;
    if (s.lot.type == 5) s.mat = 9;
  }
  if (s.mat == 7 && dot(s.n, rd) > 0.0f) { s.n = s.n * -1.0f; s.qn = s.qn * -1.0f; }
  float footprint = fmaxf(0.00005f, s.t * 1.08f / float(height));
  s.sfp = footprint / fmaxf(0.18f, fabsf(dot(s.n, rd)));
  masonryUV(s.q, s.qn, s.u, s.v);
}
// Material colour with the palette tint (materials.cu, shade.cu:71).
SD f3 pixelAlbedo(const SurfacePoint& s) {
  f3 base = substrateMean(s.mat);
  if (s.mat == 0 || s.mat == 1) base = substrate(s.u, s.v, s.seed, s.mat);
  return surfaceColor(s.q, s.qn, s.mat, s.seed, s.sfp, base) * paletteTint(s.palette, s.mat);
}
// Lighting of a hit pixel of this albedo (shade.cu:72-102): mortar relief
// normal, sun shadow, ambient visibility, GGX, reflections, fog, debug views.
SD f3 pixelLight(const float* __restrict__ W, const FrameConst& F, const SurfacePoint& s, f3 rd, int id, f3 albedo) {
  const f3 sun = F.sun;
  const f3 p = s.p, q = s.q, qn = s.qn;
  const int mat = s.mat;
  const float t = s.t, sfp = s.sfp, u = s.u, v = s.v, seed = s.seed;
  f3 n = s.n, result;
  f3 originalN = n;
  if ((mat == 0 || mat == 1) && fabsf(qn.y) < 0.5f) {  // mortar relief normal by central differences
    float eps = fmaxf(0.002f, sfp * 0.6f);
    float du = (masonryHeightD(u + eps, v, mat) - masonryHeightD(u - eps, v, mat)) / (2.0f * eps);
    float dv = (masonryHeightD(u, v + eps, mat) - masonryHeightD(u, v - eps, mat)) / (2.0f * eps);
    if (sfp < 0.005f) {
      float me = fmaxf(0.00016f, sfp * 0.8f);
      du += (microRelief(u + me, v, sfp) - microRelief(u - me, v, sfp)) / (2.0f * me);
      dv += (microRelief(u, v + me, sfp) - microRelief(u, v - me, sfp)) / (2.0f * me);
    }
    f3 tangent = fabsf(qn.x) > 0.5f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    float fade = freqWeight(sfp, 5.0f);
    f3 localN = unit(qn - tangent * (du * fade) - mk(0.0f, dv * fade, 0.0f));
    n = fromLot(localN, s.lot.turn);
  }
  if (mat == 9) n = unit(n + mk(cosf(q.x * 3.7f + q.z * 1.1f) * 0.06f, 0.0f, sinf(q.z * 4.4f - q.x * 0.9f) * 0.08f));
  float nl = fmaxf(0.0f, dot(n, sun)), nv = fmaxf(0.03f, -dot(n, rd));
  float shadow = F.shadowsOff > 0.5f ? 1.0f
                                     : buildingShadow(W, F.o[0], F.o[1], F.o[2], F.o[3], p + originalN * 0.035f, sun, F.seed);
  float ao = ambientVisibility(W, F.o[0], F.o[2], p), rough = 0.75f;
  if (mat == 3 || mat == 6) rough = 0.38f;
  if (mat == 4) rough = 0.18f;
  if (mat == 9) rough = 0.12f;
  if (mat == 8) rough = 0.3f;
  f3 halfv = unit(sun - rd);
  float nh = fmaxf(0.0f, dot(n, halfv)), vh = fmaxf(0.0f, -dot(rd, halfv));
  float a = rough * rough, denom = nh * nh * (a * a - 1.0f) + 1.0f;
  float distribution = a * a / (kPi * denom * denom + 0.000001f);
  float k = (rough + 1.0f) * (rough + 1.0f) / 8.0f;
  float geometry = nv / (nv * (1.0f - k) + k) * nl / (nl * (1.0f - k) + k + 0.00001f);
  float f0 = mat == 3 || mat == 6 || mat == 8 ? 0.35f : 0.045f;
  float fresnel = f0 + (1.0f - f0) * powD(1.0f - vh, 5.0f);
  float spec = distribution * geometry * fresnel / (4.0f * nv * nl + 0.0001f);
  f3 direct = mk(2.25f, 1.72f, 1.18f) * (nl * shadow);
  float skyWeight = 0.22f + 0.29f * sat(n.y * 0.5f + 0.5f);
  f3 ambient = mk(0.25f, 0.34f, 0.44f) * (skyWeight * ao);
  ambient = ambient + mk(0.65f, 0.43f, 0.25f) * ((1.0f - sat(n.y)) * 0.10f * ao);
  result = albedo * (direct + ambient) + mk(1.0f, 0.87f, 0.63f) * (spec * nl * shadow * 2.1f);
  if (mat == 4 || mat == 9) {
    f3 reflection = rd - n * (2.0f * dot(rd, n));
    float fr = 0.10f + 0.72f * powD(1.0f - nv, 4.0f);
    result = mix(result, skyColor(reflection, sun) * 0.60f, fr);
    if (mat == 4) {
      float room = hash1(int(seed));
      result = result * 0.73f + mk(0.13f, 0.075f, 0.028f) * (room > 0.78f ? 0.3f : 0.03f);
    }
  }
  if (mat == 8) result = result + mk(1.1f, 0.62f, 0.19f) * 0.8f;
  if (mat == 7) result = result + albedo * (powD(fmaxf(0.0f, dot(rd, sun)), 4.0f) * 0.35f);
  float fog = 1.0f - expf(-t * 0.00068f);
  fog = lerp(fog, 1.0f, smooth(kFar * 0.68f, kFar, t));
  f3 haze = skyColor(unit(mk(rd.x, 0.004f, rd.z)), sun);
  result = mix(result, haze, fog);
  if (F.view == 1.0f) result = paletteTint(s.lot.palette, 0) * mk(0.4f, 0.55f, 0.6f);
  if (F.view == 2.0f) {
    int g = id >= 0 ? id / kMaxFeatures : 0;
    result = mk(0.15f + 0.75f * hash1(g), 0.15f + 0.75f * hash1(g + 31), 0.15f + 0.75f * hash1(g + 98));
  }
  if (F.view == 3.0f) result = (n + mk(1.0f, 1.0f, 1.0f)) * 0.5f;
  return result;
}


// Linear colour of one pixel (shade.cu:45-102).
SD f3 shadePixel(const float* __restrict__ W, const FrameConst& F, float4 hit, float4 surf, f3 rd, int height) {
  const int id = int(hit.y);
  if (id == kSkyId) return skyColor(rd, F.sun);  // (a hit pixel's colour never reads the sky term)
  SurfacePoint s;
  surfacePoint(W, F, hit, surf, rd, height, s);
  return pixelLight(W, F, s, rd, id, pixelAlbedo(s));
}

SD float aces(float x) { return sat(x * (2.51f * x + 0.03f) / (x * (2.43f * x + 0.59f) + 0.14f)); }

// Contact occlusion, running mean and tone map of one pixel (shade.cu:104-123).
// Eight taps at angles k*pi/4 + 0.2: their cos/sin are per-launch constants.
struct ResolveTaps { float c[8], s[8]; };
SD ResolveTaps makeTaps() {
  ResolveTaps r;
  for (int k = 0; k < 8; k++) {
    float a = float(k) * kPi * 0.25f + 0.2f;
    r.c[k] = cosR(a); r.s[k] = sinR(a);
  }
  return r;
}
// `c` is the pixel's linear colour (Linear[b].rgb).
SD void resolvePixel(f3 c, float4* Hist, uint32_t* Px, const FrameConst& F, const ResolveTaps& taps,
                     const float4* __restrict__ Hit, const float4* __restrict__ Surf, int width, int height, int x,
                     int y) {
  const size_t b = size_t(y) * width + x;
  float4 h4 = Hit[b];
  if (F.view < 0.5f && int(h4.y) != kSkyId && h4.x < 250.0f) {
    f3 ro = F.cam.pos, point = ro + primaryDir(F.cam, x, y, width, height) * h4.x;
    float4 s4 = Surf[b];
    f3 n = mk(s4.x, s4.y, s4.z);
    float occ = 0.0f;
    float radius = clampv(float(height) / (fmaxf(h4.x, 0.5f) * 1.08f) * 0.8f, 3.0f, 28.0f);
#pragma unroll 1
    for (int k = 0; k < 8; k++) {
      int xx = int(clampv(float(x) + taps.c[k] * radius, 0.0f, float(width - 1)));
      int yy = int(clampv(float(y) + taps.s[k] * radius, 0.0f, float(height - 1)));
      float4 o4 = Hit[size_t(yy) * width + xx];
      if (int(o4.y) != kSkyId) {
        f3 other = ro + primaryDir(F.cam, xx, yy, width, height) * o4.x, delta = other - point;
        float l = len(delta);
        if (l > 0.04f && l < 2.0f) occ += fmaxf(0.0f, dot(n, delta / l) - 0.12f) * expf(-l * 1.4f) * 0.28f;
      }
    }
    c = c * clampv(1.0f - occ, 0.55f, 1.0f);
  }
  float4 old4 = Hist[b];
  float oldCount = old4.w, count = F.sample <= 1.0f ? 1.0f : fminf(64.0f, oldCount + 1.0f);
  f3 old = mk(old4.x, old4.y, old4.z);
  if (F.sample >= 64.0f && oldCount >= 64.0f) c = old;
  else c = mix(old, c, 1.0f / count);
  Hist[b] = make_float4(c.x, c.y, c.z, count);
  float sx = (float(x) / float(width) - 0.5f) * 1.3f, sy = (float(y) / float(height) - 0.5f) * 1.3f;
  c = c * (F.exposure * (1.0f - (sx * sx + sy * sy) * 0.12f));
  c = mk(powD(aces(c.x), 1.0f / 2.2f), powD(aces(c.y), 1.0f / 2.2f), powD(aces(c.z), 1.0f / 2.2f));
  Px[b] = packRGBA8(c);
}

}  // namespace st
