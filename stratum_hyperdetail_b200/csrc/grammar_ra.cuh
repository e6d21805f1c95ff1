// Random access into the feature grammar: feature #i of (lot, group) computed
// directly, without emitting features 0..i-1.
//
// The grammar (kernels/assets.cu:3-265 of the reference, grammar.cuh here) is a
// fixed sequence of sections per group -- single features and loop nests whose
// trip counts depend only on the lot type and floor count.  groupCount() gives
// the length of that sequence and featureAt() decodes an index into its section
// and loop counters and evaluates that one feature with the same floating-point
// expressions, so featureAt(L, g, i) equals the i-th emission of runGroup bit
// for bit (tested against the CPU oracle on every lot family, floor count and
// group).  This lets 32 lanes of a warp produce one group's features in
// parallel, one feature per lane.
#pragma once
#include "grammar.cuh"

namespace st {

// kernels/sink.cu:10-13 roof rescale, then the record.
HD Feat makeFeat(const LotDesc& L, f3 p, f3 h, int shape, int mat, int turn, float seed) {
  if (p.y >= L.h) { p.y = L.h + (p.y - L.h) * L.roofScale; h.y *= L.roofScale; }
  return Feat{p, h, shape, mat, turn, seed};
}
// kernels/sink.cu:27-33 facade box.
HD Feat makeWall(const LotDesc& L, int face, float cx, float cz, float w, float d, float u, float y, float o, float hw,
                 float hy, float hd, int mat, float seed) {
  f3 p = mk(cx + u, y, cz + d + o), h = mk(hw, hy, hd);
  if (face == 1) { p = mk(cx + w + o, y, cz + u); h = mk(hd, hy, hw); }
  if (face == 2) p = mk(cx + u, y, cz - d - o);
  if (face == 3) { p = mk(cx - w - o, y, cz + u); h = mk(hd, hy, hw); }
  return makeFeat(L, p, h, 0, mat, 0, seed);
}

HD int groupCount(const LotDesc& L, int g) {
  const int type = L.type, floors = L.floors;
  if (g < 0 || g >= kGroups || type == 5) return 0;
  if (type == 4) return g == 0 ? 27 : 0;
  if (type == 3) return g == 0 ? 1 : (g <= 8 ? 29 : (g == 9 ? 5 : 0));
  if (g == 0) return 28;
  if (g == 1) return type == 0 ? 15 : (type == 1 ? 5 : 18);
  if (g <= 5) return 2 * (floors + 1 > 0 ? floors + 1 : 0) + 5 + 8 + 4 + 4;
  if (g < 30) return (g - 6) % 6 < floors ? 48 : 0;
  if (g == 30) return 56;
  if (g == 31) return (type == 0 ? 12 : 0) + 38;
  if (g < 56) return (g - 32) % 6 < floors ? 48 : 0;
  if (g < 60) return 28 + (type == 2 ? 2 : 0);
  if (g < 62) return type == 0 ? 32 : 0;
  return 32;
}

// Feature #i (0 <= i < groupCount) of group g.
HD Feat featureAt(const LotDesc& L, int group, int i) {
  const float x = 0.0f, z = 0.0f, w = L.w, d = L.d, h = L.h, seed = L.seed, storey = L.storey;
  const int type = L.type, mat = L.mat, floors = L.floors;
  if (type == 4) {  // canal bridge: deck, two parapets, 12 x 2 posts
    if (i == 0) return makeFeat(L, mk(x, 0.25f, z), mk(18.0f, 0.5f, 5.0f), 0, 0, 0, seed);
    if (i == 1) return makeFeat(L, mk(x, 1.25f, z - 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
    if (i == 2) return makeFeat(L, mk(x, 1.25f, z + 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
    int m = i - 3, k = m >> 1;
    float u = -16.5f + float(k) * 3.0f;
    return makeFeat(L, mk(x + u, 0.8f, (m & 1) ? z + 5.0f : z - 5.0f), mk(0.12f, 0.6f, 0.12f), 2, 6, 0, seed);
  }
  if (type == 3) {  // park: paving; trees (trunk + 28 foliage envelopes); fountain
    if (group == 0) return makeFeat(L, mk(x, -0.12f, z), mk(15.5f, 0.22f, 15.5f), 0, 11, 0, seed);
    if (group <= 8) {
      int k = group - 1;
      float tx = x + (k < 4 ? -10.0f : 10.0f), tz = z + (float(k % 4) - 1.5f) * 6.7f;
      float th = 5.0f + hash1(int(seed) + k) * 3.0f;
      if (i == 0) return makeFeat(L, mk(tx, th * 0.4f, tz), mk(0.19f, th * 0.4f, 0.19f), 2, 15, 0, seed);
      int j = i - 1;
      float yy = hash1(int(seed) + j + 991) * 3.3f - 0.5f;
      float rr = sqrtf(hash1(int(seed) + j + 330)) * 2.1f * (1.0f - yy * 0.12f);
      float size = 0.48f + hash1(int(seed) + j + 62) * 0.30f;
      return makeFeat(L, mk(tx + TreeCos(j) * rr, th + yy, tz + TreeSin(j) * rr), mk(size, size * 1.25f, size), 1, 7, 0,
                      seed + float(j));
    }
    switch (i) {
      case 0: return makeFeat(L, mk(x, 0.8f, z), mk(3.6f, 0.45f, 3.6f), 2, 0, 0, seed);
      case 1: return makeFeat(L, mk(x, 1.24f, z), mk(3.3f, 0.04f, 3.3f), 2, 9, 0, seed);
      case 2: return makeFeat(L, mk(x, 2.0f, z), mk(0.65f, 1.0f, 0.65f), 2, 0, 0, seed);
      case 3: return makeFeat(L, mk(x, 2.85f, z), mk(1.4f, 0.18f, 1.4f), 2, 13, 0, seed);
      default: return makeFeat(L, mk(x, 3.15f, z), mk(0.5f, 0.5f, 0.5f), 1, 3, 0, seed);
    }
  }
  // buildings
  if (group == 0) {  // plinth, mass, cornice, arcade void; 12 x (column, capital)
    if (i == 0) return makeFeat(L, mk(x, 0.15f, z), mk(w + 1.1f, 0.25f, d + 1.1f), 0, 0, 0, seed);
    if (i == 1) return makeFeat(L, mk(x, (h + 4.0f) * 0.5f, z), mk(w, (h - 4.0f) * 0.5f, d), 0, mat, 0, seed);
    if (i == 2) return makeFeat(L, mk(x, 4.0f, z), mk(w + 0.24f, 0.24f, d + 0.24f), 0, 13, 0, seed);
    if (i == 3) return makeFeat(L, mk(x, 1.9f, z), mk(w - 3.5f, 1.9f, d - 3.5f), 0, 5, 0, seed);
    int m = i - 4, c = m >> 1, f = c / 3, k = c % 3;
    float ext = (f % 2 == 0 ? w : d) - 0.65f, u = (float(k) - 1.0f) * ext;
    float px = f % 2 == 0 ? x + u : x + (f == 1 ? w - 0.5f : -w + 0.5f);
    float pz = f % 2 == 0 ? z + (f == 0 ? d - 0.5f : -d + 0.5f) : z + u;
    if ((m & 1) == 0) return makeFeat(L, mk(px, 2.0f, pz), mk(0.38f, 1.75f, 0.38f), 2, 0, 0, seed + float(k));
    return makeFeat(L, mk(px, 3.66f, pz), mk(0.64f, 0.18f, 0.64f), 0, 13, 0, seed);
  }
  if (group == 1) {  // roof
    if (i == 0) return makeFeat(L, mk(x, h + 0.25f, z), mk(w + 0.6f, 0.24f, d + 0.6f), 0, 13, 0, seed);
    if (type == 0) {
      int roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
      if (i == 1) return makeFeat(L, mk(x, h + 0.35f, z), mk(w + 0.45f, 4.4f, d + 0.45f), 3, roofmat, 0, seed);
      if (i == 2) return makeFeat(L, mk(x, h + 4.8f, z), mk(0.12f, 0.14f, d + 0.7f), 0, 3, 0, seed);
      int m = i - 3, k = m / 3, r = m % 3;
      float xx = x + (k % 2 == 0 ? -w * 0.52f : w * 0.52f), zz = z + (float(k / 2) - 0.5f) * d;
      if (r == 0) return makeFeat(L, mk(xx, h + storey, zz), mk(0.48f, 2.2f, 0.55f), 0, 1, 0, seed);
      if (r == 1) return makeFeat(L, mk(xx, h + 6.0f, zz), mk(0.66f, 0.17f, 0.72f), 0, 0, 0, seed);
      return makeFeat(L, mk(xx, h + 6.32f, zz), mk(0.2f, 0.25f, 0.2f), 2, 14, 0, seed);
    }
    if (type == 1) {
      switch (i) {
        case 1: return makeFeat(L, mk(x, h + 2.2f, z), mk(w * 0.72f, 2.0f, w * 0.72f), 2, 0, 0, seed);
        case 2: return makeFeat(L, mk(x, h + 3.1f, z), mk(w * 0.79f, 8.4f, w * 0.79f), 1, 3, 0, seed);
        case 3: return makeFeat(L, mk(x, h + 12.2f, z), mk(0.24f, 1.45f, 0.24f), 2, 6, 0, seed);
        default: return makeFeat(L, mk(x, h + 13.8f, z), mk(0.6f, 0.6f, 0.6f), 1, 8, 0, seed);
      }
    }
    if (i == 1) return makeFeat(L, mk(x, h + 0.4f, z), mk(w * 0.72f, 5.2f, d + 0.2f), 3, 2, 0, seed);
    int m = i - 2, k = m >> 3, r = m & 7;
    float xx = x + (k == 0 ? -w * 0.75f : w * 0.75f), zz = z + d * 0.60f;
    switch (r) {
      case 0: return makeFeat(L, mk(xx, h + 3.5f, zz), mk(2.3f, 7.2f, 2.3f), 0, 0, 0, seed);
      case 1: return makeFeat(L, mk(xx, h + 10.9f, zz), mk(2.65f, 0.35f, 2.65f), 0, 13, 0, seed);
      case 2: return makeFeat(L, mk(xx, h + 11.2f, zz), mk(2.55f, 4.4f, 2.55f), 3, 3, 0, seed);
      case 3: return makeFeat(L, mk(xx, h + 16.0f, zz), mk(0.17f, 1.2f, 0.17f), 2, 8, 0, seed);
      default: {
        int j = r - 4;
        return makeFeat(L, mk(xx + QuarterCos(j) * 2.2f, h + 12.0f, zz + QuarterSin(j) * 2.2f), mk(0.17f, 1.1f, 0.17f), 2,
                        0, 0, seed);
      }
    }
  }
  if (group <= 5) {  // string courses, pilasters, dentils, hyperdetail courses and reveals
    int face = group - 2;
    float ext = face % 2 == 0 ? w : d;
    int n1 = 2 * (floors + 1 > 0 ? floors + 1 : 0);
    if (i < n1) {
      int j = i >> 1;
      float y = 4.2f + float(j) * storey;
      if ((i & 1) == 0) return makeWall(L, face, x, z, w, d, 0.0f, y, 0.17f, ext + 0.15f, 0.11f, 0.22f, 13, seed);
      return makeWall(L, face, x, z, w, d, 0.0f, y + 0.21f, 0.1f, ext + 0.10f, 0.052f, 0.16f, 0, seed);
    }
    int m = i - n1;
    if (m < 5) {
      float u = (float(m) / 4.0f * 2.0f - 1.0f) * (ext - 0.3f);
      return makeWall(L, face, x, z, w, d, u, (h + 4.0f) * 0.5f, 0.16f, 0.19f, (h - 4.0f) * 0.5f, 0.22f, 13, seed);
    }
    m -= 5;
    if (m < 8) {
      float u = (float(m) - 3.5f) * (ext / 4.0f);
      return makeWall(L, face, x, z, w, d, u, h - 0.24f, 0.4f, 0.15f, 0.12f, 0.19f, 13, seed);
    }
    m -= 8;
    if (m < 4) {
      float yy = 5.05f + float(m) * fmaxf(1.0f, (h - 6.0f) / 4.0f);
      return makeWall(L, face, x, z, w, d, 0.0f, yy, 0.205f, ext + 0.08f, 0.035f, 0.055f, 13, seed + 410.0f + float(m));
    }
    m -= 4;
    float u = (float(m) - 1.5f) * (ext * 0.48f);
    return makeWall(L, face, x, z, w, d, u, h - 0.72f, 0.255f, 0.055f, 0.34f, 0.07f, 0, seed + 450.0f + float(m));
  }
  if (group < 30) {  // windows of one storey: 4 x 8 parts, then frames and sills
    int face = (group - 6) / 6, row = (group - 6) % 6;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
    if (i < 32) {
      int j = i >> 3, r = i & 7;
      float u = (float(j) - 1.5f) * (ext * 0.48f), wy = 1.2f;
      switch (r) {
        case 0: return makeWall(L, face, x, z, w, d, u, y, 0.032f, 0.91f, wy, 0.045f, 4, seed + float(row * 17 + j * 9 + face * 59));
        case 1: return makeWall(L, face, x, z, w, d, u, y - wy - 0.13f, 0.22f, 1.13f, 0.14f, 0.29f, 13, seed);
        case 2: return makeWall(L, face, x, z, w, d, u, y + wy + 0.12f, 0.18f, 1.11f, 0.14f, 0.23f, 13, seed);
        case 3: return makeWall(L, face, x, z, w, d, u - 1.02f, y, 0.12f, 0.11f, wy, 0.17f, 13, seed);
        case 4: return makeWall(L, face, x, z, w, d, u + 1.02f, y, 0.12f, 0.11f, wy, 0.17f, 13, seed);
        case 5: return makeWall(L, face, x, z, w, d, u, y, 0.12f, 0.044f, wy, 0.08f, 5, seed);
        case 6: return makeWall(L, face, x, z, w, d, u, y + 0.3f, 0.12f, 0.94f, 0.035f, 0.08f, 5, seed);
        default: return makeWall(L, face, x, z, w, d, u, y - wy + 0.46f, 0.56f, 1.10f, 0.035f, 0.035f, 6, seed);
      }
    }
    int m = i - 32;
    if (m < 8) {
      int j = m >> 1;
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      if ((m & 1) == 0) return makeWall(L, face, x, z, w, d, u - 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 500.0f + float(j));
      return makeWall(L, face, x, z, w, d, u + 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 520.0f + float(j));
    }
    m -= 8;
    int j = m >> 1;
    float u = (float(j) - 1.5f) * (ext * 0.48f);
    if ((m & 1) == 0) return makeWall(L, face, x, z, w, d, u, y - 1.31f, 0.30f, 1.18f, 0.045f, 0.07f, 13, seed + 540.0f + float(j));
    return makeWall(L, face, x, z, w, d, u, y + 1.31f, 0.18f, 1.08f, 0.038f, 0.055f, 13, seed + 560.0f + float(j));
  }
  if (group == 30) {  // street furniture, clutter and benches
    if (i < 8) {
      int k = i >> 2, r = i & 3;
      float px = x + (k == 0 ? -16.0f : 16.0f), pz = z + 15.9f;
      switch (r) {
        case 0: return makeFeat(L, mk(px, 2.0f, pz), mk(0.068f, 2.0f, 0.068f), 2, 6, 0, seed);
        case 1: return makeFeat(L, mk(px, 4.0f, pz), mk(0.29f, 0.38f, 0.29f), 0, 8, 0, seed);
        case 2: return makeFeat(L, mk(px, 4.44f, pz), mk(0.37f, 0.1f, 0.37f), 3, 6, 0, seed);
        default: return makeFeat(L, mk(px, 0.15f, pz), mk(0.27f, 0.18f, 0.27f), 2, 0, 0, seed);
      }
    }
    int m = i - 8;
    if (m < 8) return makeFeat(L, mk(x - 14.9f, 0.43f, z - 12.0f + float(m) * 3.3f), mk(0.10f, 0.43f, 0.10f), 2, 6, 0, seed);
    m -= 8;
    if (m < 8) {
      int face = m >> 1, k = m & 1;
      float ext = (face % 2 == 0 ? w : d) - 0.65f, u = (k == 0 ? -0.5f : 0.5f) * ext;
      f3 c = mk(x + u, 3.16f, z + (face == 0 ? d - 0.5f : -d + 0.5f));
      if (face % 2 == 1) c = mk(x + (face == 1 ? w - 0.5f : -w + 0.5f), 3.16f, z + u);
      return makeFeat(L, c, mk(ext * 0.5f, 0.88f, 0.49f), 4, 13, face % 2, seed);
    }
    m -= 8;
    if (m < 4) {
      float side = m < 2 ? -1.0f : 1.0f, along = (m % 2 == 0 ? -0.58f : 0.58f);
      return makeFeat(L, mk(x + side * (w + 0.34f), h * 0.38f, z + along * d), mk(0.075f, h * 0.38f, 0.075f), 2, 6, 0,
                      seed + 700.0f + float(m));
    }
    m -= 4;
    if (m < 4)
      return makeFeat(L, mk(x - 12.0f + float(m) * 8.0f, 0.48f, z + d + 2.0f), mk(0.12f, 0.48f, 0.12f), 2, 6, 0,
                      seed + 720.0f + float(m));
    m -= 4;
    if (m < 8)
      return makeFeat(L, mk(x - 14.0f + float(m) * 4.0f, 0.055f, z - d - 2.2f), mk(1.75f, 0.035f, 0.045f), 0, 13, 0,
                      seed + 740.0f + float(m));
    m -= 8;
    int bench = m >> 3, r = m & 7;
    float bx = bench == 0 ? -7.0f : 7.0f, bz = d + 1.8f;
    if (r < 4)
      return makeFeat(L, mk(bx, 0.59f, bz + (float(r) - 1.5f) * 0.13f), mk(1.3f, 0.045f, 0.053f), 0, 5, 0,
                      seed + 900.0f + float(r));
    if (r < 6) return makeFeat(L, mk(bx + (r == 4 ? -0.95f : 0.95f), 0.3f, bz), mk(0.065f, 0.3f, 0.27f), 0, 6, 0, seed);
    return makeFeat(L, mk(bx, 0.88f + float(r - 6) * 0.19f, bz + 0.23f), mk(1.3f, 0.075f, 0.045f), 0, 5, 0, seed);
  }
  if (group == 31) {  // dormers, arcade glazing, planters, roof services, antennas, awnings
    int m = i;
    if (type == 0) {
      if (m < 12) {
        int k = m / 3, r = m % 3;
        float xx = x + (k % 2 == 0 ? -w * 0.68f : w * 0.68f), zz = z + (float(k / 2) - 0.5f) * d * 0.96f;
        if (r == 0) return makeFeat(L, mk(xx, h + 2.5f, zz), mk(1.35f, 1.05f, 1.05f), 0, 0, 0, seed);
        if (r == 1) return makeFeat(L, mk(xx, h + 3.55f, zz), mk(1.45f, 1.0f, 1.2f), 3, 2, 1, seed);
        return makeFeat(L, mk(xx + (k % 2 == 0 ? -1.36f : 1.36f), h + 2.5f, zz), mk(0.035f, 0.70f, 0.65f), 0, 4, 0, seed);
      }
      m -= 12;
    }
    if (m < 12) {
      int face = m / 3, r = m % 3;
      if (r == 0) return makeWall(L, face, x, z, w - 3.5f, d - 3.5f, 0.0f, 1.6f, 0.045f, 1.05f, 1.4f, 0.055f, 4, seed);
      if (r == 1) return makeWall(L, face, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.13f, 0.09f, 1.25f, 0.15f, 0.12f, 13, seed);
      return makeWall(L, face, x, z, w - 3.5f, d - 3.5f, 0.0f, 0.18f, 0.18f, 1.25f, 0.10f, 0.35f, 0, seed);
    }
    m -= 12;
    if (m < 6) {
      int k = m >> 1;
      float xx = x + (float(k) - 1.0f) * 7.0f;
      if ((m & 1) == 0) return makeFeat(L, mk(xx, 0.48f, z + d + 1.5f), mk(0.52f, 0.42f, 0.52f), 2, 14, 0, seed);
      return makeFeat(L, mk(xx, 1.13f, z + d + 1.5f), mk(0.7f, 0.8f, 0.7f), 1, 7, 0, seed + float(k));
    }
    m -= 6;
    if (m < 8) {
      int k = m >> 1;
      float xx = x + (float(k % 2) - 0.5f) * w, zz = z + (float(k / 2) - 0.5f) * d;
      if ((m & 1) == 0) return makeFeat(L, mk(xx, h + 0.72f, zz), mk(0.34f, 0.48f, 0.34f), 2, 6, 0, seed + 800.0f + float(k));
      return makeFeat(L, mk(xx, h + 1.18f, zz), mk(0.46f, 0.055f, 0.46f), 0, 13, 0, seed + 820.0f + float(k));
    }
    m -= 8;
    if (m < 8)
      return makeFeat(L, mk(x + EighthCos(m) * w * 0.44f, h + 0.42f, z + EighthSin(m) * d * 0.44f),
                      mk(0.055f, 0.42f, 0.055f), 2, 6, 0, seed + 840.0f + float(m));
    m -= 8;
    return makeWall(L, m, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.1f, 0.6f, 1.38f, 0.10f, 0.7f, (int(seed)) % 2 == 0 ? 14 : 2,
                    seed + 940.0f + float(m));
  }
  if (group < 56) {  // balconies of one storey, rails and brackets
    int face = (group - 32) / 6, row = (group - 32) % 6;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
    if (i < 32) {
      int j = i >> 3, r = i & 7;
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      if (r == 0) return makeWall(L, face, x, z, w, d, u, y - 1.18f, 0.56f, 1.16f, 0.085f, 0.65f, 13, seed);
      if (r == 1) return makeWall(L, face, x, z, w, d, u, y - 0.28f, 1.12f, 1.15f, 0.035f, 0.035f, 6, seed);
      if (r == 2) return makeWall(L, face, x, z, w, d, u, y - 1.00f, 1.12f, 1.15f, 0.026f, 0.026f, 6, seed);
      int k = r - 3;
      return makeWall(L, face, x, z, w, d, u + (float(k) - 2.0f) * 0.53f, y - 0.64f, 1.12f, 0.025f, 0.37f, 0.026f, 6, seed);
    }
    int m = i - 32;
    if (m < 8) {
      int j = m >> 1;
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      if ((m & 1) == 0) return makeWall(L, face, x, z, w, d, u, y - 0.22f, 1.17f, 1.20f, 0.028f, 0.035f, 6, seed + 600.0f + float(j));
      return makeWall(L, face, x, z, w, d, u, y - 1.23f, 0.62f, 1.19f, 0.038f, 0.038f, 6, seed + 620.0f + float(j));
    }
    m -= 8;
    int j = m >> 1;
    float u = (float(j) - 1.5f) * (ext * 0.48f);
    if ((m & 1) == 0) return makeWall(L, face, x, z, w, d, u - 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 640.0f + float(j));
    return makeWall(L, face, x, z, w, d, u + 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 660.0f + float(j));
  }
  if (group < 60) {  // quoins, and the rose window of towers
    int face = group - 56;
    float ext = face % 2 == 0 ? w : d;
    if (i < 28) {
      int k = i >> 1;
      float yy = 4.45f + float(k) * (h - 4.0f) / 14.0f, width = k % 2 == 0 ? 0.52f : 0.30f;
      if ((i & 1) == 0) return makeWall(L, face, x, z, w, d, -ext + width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
      return makeWall(L, face, x, z, w, d, ext - width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
    }
    f3 c = mk(x, h - 2.3f, z + (face == 0 ? d + 0.21f : -d - 0.21f));
    if (face % 2 == 1) c = mk(x + (face == 1 ? w + 0.21f : -w - 0.21f), h - 2.3f, z);
    if (i == 28) return makeFeat(L, c, mk(2.35f, 2.35f, 0.26f), 7, 13, face % 2, seed);
    return makeFeat(L, c, mk(1.85f, 1.85f, 0.032f), 1, 17, face % 2, seed);
  }
  if (group < 62) {  // roof slats of one side
    int side = group - 60, roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
    float zz = z - d + (float(i + side * 32) + 0.5f) * d / 32.0f;
    return makeFeat(L, mk(x, h + 0.395f, zz), mk(w + 0.46f, 4.42f, 0.023f), 3, roofmat, 0, seed);
  }
  if (group == 62) {  // curbs
    int side = i >> 4, k = i & 15;
    float u = -15.5f + float(k) * 2.0f;
    return makeFeat(L, mk(x + u, 0.16f, z + (side == 0 ? -16.3f : 16.3f)), mk(0.98f, 0.19f, 0.19f), 0, 0, 0, seed);
  }
  int face = i >> 3, k = i & 7;  // group 63: roofline brackets
  float ext = face % 2 == 0 ? w : d, u = (float(k) - 3.5f) * ext * 0.25f;
  return makeWall(L, face, x, z, w, d, u, h - 0.36f, 0.48f, 0.12f, 0.24f, 0.24f, 13, seed);
}

}  // namespace st
