// The deterministic feature grammar (kernels/assets.cu:3-265 of the reference)
// as a device template over an emitter.
//
// One grammar serves the three sink modes of kernels/sink.cu: nearest-hit
// query, conservative group bounds and enumeration of feature #k.  The
// emitter decides what happens to each feature; the grammar only produces
// them, in the reference's order (the order defines each feature's index,
// fid = group * 64 + index).  The reference's level of detail is fixed at 5,
// so every `lod >= n` guard in it is true and is omitted here.  Loops carry
// `#pragma unroll 1` so each emission site exists once in the binary.
#pragma once
#include "stratum_math.cuh"
#include "trig_table.h"

namespace st {

struct Feat { f3 p, h; int shape, material, turn; float seed; };

template <class E> struct Emit {
  E& e;
  float roofBase, roofScale;
  int count;
  // kernels/sink.cu:10-13: features at or above the eave scale vertically.
  HD void operator()(f3 p, f3 h, int shape, int mat, int turn, float seed) {
    if (p.y >= roofBase) { p.y = roofBase + (p.y - roofBase) * roofScale; h.y *= roofScale; }
    e.take(Feat{p, h, shape, mat, turn, seed}, count);
    count++;
  }
  // kernels/sink.cu:27-33: a box on facade `face`, pushed `o` out of the wall.
  HD void wall(int face, float cx, float cz, float w, float d, float u, float y, float o, float hw, float hy, float hd,
               int mat, float seed) {
    f3 p = mk(cx + u, y, cz + d + o), h = mk(hw, hy, hd);
    if (face == 1) { p = mk(cx + w + o, y, cz + u); h = mk(hd, hy, hw); }
    if (face == 2) p = mk(cx + u, y, cz - d - o);
    if (face == 3) { p = mk(cx - w - o, y, cz + u); h = mk(hd, hy, hw); }
    (*this)(p, h, 0, mat, 0, seed);
  }
};

// Emits every feature of `group` of `lot` into `sink.take(feature, index)`;
// returns the feature count.
template <class E> HD int runGroup(const LotDesc& lot, int group, E& sink) {
  Emit<E> e{sink, lot.h, lot.roofScale, 0};
  const float x = 0.0f, z = 0.0f, w = lot.w, d = lot.d, h = lot.h, seed = lot.seed, storey = lot.storey;
  const int type = lot.type, mat = lot.mat, floors = lot.floors;
  if (type == 5) return 0;
  if (type == 4) {  // canal bridge
    if (group == 0) {
      e(mk(x, 0.25f, z), mk(18.0f, 0.5f, 5.0f), 0, 0, 0, seed);
      e(mk(x, 1.25f, z - 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
      e(mk(x, 1.25f, z + 5.0f), mk(18.0f, 0.2f, 0.23f), 0, 0, 0, seed);
#pragma unroll 1
      for (int k = 0; k < 12; k++) {
        float u = -16.5f + float(k) * 3.0f;
        e(mk(x + u, 0.8f, z - 5.0f), mk(0.12f, 0.6f, 0.12f), 2, 6, 0, seed);
        e(mk(x + u, 0.8f, z + 5.0f), mk(0.12f, 0.6f, 0.12f), 2, 6, 0, seed);
      }
    }
    return e.count;
  }
  if (type == 3) {  // park
    if (group == 0) e(mk(x, -0.12f, z), mk(15.5f, 0.22f, 15.5f), 0, 11, 0, seed);
    if (group >= 1 && group <= 8) {
      int k = group - 1;
      float tx = x + (k < 4 ? -10.0f : 10.0f), tz = z + (float(k % 4) - 1.5f) * 6.7f;
      float th = 5.0f + hash1(int(seed) + k) * 3.0f;
      e(mk(tx, th * 0.4f, tz), mk(0.19f, th * 0.4f, 0.19f), 2, 15, 0, seed);
#pragma unroll 1
      for (int j = 0; j < 28; j++) {
        float yy = hash1(int(seed) + j + 991) * 3.3f - 0.5f;
        float rr = sqrtf(hash1(int(seed) + j + 330)) * 2.1f * (1.0f - yy * 0.12f);
        float size = 0.48f + hash1(int(seed) + j + 62) * 0.30f;
        e(mk(tx + TreeCos(j) * rr, th + yy, tz + TreeSin(j) * rr), mk(size, size * 1.25f, size), 1, 7, 0,
          seed + float(j));
      }
    }
    if (group == 9) {
      e(mk(x, 0.8f, z), mk(3.6f, 0.45f, 3.6f), 2, 0, 0, seed);
      e(mk(x, 1.24f, z), mk(3.3f, 0.04f, 3.3f), 2, 9, 0, seed);
      e(mk(x, 2.0f, z), mk(0.65f, 1.0f, 0.65f), 2, 0, 0, seed);
      e(mk(x, 2.85f, z), mk(1.4f, 0.18f, 1.4f), 2, 13, 0, seed);
      e(mk(x, 3.15f, z), mk(0.5f, 0.5f, 0.5f), 1, 3, 0, seed);
    }
    return e.count;
  }
  // buildings: type 0 pitched roof, 1 dome, 2 tower
  if (group == 0) {
    e(mk(x, 0.15f, z), mk(w + 1.1f, 0.25f, d + 1.1f), 0, 0, 0, seed);
    e(mk(x, (h + 4.0f) * 0.5f, z), mk(w, (h - 4.0f) * 0.5f, d), 0, mat, 0, seed);
    e(mk(x, 4.0f, z), mk(w + 0.24f, 0.24f, d + 0.24f), 0, 13, 0, seed);
    e(mk(x, 1.9f, z), mk(w - 3.5f, 1.9f, d - 3.5f), 0, 5, 0, seed);
#pragma unroll 1
    for (int i = 0; i < 12; i++) {
      int f = i / 3, k = i % 3;
      float ext = (f % 2 == 0 ? w : d) - 0.65f, u = (float(k) - 1.0f) * ext;
      float px = f % 2 == 0 ? x + u : x + (f == 1 ? w - 0.5f : -w + 0.5f);
      float pz = f % 2 == 0 ? z + (f == 0 ? d - 0.5f : -d + 0.5f) : z + u;
      e(mk(px, 2.0f, pz), mk(0.38f, 1.75f, 0.38f), 2, 0, 0, seed + float(k));
      e(mk(px, 3.66f, pz), mk(0.64f, 0.18f, 0.64f), 0, 13, 0, seed);
    }
  }
  if (group == 1) {
    e(mk(x, h + 0.25f, z), mk(w + 0.6f, 0.24f, d + 0.6f), 0, 13, 0, seed);
    if (type == 0) {
      int roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
      e(mk(x, h + 0.35f, z), mk(w + 0.45f, 4.4f, d + 0.45f), 3, roofmat, 0, seed);
      e(mk(x, h + 4.8f, z), mk(0.12f, 0.14f, d + 0.7f), 0, 3, 0, seed);
#pragma unroll 1
      for (int k = 0; k < 4; k++) {
        float xx = x + (k % 2 == 0 ? -w * 0.52f : w * 0.52f), zz = z + (float(k / 2) - 0.5f) * d;
        e(mk(xx, h + storey, zz), mk(0.48f, 2.2f, 0.55f), 0, 1, 0, seed);
        e(mk(xx, h + 6.0f, zz), mk(0.66f, 0.17f, 0.72f), 0, 0, 0, seed);
        e(mk(xx, h + 6.32f, zz), mk(0.2f, 0.25f, 0.2f), 2, 14, 0, seed);
      }
    } else if (type == 1) {
      e(mk(x, h + 2.2f, z), mk(w * 0.72f, 2.0f, w * 0.72f), 2, 0, 0, seed);
      e(mk(x, h + 3.1f, z), mk(w * 0.79f, 8.4f, w * 0.79f), 1, 3, 0, seed);
      e(mk(x, h + 12.2f, z), mk(0.24f, 1.45f, 0.24f), 2, 6, 0, seed);
      e(mk(x, h + 13.8f, z), mk(0.6f, 0.6f, 0.6f), 1, 8, 0, seed);
    } else {
      e(mk(x, h + 0.4f, z), mk(w * 0.72f, 5.2f, d + 0.2f), 3, 2, 0, seed);
#pragma unroll 1
      for (int k = 0; k < 2; k++) {
        float xx = x + (k == 0 ? -w * 0.75f : w * 0.75f), zz = z + d * 0.60f;
        e(mk(xx, h + 3.5f, zz), mk(2.3f, 7.2f, 2.3f), 0, 0, 0, seed);
        e(mk(xx, h + 10.9f, zz), mk(2.65f, 0.35f, 2.65f), 0, 13, 0, seed);
        e(mk(xx, h + 11.2f, zz), mk(2.55f, 4.4f, 2.55f), 3, 3, 0, seed);
        e(mk(xx, h + 16.0f, zz), mk(0.17f, 1.2f, 0.17f), 2, 8, 0, seed);
#pragma unroll 1
        for (int j = 0; j < 4; j++)
          e(mk(xx + QuarterCos(j) * 2.2f, h + 12.0f, zz + QuarterSin(j) * 2.2f), mk(0.17f, 1.1f, 0.17f), 2, 0, 0,
            seed);
      }
    }
  }
  if (group >= 2 && group <= 5) {
    int face = group - 2;
    float ext = face % 2 == 0 ? w : d;
#pragma unroll 1
    for (int j = 0; j <= floors; j++) {
      float y = 4.2f + float(j) * storey;
      e.wall(face, x, z, w, d, 0.0f, y, 0.17f, ext + 0.15f, 0.11f, 0.22f, 13, seed);
      e.wall(face, x, z, w, d, 0.0f, y + 0.21f, 0.1f, ext + 0.10f, 0.052f, 0.16f, 0, seed);
    }
#pragma unroll 1
    for (int j = 0; j < 5; j++) {
      float u = (float(j) / 4.0f * 2.0f - 1.0f) * (ext - 0.3f);
      e.wall(face, x, z, w, d, u, (h + 4.0f) * 0.5f, 0.16f, 0.19f, (h - 4.0f) * 0.5f, 0.22f, 13, seed);
    }
#pragma unroll 1
    for (int j = 0; j < 8; j++) {
      float u = (float(j) - 3.5f) * (ext / 4.0f);
      e.wall(face, x, z, w, d, u, h - 0.24f, 0.4f, 0.15f, 0.12f, 0.19f, 13, seed);
    }
  }
  if (group >= 6 && group < 30) {
    int face = (group - 6) / 6, row = (group - 6) % 6;
    if (row >= floors) return e.count;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
#pragma unroll 1
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
  if (group == 30) {
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
      float px = x + (k == 0 ? -16.0f : 16.0f), pz = z + 15.9f;
      e(mk(px, 2.0f, pz), mk(0.068f, 2.0f, 0.068f), 2, 6, 0, seed);
      e(mk(px, 4.0f, pz), mk(0.29f, 0.38f, 0.29f), 0, 8, 0, seed);
      e(mk(px, 4.44f, pz), mk(0.37f, 0.1f, 0.37f), 3, 6, 0, seed);
      e(mk(px, 0.15f, pz), mk(0.27f, 0.18f, 0.27f), 2, 0, 0, seed);
    }
#pragma unroll 1
    for (int k = 0; k < 8; k++) e(mk(x - 14.9f, 0.43f, z - 12.0f + float(k) * 3.3f), mk(0.10f, 0.43f, 0.10f), 2, 6, 0, seed);
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
      int face = i / 2, k = i % 2;
      float ext = (face % 2 == 0 ? w : d) - 0.65f, u = (k == 0 ? -0.5f : 0.5f) * ext;
      f3 c = mk(x + u, 3.16f, z + (face == 0 ? d - 0.5f : -d + 0.5f));
      if (face % 2 == 1) c = mk(x + (face == 1 ? w - 0.5f : -w + 0.5f), 3.16f, z + u);
      e(c, mk(ext * 0.5f, 0.88f, 0.49f), 4, 13, face % 2, seed);
    }
  }
  if (group == 31) {
    if (type == 0) {
#pragma unroll 1
      for (int k = 0; k < 4; k++) {
        float xx = x + (k % 2 == 0 ? -w * 0.68f : w * 0.68f), zz = z + (float(k / 2) - 0.5f) * d * 0.96f;
        e(mk(xx, h + 2.5f, zz), mk(1.35f, 1.05f, 1.05f), 0, 0, 0, seed);
        e(mk(xx, h + 3.55f, zz), mk(1.45f, 1.0f, 1.2f), 3, 2, 1, seed);
        e(mk(xx + (k % 2 == 0 ? -1.36f : 1.36f), h + 2.5f, zz), mk(0.035f, 0.70f, 0.65f), 0, 4, 0, seed);
      }
    }
#pragma unroll 1
    for (int face = 0; face < 4; face++) {
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 1.6f, 0.045f, 1.05f, 1.4f, 0.055f, 4, seed);
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.13f, 0.09f, 1.25f, 0.15f, 0.12f, 13, seed);
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 0.18f, 0.18f, 1.25f, 0.10f, 0.35f, 0, seed);
    }
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
      float xx = x + (float(k) - 1.0f) * 7.0f;
      e(mk(xx, 0.48f, z + d + 1.5f), mk(0.52f, 0.42f, 0.52f), 2, 14, 0, seed);
      e(mk(xx, 1.13f, z + d + 1.5f), mk(0.7f, 0.8f, 0.7f), 1, 7, 0, seed + float(k));
    }
  }
  if (group >= 32 && group < 56) {
    int face = (group - 32) / 6, row = (group - 32) % 6;
    if (row >= floors) return e.count;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
#pragma unroll 1
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, y - 1.18f, 0.56f, 1.16f, 0.085f, 0.65f, 13, seed);
      e.wall(face, x, z, w, d, u, y - 0.28f, 1.12f, 1.15f, 0.035f, 0.035f, 6, seed);
      e.wall(face, x, z, w, d, u, y - 1.00f, 1.12f, 1.15f, 0.026f, 0.026f, 6, seed);
#pragma unroll 1
      for (int k = 0; k < 5; k++)
        e.wall(face, x, z, w, d, u + (float(k) - 2.0f) * 0.53f, y - 0.64f, 1.12f, 0.025f, 0.37f, 0.026f, 6, seed);
    }
  }
  if (group >= 56 && group < 60) {
    int face = group - 56;
    float ext = face % 2 == 0 ? w : d;
#pragma unroll 1
    for (int k = 0; k < 14; k++) {
      float yy = 4.45f + float(k) * (h - 4.0f) / 14.0f, width = k % 2 == 0 ? 0.52f : 0.30f;
      e.wall(face, x, z, w, d, -ext + width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
      e.wall(face, x, z, w, d, ext - width, yy, 0.12f, width, 0.16f, 0.16f, 0, seed);
    }
    if (type == 2) {
      f3 c = mk(x, h - 2.3f, z + (face == 0 ? d + 0.21f : -d - 0.21f));
      if (face % 2 == 1) c = mk(x + (face == 1 ? w + 0.21f : -w - 0.21f), h - 2.3f, z);
      e(c, mk(2.35f, 2.35f, 0.26f), 7, 13, face % 2, seed);
      e(c, mk(1.85f, 1.85f, 0.032f), 1, 17, face % 2, seed);
    }
  }
  if ((group == 60 || group == 61) && type == 0) {
    int side = group - 60, roofmat = hash1(int(seed)) > 0.5f ? 14 : 2;
#pragma unroll 1
    for (int j = 0; j < 32; j++) {
      float zz = z - d + (float(j + side * 32) + 0.5f) * d / 32.0f;
      e(mk(x, h + 0.395f, zz), mk(w + 0.46f, 4.42f, 0.023f), 3, roofmat, 0, seed);
    }
  }
  if (group == 62) {
#pragma unroll 1
    for (int i = 0; i < 32; i++) {
      int side = i / 16, k = i % 16;
      float u = -15.5f + float(k) * 2.0f;
      e(mk(x + u, 0.16f, z + (side == 0 ? -16.3f : 16.3f)), mk(0.98f, 0.19f, 0.19f), 0, 0, 0, seed);
    }
  }
  if (group == 63) {
#pragma unroll 1
    for (int i = 0; i < 32; i++) {
      int face = i / 8, k = i % 8;
      float ext = face % 2 == 0 ? w : d, u = (float(k) - 3.5f) * ext * 0.25f;
      e.wall(face, x, z, w, d, u, h - 0.36f, 0.48f, 0.12f, 0.24f, 0.24f, 13, seed);
    }
  }
  // hyperdetail bands (assets.cu:199-249)
  if (group >= 2 && group <= 5) {
    int face = group - 2;
    float ext = face % 2 == 0 ? w : d;
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
      float yy = 5.05f + float(k) * fmaxf(1.0f, (h - 6.0f) / 4.0f);
      e.wall(face, x, z, w, d, 0.0f, yy, 0.205f, ext + 0.08f, 0.035f, 0.055f, 13, seed + 410.0f + float(k));
    }
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
      float u = (float(k) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, h - 0.72f, 0.255f, 0.055f, 0.34f, 0.07f, 0, seed + 450.0f + float(k));
    }
  }
  if (group >= 6 && group < 30) {  // rows beyond `floors` returned above
    int face = (group - 6) / 6, row = (group - 6) % 6;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
#pragma unroll 1
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u - 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 500.0f + float(j));
      e.wall(face, x, z, w, d, u + 0.46f, y, 0.145f, 0.026f, 1.10f, 0.055f, 5, seed + 520.0f + float(j));
    }
#pragma unroll 1
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, y - 1.31f, 0.30f, 1.18f, 0.045f, 0.07f, 13, seed + 540.0f + float(j));
      e.wall(face, x, z, w, d, u, y + 1.31f, 0.18f, 1.08f, 0.038f, 0.055f, 13, seed + 560.0f + float(j));
    }
  }
  if (group >= 32 && group < 56) {  // rows beyond `floors` returned above
    int face = (group - 32) / 6, row = (group - 32) % 6;
    float ext = face % 2 == 0 ? w : d, y = 4.2f + storey * 0.5f + float(row) * storey;
#pragma unroll 1
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u, y - 0.22f, 1.17f, 1.20f, 0.028f, 0.035f, 6, seed + 600.0f + float(j));
      e.wall(face, x, z, w, d, u, y - 1.23f, 0.62f, 1.19f, 0.038f, 0.038f, 6, seed + 620.0f + float(j));
    }
#pragma unroll 1
    for (int j = 0; j < 4; j++) {
      float u = (float(j) - 1.5f) * (ext * 0.48f);
      e.wall(face, x, z, w, d, u - 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 640.0f + float(j));
      e.wall(face, x, z, w, d, u + 0.72f, y - 1.42f, 0.46f, 0.075f, 0.22f, 0.42f, 0, seed + 660.0f + float(j));
    }
  }
  if (group == 30) {
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
      float side = k < 2 ? -1.0f : 1.0f, along = (k % 2 == 0 ? -0.58f : 0.58f);
      e(mk(x + side * (w + 0.34f), h * 0.38f, z + along * d), mk(0.075f, h * 0.38f, 0.075f), 2, 6, 0,
        seed + 700.0f + float(k));
    }
#pragma unroll 1
    for (int k = 0; k < 4; k++)
      e(mk(x - 12.0f + float(k) * 8.0f, 0.48f, z + d + 2.0f), mk(0.12f, 0.48f, 0.12f), 2, 6, 0, seed + 720.0f + float(k));
#pragma unroll 1
    for (int k = 0; k < 8; k++)
      e(mk(x - 14.0f + float(k) * 4.0f, 0.055f, z - d - 2.2f), mk(1.75f, 0.035f, 0.045f), 0, 13, 0,
        seed + 740.0f + float(k));
  }
  if (group == 31) {
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
      float xx = x + (float(k % 2) - 0.5f) * w, zz = z + (float(k / 2) - 0.5f) * d;
      e(mk(xx, h + 0.72f, zz), mk(0.34f, 0.48f, 0.34f), 2, 6, 0, seed + 800.0f + float(k));
      e(mk(xx, h + 1.18f, zz), mk(0.46f, 0.055f, 0.46f), 0, 13, 0, seed + 820.0f + float(k));
    }
#pragma unroll 1
    for (int k = 0; k < 8; k++)
      e(mk(x + EighthCos(k) * w * 0.44f, h + 0.42f, z + EighthSin(k) * d * 0.44f), mk(0.055f, 0.42f, 0.055f), 2, 6, 0,
        seed + 840.0f + float(k));
  }
  // street benches and the awnings (assets.cu:252-263)
  if (group == 30) {
#pragma unroll 1
    for (int bench = 0; bench < 2; bench++) {
      float bx = bench == 0 ? -7.0f : 7.0f, bz = d + 1.8f;
#pragma unroll 1
      for (int slat = 0; slat < 4; slat++)
        e(mk(bx, 0.59f, bz + (float(slat) - 1.5f) * 0.13f), mk(1.3f, 0.045f, 0.053f), 0, 5, 0, seed + 900.0f + float(slat));
#pragma unroll 1
      for (int leg = 0; leg < 2; leg++) e(mk(bx + (leg == 0 ? -0.95f : 0.95f), 0.3f, bz), mk(0.065f, 0.3f, 0.27f), 0, 6, 0, seed);
#pragma unroll 1
      for (int rail = 0; rail < 2; rail++)
        e(mk(bx, 0.88f + float(rail) * 0.19f, bz + 0.23f), mk(1.3f, 0.075f, 0.045f), 0, 5, 0, seed);
    }
  }
  if (group == 31) {
#pragma unroll 1
    for (int face = 0; face < 4; face++)
      e.wall(face, x, z, w - 3.5f, d - 3.5f, 0.0f, 3.1f, 0.6f, 1.38f, 0.10f, 0.7f, (int(seed)) % 2 == 0 ? 14 : 2,
             seed + 940.0f + float(face));
  }
  return e.count;
}

// ---- emitters ---------------------------------------------------------------
// Bounds mode (kernels/sink.cu:15-20): AABB union with a 0.025 m pad.
struct BoundsSink {
  f3 lo{1000000.0f, 1000000.0f, 1000000.0f}, hi{-1000000.0f, -1000000.0f, -1000000.0f};
  HD void take(const Feat& f, int) {
    f3 ext = f.h;
    if (f.turn % 2 == 1) ext = mk(f.h.z, f.h.y, f.h.x);
    f3 a = f.p - ext, b = f.p + ext;
    if (f.shape == 3 || f.shape == 4) a.y = f.p.y;
    const f3 pad = mk(0.025f, 0.025f, 0.025f);
    lo = vmin(lo, a - pad);
    hi = vmax(hi, b + pad);
  }
};
// Enumeration mode (kernels/sink.cu:21): keep feature #target.
struct PickSink {
  int target;
  Feat f{mk(0.f, 0.f, 0.f), mk(1.f, 1.f, 1.f), -1, 0, 0, 0.0f};
  HD void take(const Feat& ft, int id) { if (id == target) f = ft; }
};

}  // namespace st
