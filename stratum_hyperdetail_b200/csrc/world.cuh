// Per-view camera step and per-slot lot refresh (kernels/world.cu:64-105 of the
// reference), shared by the single-view entry points and the batched kernels.
#pragma once
#include "stratum_math.cuh"

namespace st {

SD float expR(float a) { return float(exp(double(a))); }

// Input integration, bookmarks, tour, origin rebase with 64-bit carry, and the
// 64-sample counter (world.cu:64-92).  One thread per view.
__device__ __noinline__ static void stepOne(float* C, uint32_t* O, const float* I, float dt, int width, int height) {
  C[5] += dt; C[6] += 1.0f; C[13] = float(height); C[20] = float(width) / float(height);
  C[15] = I[23] > 0.5f ? 1.0f : 0.0f;
  int bm = int(I[8]);
  if (bm > 0) {  // bookmarks
    for (int i = 0; i < 4; i++) O[i] = 0u;
    if (bm == 1) { C[0] = 112.0f; C[1] = 76.0f; C[2] = 155.0f; C[3] = -2.53f; C[4] = -0.30f; C[12] = 38.0f; }
    if (bm == 2) { C[0] = 18.0f; C[1] = 1.75f; C[2] = 49.0f; C[3] = -2.80f; C[4] = 0.17f; C[12] = 6.0f; }
    if (bm == 3 || bm == 6) { C[0] = 17.0f; C[1] = 6.9f; C[2] = 0.0f; C[3] = -kPi * 0.5f; C[4] = 0.015f; C[12] = 0.8f; }
    if (bm == 4) { C[0] = 400.0f; C[1] = 650.0f; C[2] = 750.0f; C[3] = -2.61f; C[4] = -0.66f; C[12] = 180.0f; }
    if (bm == 5) { C[0] = 28.0f * kCell + 20.0f; C[1] = 8.0f; C[2] = 75.0f; C[3] = -2.65f; C[4] = -0.04f; C[12] = 12.0f; }
    C[15] = 1.0f;
  }
  if (I[3] != 0.0f || I[4] != 0.0f) {  // look
    C[3] += I[3] * 0.0022f;
    C[4] = clampv(C[4] - I[4] * 0.0022f, -1.53f, 1.53f);
    C[15] = 1.0f;
  }
  if (I[7] != 0.0f) C[12] = clampv(C[12] * expR(-I[7] * 0.0015f), 0.03f, 800.0f);
  float speed = C[12] * (I[5] > 0.5f ? 3.0f : 1.0f) * (I[6] > 0.5f ? 0.15f : 1.0f);
  float s3 = sinR(C[3]), c3 = cosR(C[3]), s4 = sinR(C[4]), c4 = cosR(C[4]);
  f3 fwd = mk(s3 * c4, s4, c3 * c4), right = mk(c3, 0.0f, -s3);
  f3 move = fwd * I[0] + right * I[1] + mk(0.0f, I[2], 0.0f);
  if (dot(move, move) > 0.0f) {
    move = unit(move) * speed * dt;
    C[0] += move.x; C[1] = clampv(C[1] + move.y, 0.08f, 1500.0f); C[2] += move.z; C[15] = 1.0f;
  }
  if (I[9] != 0.0f) { C[7] += I[9] * dt * 0.35f; C[15] = 1.0f; }
  if (I[10] > 0.0f) { C[11] = float((int(C[11]) + 1) % 4); C[15] = 1.0f; }
  if (I[13] != 0.0f) { C[9] = clampv(C[9] + I[13] * dt, 0.25f, 3.0f); C[15] = 1.0f; }
  if (I[14] > 0.0f) { C[18] = 1.0f - C[18]; C[15] = 1.0f; }
  if (I[16] > 0.0f) C[22] = 1.0f - C[22];
  if (C[22] > 0.5f) {  // guided tour
    C[3] += dt * 0.032f;
    float t3 = sinR(C[3]), u3 = cosR(C[3]);
    f3 f = mk(t3 * c4, s4, u3 * c4);
    C[0] += f.x * dt * 14.0f; C[2] += f.z * dt * 14.0f; C[15] = 1.0f;
  }
  int dx = int(floorf((C[0] + 18.0f) / kCell)), dz = int(floorf((C[2] + 18.0f) / kCell));
  if (dx != 0 || dz != 0) {  // floating-origin rebase
    Addr a = shiftAddr(O[0], O[1], O[2], O[3], dx, dz);
    O[0] = a.xl; O[1] = a.xh; O[2] = a.zl; O[3] = a.zh;
    C[0] -= float(dx) * kCell; C[2] -= float(dz) * kCell;
  }
  C[19] = C[15] > 0.5f ? 1.0f : fminf(64.0f, C[19] + 1.0f);
}

// Recompute one slot's 64-bit address; when the stored tag differs, describe
// the lot, store descriptor and tag, and append the slot to the refresh queue
// (world.cu:94-105).  Queue order is the order of the atomics, so it varies
// between runs; its contents do not.
SD void refreshSlot(int slot, const uint32_t* O, int seed, float* W, uint32_t* T, uint32_t* Q) {
  const uint32_t o0 = O[0], o1 = O[1], o2 = O[2], o3 = O[3];
  int cx, cz;
  slotCell(o0, o2, slot, cx, cz);
  Addr a = shiftAddr(o0, o1, o2, o3, cx, cz);
  float4* w4 = reinterpret_cast<float4*>(W + slot * kLotFloats);
  uint4* t4 = reinterpret_cast<uint4*>(T + slot * 4);
  uint4 tag = *t4;
  float4 last = w4[3];
  if (last.w > 0.5f && tag.x == a.xl && tag.y == a.xh && tag.z == a.zl && tag.w == a.zh) return;
  LotDesc l = describe(a, seed);
  w4[0] = make_float4(l.w, l.d, l.h, float(l.type));
  w4[1] = make_float4(float(l.mat), float(l.floors), l.seed, l.storey);
  w4[2] = make_float4(l.roofScale, float(l.turn), l.ox, l.oz);
  w4[3] = make_float4(l.palette, last.y, last.z, 1.0f);  // words 13-14 are left as they were
  *t4 = make_uint4(a.xl, a.xh, a.zl, a.zh);
  uint32_t i = atomicAdd(&Q[0], 1u);
  if (i < uint32_t(kLots)) Q[i + 1] = uint32_t(slot);  // an uncleared queue never writes past its end
}

}  // namespace st
