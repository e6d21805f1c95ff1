// Primary-ray traversal (kernels/trace.cu of the reference): ground plane,
// vertical slab, 2-D lot DDA over the scrolling table, and the near-first
// descent of each lot's 127-node hierarchy that re-runs the grammar for every
// reached group.  Shared by the drop-in kernel and the batched renderer.
#pragma once
#include "geometry.cuh"

namespace st {

struct TraceResult {
  float t, seed;
  int fid, material, slot;
  f3 normal;
};

// Node = two 128-bit loads: [lo.xyz, count], [hi.xyz, group].
SD float nodeEntry(const float4* __restrict__ N, int node, f3 ro, f3 inv, float best) {
  float4 a = __ldg(N + 2 * node);
  if (a.w < 0.5f) return kFar;
  float4 b = __ldg(N + 2 * node + 1);
  Span r = slabInv(ro, inv, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
  if (r.hi < fmaxf(0.001f, r.lo) || r.lo > best) return kFar;
  return fmaxf(0.001f, r.lo);
}

// Nearest hit inside one lot (trace.cu:8-28).  Returns true when a feature
// nearer than `best` was found; then best/fid/feature are updated.  Called only
// once the lot's root entry was found nearer than `best` (trace.cu:53).
SD bool queryLot(const LotDesc& lot, const float4* __restrict__ N, int slot, f3 ro, f3 rd, float cone, float& best,
                 int& fid, Feat& feature) {
  const f3 inv = invDir(rd);
  const int base = slot * kNodes;
  int stack[8], top = 0, node = 1, steps = 0;
  bool found = false;
  // A node reached from its parent (or the root, tested by the caller) was
  // found nearer than the same best a moment ago: the reference tests it again
  // with the same result, so only nodes popped from the stack are re-tested.
  bool fresh = true;
#pragma unroll 1
  while (node > 0 && steps < kNodes) {
    steps++;
    const bool near = fresh || nodeEntry(N, base + node, ro, inv, best) < best;
    fresh = false;
    if (near && node < kGroups) {
      int left = node * 2, right = left + 1;
      float ln = nodeEntry(N, base + left, ro, inv, best), rn = nodeEntry(N, base + right, ro, inv, best);
      bool lh = ln < best, rh = rn < best;
      fresh = lh || rh;
      if (lh && rh) {
        int next = ln < rn ? left : right, other = ln < rn ? right : left;
        stack[top++] = other;  // at most one push per level of the 6-level tree
        node = next;
      } else if (lh) node = left;
      else if (rh) node = right;
      else { node = 0; if (top > 0) node = stack[--top]; }
    } else {
      if (near && node >= kGroups) {
        HitSink s{ro, rd, cone, best, -1, Feat{}};
        runGroup(lot, node - kGroups, s);
        if (s.fid >= 0 && s.t < best) {
          best = s.t;
          fid = (node - kGroups) * kMaxFeatures + s.fid;
          feature = s.f;
          found = true;
        }
      }
      node = 0;
      if (top > 0) node = stack[--top];
    }
  }
  return found;
}

// Full primary visibility of one ray (trace.cu:29-61).
SD TraceResult traceRay(const float* __restrict__ W, const float4* __restrict__ N, uint32_t o0, uint32_t o2, f3 ro,
                        f3 rd, float cone) {
  TraceResult r;
  r.t = kFar; r.seed = 0.0f; r.fid = kSkyId; r.material = 10; r.slot = -1;
  r.normal = mk(0.0f, 1.0f, 0.0f);
  if (rd.y < -0.000001f) {
    float ground = -ro.y / rd.y;
    if (ground > 0.001f && ground < r.t) { r.t = ground; r.fid = kGroundId; }
  }
  float nearT = 0.001f, farT = r.t;
  if (fabsf(rd.y) > 0.0000001f) {
    float a = (-0.5f - ro.y) / rd.y, c = (kTop - ro.y) / rd.y;
    nearT = fmaxf(nearT, fminf(a, c));
    farT = fminf(farT, fmaxf(a, c));
  } else if (ro.y > kTop || ro.y < -0.5f) farT = -1.0f;
  if (nearT <= farT) {
    float t = nearT + 0.0002f;
    f3 start = ro + rd * t;
    int cx = int(floorf((start.x + 18.0f) / kCell)), cz = int(floorf((start.z + 18.0f) / kCell));
    int sx = rd.x > 0.0f ? 1 : -1, sz = rd.z > 0.0f ? 1 : -1;
    float ix = guardedInv(rd.x), iz = guardedInv(rd.z);
    float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * ix;
    float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * iz;
    float dx = kCell * fabsf(ix), dz = kCell * fabsf(iz);
    Feat feature;
#pragma unroll 1
    for (int step = 0; step < 160; step++) {
      if (t > r.t || t > farT || t > kFar) break;
      int slot = tableSlot(o0, o2, cx, cz);
      LotDesc lot = loadLot(W, slot);
      f3 cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
      f3 lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
      if (nodeEntry(N, slot * kNodes + 1, lr, invDir(ld), r.t) < r.t) {
        float best = r.t;
        int fid = -1;
        if (queryLot(lot, N, slot, lr, ld, cone, best, fid, feature) && best < r.t) {
          r.t = best; r.fid = fid; r.material = feature.material; r.seed = feature.seed;
          r.normal = fromLot(featureNormal(feature, lr + ld * best), lot.turn);
          r.slot = slot;
        }
      }
      if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
    }
  }
  return r;
}

SD void storeTrace(float* Hit, float* Surface, size_t px, const TraceResult& r) {
  reinterpret_cast<float4*>(Hit)[px] = make_float4(r.t, float(r.fid), float(r.material), r.seed);
  reinterpret_cast<float4*>(Surface)[px] = make_float4(r.normal.x, r.normal.y, r.normal.z, float(r.slot));
}

}  // namespace st
