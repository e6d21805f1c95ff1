// Ray-batch queries against a view's lot table: the nearest feature hit of
// arbitrary rays, through the hierarchy (kernels/trace.cu:8-61 of the
// reference) or exhaustively -- the same lot DDA, but every group of every
// visited lot evaluated in index order with no node culling.  The second form
// is the check of the first (the reference's own hierarchy-vs-exhaustive test,
// tests/native_harness.cpp:68-79, at any scale).
#include "common_api.cuh"
#include "traverse.cuh"

namespace st {

// The DDA of trace.cu:40-57 with every group of each visited lot evaluated in
// order (first wins on ties).
SD TraceResult traceExhaustive(const float* __restrict__ W, uint32_t o0, uint32_t o2, f3 ro, f3 rd, float cone) {
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
  if (!(nearT <= farT)) return r;
  float t = nearT + 0.0002f;
  f3 start = ro + rd * t;
  int cx = int(floorf((start.x + 18.0f) / kCell)), cz = int(floorf((start.z + 18.0f) / kCell));
  int sx = rd.x > 0.0f ? 1 : -1, sz = rd.z > 0.0f ? 1 : -1;
  float ix = guardedInv(rd.x), iz = guardedInv(rd.z);
  float tx = (float(cx) * kCell + (sx > 0 ? 18.0f : -18.0f) - ro.x) * ix;
  float tz = (float(cz) * kCell + (sz > 0 ? 18.0f : -18.0f) - ro.z) * iz;
  float dx = kCell * fabsf(ix), dz = kCell * fabsf(iz);
#pragma unroll 1
  for (int step = 0; step < 160; step++) {
    if (t > r.t || t > farT || t > kFar) break;
    int slot = tableSlot(o0, o2, cx, cz);
    LotDesc lot = loadLot(W, slot);
    f3 cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
    f3 lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
#pragma unroll 1
    for (int g = 0; g < kGroups; g++) {
      HitSink s{lr, ld, cone, r.t, -1, Feat{}};
      runGroup(lot, g, s);
      if (s.fid >= 0 && s.t < r.t) {
        r.t = s.t; r.fid = g * kMaxFeatures + s.fid; r.material = s.f.material; r.seed = s.f.seed; r.slot = slot;
        r.normal = fromLot(featureNormal(s.f, lr + ld * s.t), lot.turn);
      }
    }
    if (tx < tz) { t = tx; tx += dx; cx += sx; } else { t = tz; tz += dz; cz += sz; }
  }
  return r;
}

// Rays: n x 7 floats [ro.xyz, rd.xyz, cone] in the table's floating-origin
// frame.  Out: n x 8 floats [t, fid, material, seed, n.xyz, slot].
__global__ void __launch_bounds__(64) traceRaysK(const float* __restrict__ W, const float* __restrict__ N,
                                                const uint32_t* __restrict__ O, const float* __restrict__ rays, int n,
                                                int exhaustive, float* out) {
  int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float* q = rays + size_t(i) * 7;
  f3 ro = mk(q[0], q[1], q[2]), rd = mk(q[3], q[4], q[5]);
  TraceResult r = exhaustive ? traceExhaustive(W, O[0], O[2], ro, rd, q[6])
                             : traceRay(W, reinterpret_cast<const float4*>(N), O[0], O[2], ro, rd, q[6]);
  float4* o = reinterpret_cast<float4*>(out + size_t(i) * 8);
  o[0] = make_float4(r.t, float(r.fid), float(r.material), r.seed);
  o[1] = make_float4(r.normal.x, r.normal.y, r.normal.z, float(r.slot));
}

// One named feature of a table against one ray: the lot of `slot` (its
// descriptor, cell and turn, kernels/world.cu:37-56), record fid % 64 of group
// fid / 64 (the enumeration sink of kernels/sink.cu:21), intersected in that
// lot's frame exactly as the trace forms it (kernels/trace.cu:49-50).
// Out: [t, normal.xyz] (t = FAR if the ray misses it or the id names nothing).
__global__ void __launch_bounds__(64) retestFeaturesK(const float* __restrict__ W, const uint32_t* __restrict__ O,
                                                     const float* __restrict__ rays, const int* __restrict__ ids,
                                                     int n, float* out) {
  int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float* q = rays + size_t(i) * 7;
  const int slot = ids[2 * i], fid = ids[2 * i + 1];
  float4 r = make_float4(kFar, 0.0f, 0.0f, 0.0f);
  if (slot >= 0 && slot < kLots && fid >= 0 && fid < kGroups * kMaxFeatures) {
    const LotDesc lot = loadLot(W, slot);
    int cx, cz;
    slotCell(O[0], O[2], slot, cx, cz);
    const f3 ro = mk(q[0], q[1], q[2]), rd = mk(q[3], q[4], q[5]);
    const f3 cp = mk(float(cx) * kCell + lot.ox, 0.0f, float(cz) * kCell + lot.oz);
    const f3 lr = toLot(ro - cp, lot.turn), ld = toLot(rd, lot.turn);
    PickSink pick{fid % kMaxFeatures};
    runGroup(lot, fid / kMaxFeatures, pick);
    if (pick.f.shape >= 0) {
      const float t = featureHitCall(pick.f, lr, ld, q[6]);
      if (t > 0.001f && t < kFar) {
        const f3 nn = fromLot(featureNormal(pick.f, lr + ld * t), lot.turn);
        r = make_float4(t, nn.x, nn.y, nn.z);
      }
    }
  }
  reinterpret_cast<float4*>(out)[i] = r;
}

}  // namespace st

using namespace st;

extern "C" int stratum_retestFeatures(const float* World, const unsigned* Origin, const float* Rays, const int* Ids,
                                      int n, float* Out, stratum_stream_t stream) {
  if (!World || !Origin || !Rays || !Ids || !Out || n < 0) return STRATUM_EINVAL;
  if (n == 0) return STRATUM_OK;
  retestFeaturesK<<<(n + 63) / 64, 64, 0, asStream(stream)>>>(World, Origin, Rays, Ids, n, Out);
  return launchStatus();
}

extern "C" int stratum_traceRays(const float* World, const float* Nodes, const unsigned* Origin, const float* Rays,
                                 int n, int exhaustive, float* Out, stratum_stream_t stream) {
  if (!World || !Origin || !Rays || !Out || n < 0 || (!exhaustive && !Nodes)) return STRATUM_EINVAL;
  if (n == 0) return STRATUM_OK;
  traceRaysK<<<(n + 63) / 64, 64, 0, asStream(stream)>>>(World, Nodes, Origin, Rays, n, exhaustive, Out);
  return launchStatus();
}
