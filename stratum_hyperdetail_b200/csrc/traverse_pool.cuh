// Block-pooled form of the warp-cooperative trace (kernels/trace.cu:8-28,40-57
// of the reference, reorganised): the P warps of a block each own one 8x4 tile
// and advance their lanes' rays exactly as in traceWarp (leaf queue included),
// but the groups their rays wait on are served by the block.  Every pending
// lane publishes its head (view, slot, group) and its ray in the lot frame to
// shared memory; each warp then serves the distinct heads that hash to it, for
// every waiting ray of the block, compacting the waiting rays by ballot so a
// pass of the test loop has up to 32 of them whatever warp owns them; the owners
// then take the new best and winner and move to their next queued leaf.
//
// Each ray still meets its leaves in the reference's order with its own running
// best (a serve applies exactly the record loop of traceWarp to the ray's lot
// frame and best), so results equal traceWarp's bit for bit.  Every block-wide
// barrier sits in a loop whose exit condition is block-uniform
// (__syncthreads_or), so all threads of the block, rays in flight or not, reach
// the same barriers.
#pragma once
#include "traverse_coop.cuh"

namespace st {

static_assert(kSpec > 1 && kKeys == 1, "the pooled trace serves queued leaves one group at a time");

template <int P>
struct PoolShared {
  WarpStage stage[P];
  float lr[3][P * 32], ld[3][P * 32], inv[3][P * 32];
  float best[P * 32], cone[P * 32];
  int key[P * 32];  // pending head (view << 20 | slot << 6 | group), or -1
  int fid[P * 32];  // winner (group * 64 + index) after a serve that improved best
};

SD int poolKey(int view, int slot, int group) { return (view << 20) | (slot << 6) | group; }
template <int P>
SD int poolWarpOf(int key) { return int((unsigned(key) * 2654435761u) >> 16) % P; }

// One ray of the block against the group staged in `ws` (the record loop of
// traceWarp, on the ray's state in shared memory).
template <int P>
SD void poolTest(PoolShared<P>& sh, int j, const WarpStage& ws, int count, int g) {
  const f3 lr = mk(sh.lr[0][j], sh.lr[1][j], sh.lr[2][j]);
  const f3 ld = mk(sh.ld[0][j], sh.ld[1][j], sh.ld[2][j]);
  const f3 inv0 = mk(sh.inv[0][j], sh.inv[1][j], sh.inv[2][j]);
  const float cone = sh.cone[j];
  float best = sh.best[j];
  int fid = -1;
#pragma unroll 1
  for (int c = 0; c * kRun < count; c++) {
    const ChunkBox b = ws.boxes[0][c];
    const Span cr = slabInv(lr, inv0, mk(b.lo[0], b.lo[1], b.lo[2]), mk(b.hi[0], b.hi[1], b.hi[2]));
    if (cr.hi < fmaxf(0.001f, cr.lo) || cr.lo > best) continue;  // no feature of the run can win
    const int kEnd = min(count, (c + 1) * kRun);
#pragma unroll 1
    for (int k = c * kRun; k < kEnd; k++) {
      const Feat f = unstage(ws.feats[0][k]);
      const bool odd = f.turn % 2 == 1;
      const f3 inv = odd ? mk(inv0.z, inv0.y, ld.x == 0.0f ? guardedInv(-ld.x) : -inv0.x) : inv0;
      const f3 p = intoFeature(lr - f.p, f.turn);
      const Span rg = featureSlab(f, p, inv);
      if (featureSlabMiss(f, rg)) continue;
      const f3 d = odd ? mk(ld.z, ld.y, -ld.x) : ld;
      const float th = featureAfterSlab(f, lr, ld, p, d, inv, rg, cone);
      if (th > 0.001f && th < best) {  // index order: the first feature wins ties
        best = th;
        fid = g * kMaxFeatures + k;
      }
    }
  }
  if (fid >= 0) {
    sh.best[j] = best;
    sh.fid[j] = fid;
  }
}

// The heads this warp serves, each for every waiting ray of the block.
// Warp-collective.
template <int P>
SD void poolServe(PoolShared<P>& sh, const stratum_view* __restrict__ V) {
  const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
  int kk[P];
  unsigned mine[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    kk[p] = sh.key[p * 32 + lane];
    mine[p] = __ballot_sync(0xffffffffu, kk[p] >= 0 && poolWarpOf<P>(kk[p]) == warp);
  }
#pragma unroll 1
  for (;;) {
    int key = -1;
#pragma unroll
    for (int p = 0; p < P; p++)
      if (key < 0 && mine[p]) key = __shfl_sync(0xffffffffu, kk[p], __ffs(mine[p]) - 1);
    if (key < 0) break;
    unsigned wait[P];
    int total = 0;
#pragma unroll
    for (int p = 0; p < P; p++) {
      wait[p] = __ballot_sync(0xffffffffu, kk[p] == key);
      mine[p] &= ~wait[p];
      total += __popc(wait[p]);
    }
    const int v = key >> 20, slot = (key >> 6) & (kLots - 1), g = key & 63;
    WarpStage& ws = sh.stage[warp];
    const int count = stageGroup(V[v].World, groupCache(V[v].Groups), (slot << 6) | g, ws, 0);
    __syncwarp();
    // the waiting rays, compacted: lane i takes the i-th of each 32
#pragma unroll 1
    for (int base = 0; base < total; base += 32) {
      int rank = base + lane, j = -1;
#pragma unroll
      for (int p = 0; p < P; p++) {
        const int c = __popc(wait[p]);
        if (j < 0 && rank < c) j = p * 32 + int(__fns(wait[p], 0, rank + 1));
        rank -= c;
      }
      if (j >= 0) poolTest<P>(sh, j, ws, count, g);
    }
    __syncwarp();
  }
}

// One ray per thread of a block of P warps.  Every thread of the block calls
// this (inactive rays included) and receives its ray's result.
template <int P>
SD TraceResult tracePooled(PoolShared<P>& sh, const stratum_view* __restrict__ V, int view, const float* __restrict__ W,
                           const float4* __restrict__ N, uint32_t o0, uint32_t o2, f3 ro, f3 rd, float cone,
                           bool active) {
  const int tid = int(threadIdx.x);
  CoopRay r;
  coopBegin(r, ro, rd, cone, active);
#pragma unroll 1
  for (;;) {
    coopAdvance(r, W, N, o0, o2);
    bool pend = r.state == kLeafPending;
    if (pend) {
      sh.lr[0][tid] = r.lr.x; sh.lr[1][tid] = r.lr.y; sh.lr[2][tid] = r.lr.z;
      sh.ld[0][tid] = r.ld.x; sh.ld[1][tid] = r.ld.y; sh.ld[2][tid] = r.ld.z;
      sh.inv[0][tid] = r.inv0.x; sh.inv[1][tid] = r.inv0.y; sh.inv[2][tid] = r.inv0.z;
      sh.best[tid] = r.best;
      sh.cone[tid] = r.cone;
    }
    sh.key[tid] = pend ? poolKey(view, r.slot, r.pend) : -1;
    if (!__syncthreads_or(pend)) break;  // every ray of the block is done
#pragma unroll 1
    for (;;) {
      poolServe<P>(sh, V);
      __syncthreads();
      if (pend) {
        if (sh.best[tid] < r.best) {  // the served group holds a nearer feature
          r.best = sh.best[tid];
          r.fid = sh.fid[tid];
          r.wslot = r.slot; r.wcx = r.lcx; r.wcz = r.lcz;
        }
        r.queue >>= 8;
        r.qn--;
#pragma unroll 1
        while (r.qn > 0 && !(nodeEntry(N, r.slot * kNodes + kGroups + int(r.queue & 255u), r.lr, r.inv0, r.best) < r.best)) {
          r.queue >>= 8;
          r.qn--;
        }
        if (r.qn > 0) {
          r.pend = int(r.queue & 255u);
        } else {
          r.state = kInLot;  // the walk goes on from where it stopped
          pend = false;
        }
        sh.key[tid] = pend ? poolKey(view, r.slot, r.pend) : -1;
      }
      if (!__syncthreads_or(pend)) break;
    }
  }
  TraceResult out;
  out.t = r.best; out.fid = r.fid; out.material = 10; out.seed = 0.0f; out.slot = -1;
  out.normal = mk(0.0f, 1.0f, 0.0f);
  if (r.fid >= 0) {  // the winner's record, lot frame and normal (trace.cu:53-54)
    const LotDesc L = loadLot(W, r.wslot);
    const Feat f = winnerFeature(groupCache(V[view].Groups), W, r.wslot, r.fid >> 6, r.fid & 63);
    f3 cp = mk(float(r.wcx) * kCell + L.ox, 0.0f, float(r.wcz) * kCell + L.oz);
    f3 lr = toLot(ro - cp, L.turn), ld = toLot(rd, L.turn);
    out.normal = fromLot(featureNormal(f, lr + ld * r.best), L.turn);
    out.material = f.material;
    out.seed = f.seed;
    out.slot = r.wslot;
  }
  return out;
}

}  // namespace st
