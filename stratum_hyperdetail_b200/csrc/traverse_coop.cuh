// Warp-cooperative primary traversal for the batched renderer.
//
// Same algorithm as traverse.cuh (kernels/trace.cu of the reference), same
// results bit for bit, organised for a warp of 32 coherent rays (one 8x4 tile):
//
//  * each lane advances its own ray -- lot DDA, then the near-first descent of
//    the lot's hierarchy -- until it reaches a leaf (a group) that must be
//    evaluated, or finishes;
//  * the warp then evaluates pending leaves one distinct (lot, group) key at a
//    time: the group's records are staged in shared memory, one per lane --
//    loaded from the table's group cache (group_cache.cuh) when it holds the
//    group, else built by the random-access grammar (grammar_ra.cuh) and, when
//    the cache has room, stored there for every later evaluation -- and every
//    lane waiting on that key tests them in index order with one inlined
//    intersection routine and its precomputed inverse directions;
//  * the winner's normal, material and seed are recomputed once per ray.
//
// Each lane's leaves are visited in the reference's order and each test sees
// the same running best, so identity, distance and normal equal the
// per-thread traversal exactly.  The per-lot hierarchy stack is packed into
// one 64-bit word (7 bits per node, at most 6 entries).
#pragma once
#include "geometry.cuh"
#include "grammar_ra.cuh"
#include "group_cache.cuh"
#include "traverse.cuh"

namespace st {

// featureAt out of line: one copy, away from the hot test loop in the
// instruction cache (measured faster than inlining it).
static __device__ __noinline__ Feat featureAtOOL(LotDesc L, int g, int i) { return featureAt(L, g, i); }

// Sub-group culling: every run of kRun staged features gets a box (in the
// lot frame) that contains every distance any of them can return, and a lane
// tests a run's features only when its ray enters that box nearer than its
// current best, so a skipped feature could only have been rejected and
// results are unchanged.  That holds for the features whose computed distance
// is a slab entry of their own box or follows from it: plain boxes and prisms
// (the slab entry, or a roof plane behind it), masonry boxes (relief moves the
// hit at most 0.0025 m toward the ray per unit of the face normal, inside the
// 0.025 m pad) and foliage envelopes (leaf discs reach at most one 0.18 m grid
// cell, 0.31 m diagonal, beyond the envelope's box: 0.35 m pad).  Ellipsoids,
// cylinders and arches/rings solve a quadratic whose float result can land
// well outside the box at long range (cancellation; 0.17 m at 1.4 km was
// seen), so their box is only bounded along the axis the intersection code
// itself checks: a cylinder's side hit is kept only when its height is within
// +-h.y and its caps lie at +-h.y, so its distance is inside the y slab; an
// arch or ring keeps hits within +-h.z of its own frame (lot x or z by its
// turn); an ellipsoid's root is not checked at all, so its box is unbounded.
// (Testing quadrics alone in a culled run, or staging them apart, measured
// slower: lanes then diverge inside the run.)
#ifndef STRATUM_COOP_RUN
#define STRATUM_COOP_RUN 4
#endif
constexpr int kRun = STRATUM_COOP_RUN;
static_assert(kRun * kEntryBoxes >= kEntryRecords, "a group cache entry holds every chunk box of a group");
struct ChunkBox { float lo[3], hi[3]; };
SD void hitBox(const Feat& f, f3& lo, f3& hi) {
  const bool foliage = f.shape == 1 && f.material == 7;
  f3 ext = f.h;
  if (f.turn % 2 == 1) ext = mk(f.h.z, f.h.y, f.h.x);
  const float pad = foliage ? 0.35f : 0.025f;
  lo = f.p - ext - mk(pad, pad, pad);
  hi = f.p + ext + mk(pad, pad, pad);
  const float open = 1e30f;
  if (f.shape == 1 && !foliage) {  // ellipsoid: unbounded
    lo = mk(-open, -open, -open);
    hi = mk(open, open, open);
  } else if (f.shape == 2) {  // cylinder: the y slab only
    lo.x = lo.z = -open;
    hi.x = hi.z = open;
  } else if (f.shape == 4 || f.shape == 7) {  // arch, ring: its own z slab only (lot x when the turn is odd)
    lo.y = -open;
    hi.y = open;
    if (f.turn % 2 == 1) { lo.z = -open; hi.z = open; } else { lo.x = -open; hi.x = open; }
  }
}

enum LaneState : int { kEnterLot = 0, kInLot = 1, kLeafPending = 2, kDone = 3 };

// Leaves a lane may find ahead in its lot before the warp evaluates them.  With
// more than one, a lane that reaches a leaf keeps walking the lot's hierarchy
// (near-first, against the best it has) and queues up to this many leaves; each
// queued leaf is tested again against the lane's best when it comes up, so the
// lane evaluates exactly the reference's leaves in the reference's order (a
// leaf that passes has ancestors that pass: parents bound their children).
#ifndef STRATUM_SPEC_LEAVES
#define STRATUM_SPEC_LEAVES 4
#endif
constexpr int kSpec = STRATUM_SPEC_LEAVES;
static_assert(kSpec >= 1 && kSpec <= 4, "up to four queued leaves (8 bits each in one word)");

struct CoopRay {
  // ray and result
  f3 ro, rd;
  float cone, best;
  int fid, wslot, wcx, wcz;  // winner: group*64+index, slot and DDA cell of its lot
  // lot DDA
  float t, tx, tz, dx, dz, farT;
  int cx, cz, sx, sz, ddaSteps;
  // current lot
  int slot, lcx, lcz;
  f3 lr, ld, inv0;
  // hierarchy walk
  unsigned long long stack;
  int node, qsteps, pend, state;
  int fresh;  // node's entry was just found nearer than best (by its parent's test)
#if STRATUM_SPEC_LEAVES > 1
  unsigned queue;  // queued leaves of the current lot: group indices, 8 bits each, the head lowest
  int qn;
#endif
};

SD int popNode(unsigned long long& stack) {
  int n = int(stack & 127ull);
  stack >>= 7;
  return n;
}

// Ray set-up: ground plane and vertical slab (trace.cu:33-45).
SD void coopBegin(CoopRay& r, f3 ro, f3 rd, float cone, bool active) {
  r.ro = ro; r.rd = rd; r.cone = cone;
  r.best = kFar; r.fid = kSkyId; r.wslot = -1; r.wcx = r.wcz = 0;
  r.state = active ? kEnterLot : kDone;
  r.stack = 0ull; r.node = 0; r.qsteps = 0; r.pend = 0; r.slot = 0; r.lcx = r.lcz = 0; r.fresh = 0;
  r.ddaSteps = 0;
#if STRATUM_SPEC_LEAVES > 1
  r.queue = 0u; r.qn = 0;
#endif
  if (!active) return;
  if (rd.y < -0.000001f) {
    float ground = -ro.y / rd.y;
    if (ground > 0.001f && ground < r.best) { r.best = ground; r.fid = kGroundId; }
  }
  float nearT = 0.001f, farT = r.best;
  if (fabsf(rd.y) > 0.0000001f) {
    float a = (-0.5f - ro.y) / rd.y, c = (kTop - ro.y) / rd.y;
    nearT = fmaxf(nearT, fminf(a, c));
    farT = fminf(farT, fmaxf(a, c));
  } else if (ro.y > kTop || ro.y < -0.5f) farT = -1.0f;
  r.farT = farT;
  if (!(nearT <= farT)) { r.state = kDone; return; }
  r.t = nearT + 0.0002f;
  f3 start = ro + rd * r.t;
  r.cx = int(floorf((start.x + 18.0f) / kCell));
  r.cz = int(floorf((start.z + 18.0f) / kCell));
  r.sx = rd.x > 0.0f ? 1 : -1;
  r.sz = rd.z > 0.0f ? 1 : -1;
  float ix = guardedInv(rd.x), iz = guardedInv(rd.z);
  r.tx = (float(r.cx) * kCell + (r.sx > 0 ? 18.0f : -18.0f) - ro.x) * ix;
  r.tz = (float(r.cz) * kCell + (r.sz > 0 ? 18.0f : -18.0f) - ro.z) * iz;
  r.dx = kCell * fabsf(ix);
  r.dz = kCell * fabsf(iz);
}

// Advance one lane until it needs a leaf evaluated or is done.
SD void coopAdvance(CoopRay& r, const float* __restrict__ W, const float4* __restrict__ N, uint32_t o0, uint32_t o2) {
#pragma unroll 1
  while (r.state == kEnterLot || r.state == kInLot) {
    if (r.state == kEnterLot) {
      if (r.ddaSteps >= 160 || r.t > r.best || r.t > r.farT || r.t > kFar) { r.state = kDone; break; }
      r.ddaSteps++;
      r.slot = tableSlot(o0, o2, r.cx, r.cz);
      r.lcx = r.cx; r.lcz = r.cz;
      const float4 c = __ldg(reinterpret_cast<const float4*>(W + r.slot * kLotFloats) + 2);  // roofScale, turn, ox, oz
      const int turn = int(c.y);
      f3 cp = mk(float(r.cx) * kCell + c.z, 0.0f, float(r.cz) * kCell + c.w);
      r.lr = toLot(r.ro - cp, turn);
      r.ld = toLot(r.rd, turn);
      r.inv0 = invDir(r.ld);
      // the DDA steps to the next cell now; the reference does it after the
      // lot's query, and the next test reads only t and the (later) best
      if (r.tx < r.tz) { r.t = r.tx; r.tx += r.dx; r.cx += r.sx; } else { r.t = r.tz; r.tz += r.dz; r.cz += r.sz; }
      if (nodeEntry(N, r.slot * kNodes + 1, r.lr, r.inv0, r.best) < r.best) {
        r.state = kInLot; r.node = 1; r.stack = 0ull; r.qsteps = 0; r.fresh = 1;
      }
      continue;
    }
    if (r.node <= 0 || r.qsteps >= kNodes) {
#if STRATUM_SPEC_LEAVES > 1
      if (r.qn > 0) { r.state = kLeafPending; r.pend = int(r.queue & 255u); break; }  // this lot's leaves first
#endif
      r.state = kEnterLot;
      continue;
    }
    r.qsteps++;
    const int base = r.slot * kNodes;
    // A node reached from its parent was tested against the same best a
    // moment ago (the reference tests it again, with the same result); a node
    // popped from the stack is tested again against the current best.
    const bool near = r.fresh || nodeEntry(N, base + r.node, r.lr, r.inv0, r.best) < r.best;
    r.fresh = 0;
    if (near && r.node < kGroups) {
      int left = r.node * 2, right = left + 1;
      float ln = nodeEntry(N, base + left, r.lr, r.inv0, r.best), rn = nodeEntry(N, base + right, r.lr, r.inv0, r.best);
      bool lh = ln < r.best, rh = rn < r.best;
      r.fresh = lh || rh;
      if (lh && rh) {
        int next = ln < rn ? left : right, other = ln < rn ? right : left;
        r.stack = (r.stack << 7) | (unsigned long long)other;
        r.node = next;
      } else if (lh) r.node = left;
      else if (rh) r.node = right;
      else r.node = popNode(r.stack);
    } else {
#if STRATUM_SPEC_LEAVES > 1
      if (near && r.node >= kGroups) {
        r.queue |= unsigned(r.node - kGroups) << (8 * r.qn);
        r.qn++;
        r.node = popNode(r.stack);
        if (r.qn == kSpec) { r.state = kLeafPending; r.pend = int(r.queue & 255u); break; }
        continue;
      }
#else
      if (near && r.node >= kGroups) { r.state = kLeafPending; r.pend = r.node - kGroups; break; }
#endif
      r.node = popNode(r.stack);
    }
  }
}

// Inverse of the turn-1 direction (ld.z, ld.y, -ld.x): a permutation of inv0
// with one sign flipped, except for an exactly zero ld.x, whose guarded inverse
// keeps the sign of the zero.
SD f3 inv1Of(const CoopRay& r) {
  return mk(r.inv0.z, r.inv0.y, r.ld.x == 0.0f ? guardedInv(-r.ld.x) : -r.inv0.x);
}

// The winner's record for one lane: from the group cache when it holds the
// group, else from the grammar.
SD Feat winnerFeature(const GroupCache& c, const float* __restrict__ W, int slot, int g, int i) {
  const LotDesc L = loadLot(W, slot);
  const int e = c.base ? usableEntry(c, __ldcg(c.dir(slot, g))) : -1;
  if (e >= 0) {
    // the tag (nine descriptor words, group, count) and the record in one round trip
    const uint4* t4 = reinterpret_cast<const uint4*>(entryTag(c, uint32_t(e)));
    const uint4 t0 = __ldg(t4), t1 = __ldg(t4 + 1), t2 = __ldg(t4 + 2);
    const StagedFeat rec = cacheRecord(c, e, i);
    const uint4* r4 = reinterpret_cast<const uint4*>(W + size_t(slot) * kLotFloats);
    const uint4 w0 = __ldg(r4), w1 = __ldg(r4 + 1), w2 = __ldg(r4 + 2);
    const bool same = t0.x == w0.x && t0.y == w0.y && t0.z == w0.z && t0.w == w0.w && t1.x == w1.x &&
                      t1.y == w1.y && t1.z == w1.z && t1.w == w1.w && t2.x == w2.x &&
                      t2.y == uint32_t(g) && t2.z == uint32_t(groupCount(L, g));
    if (same) return unstage(rec);
  }
  return featureAtOOL(L, g, i);
}

// Groups a warp stages and tests at once: lanes waiting on different groups
// then test concurrently, each its own group's records.  One group at a time
// measured fastest on the six benchmark poses (2, 3, 4 groups: frame 6 %, 16 %,
// 27 % slower, the aerial view included), so the default is 1.
#ifndef STRATUM_COOP_KEYS
#define STRATUM_COOP_KEYS 1
#endif
constexpr int kKeys = STRATUM_COOP_KEYS;
constexpr int kRunsPerGroup = (kEntryRecords + kRun - 1) / kRun;
// Shared memory of one warp: kKeys groups of up to 56 records and their chunk boxes.
struct WarpStage {
  StagedFeat feats[kKeys][kEntryRecords];
  ChunkBox boxes[kKeys][kRunsPerGroup];
};

// Group records shared by the warps of one block, for a trace with no
// table-wide group cache (the drop-in entry point).  Write-once for the
// block's life: a warp that builds a group copies it into the next free entry
// and then marks it ready; entries are never replaced, so a warp that finds a
// ready entry reads the records in place.  Two warps that miss the same group
// at once may both insert it (harmless).  At most 32 entries: one lane checks
// each entry per lookup.
#ifndef STRATUM_BLOCK_CACHE_ENTRIES
#define STRATUM_BLOCK_CACHE_ENTRIES 32
#endif
constexpr int kBlockEntries = STRATUM_BLOCK_CACHE_ENTRIES;
static_assert(kBlockEntries >= 1 && kBlockEntries <= 32, "one lane per block-cache entry");
struct BlockCache {
  StagedFeat feats[kBlockEntries][kEntryRecords];
  ChunkBox boxes[kBlockEntries][kRunsPerGroup];
  int key[kBlockEntries];
  int count[kBlockEntries];
  volatile int ready[kBlockEntries];
  unsigned next;
};
// Every thread of the block calls this before any lookup (followed by a
// block-wide barrier).
SD void blockCacheInit(BlockCache& bc) {
  for (int i = int(threadIdx.x); i < kBlockEntries; i += int(blockDim.x)) bc.ready[i] = 0;
  if (threadIdx.x == 0) bc.next = 0u;
}
// The ready entry holding `key`, or -1.  Warp-collective.
SD int blockCacheFind(const BlockCache& bc, int key) {
  const int lane = int(threadIdx.x & 31);
  const int ready = lane < kBlockEntries ? bc.ready[lane] : 0;
  // an entry's key and records were written before its ready flag: read them after it
  __threadfence_block();
  const bool hit = ready != 0 && reinterpret_cast<const volatile int*>(bc.key)[lane] == key;
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  return m ? __ffs(m) - 1 : -1;
}
// Copy the group just staged in slot 0 of `ws` into a free entry, if any.  Warp-collective.
SD void blockCachePut(BlockCache& bc, const WarpStage& ws, int key, int count) {
  const int lane = int(threadIdx.x & 31);
  unsigned e = 0u;
  if (lane == 0) e = atomicAdd(&bc.next, 1u);
  e = __shfl_sync(0xffffffffu, e, 0);
  if (e >= unsigned(kBlockEntries)) return;
  for (int k = lane; k < count; k += 32) bc.feats[e][k] = ws.feats[0][k];
  if (lane < (count + kRun - 1) / kRun) bc.boxes[e][lane] = ws.boxes[0][lane];
  if (lane == 0) { bc.key[e] = key; bc.count[e] = count; }
  __syncwarp();
  __threadfence_block();
  if (lane == 0) bc.ready[e] = 1;
}

// Stage one group into slot q of the warp's stage: its records from the group
// cache, or built by the grammar (and stored when the cache gives an entry),
// and the chunk boxes.  Warp-collective; returns the group's record count.
SD int stageGroup(const float* __restrict__ W, const GroupCache& cache, int key, WarpStage& ws, int q) {
  const int lane = int(threadIdx.x & 31);
  const int slot = key >> 6, g = key & 63;
  // the directory word, the lot row, the entry's tag and its records in as few
  // dependent round trips as possible: the records are loaded with the tag and
  // kept only if every tag word matches the slot's current descriptor (else a miss)
  uint32_t word = cache.base ? __ldcg(cache.dir(slot, g)) : 0u;
  const LotDesc L = loadLot(W, slot);
  const int count = groupCount(L, g);
  int e = cache.base ? usableEntry(cache, word) : -1;
  if (e >= 0) {
    bool same = true;
    if (lane < kEntryTagWords)
      same = __ldg(entryTag(cache, uint32_t(e)) + lane) == tagWord(W + size_t(slot) * kLotFloats, g, count, lane);
    StagedFeat r0{}, r1{};
    if (lane < count) r0 = cacheRecord(cache, e, lane);
    if (lane + 32 < count) r1 = cacheRecord(cache, e, lane + 32);
    const int runs = (count + kRun - 1) / kRun;
    float2 ba{}, bb{}, bc{};
    if (lane < runs) {
      const float2* bp = reinterpret_cast<const float2*>(entryBoxes(cache, uint32_t(e)) + lane * 6);
      ba = __ldg(bp); bb = __ldg(bp + 1); bc = __ldg(bp + 2);
    }
    if (__all_sync(0xffffffffu, same)) {  // records and chunk boxes as stored
      if (lane < count) ws.feats[q][lane] = r0;
      if (lane + 32 < count) ws.feats[q][lane + 32] = r1;
      if (lane < runs) ws.boxes[q][lane] = ChunkBox{{ba.x, ba.y, bb.x}, {bb.y, bc.x, bc.y}};
    } else {
      e = -1;
    }
  }
  const bool cached = e >= 0;
  if (!cached) e = cacheClaim(cache, slot, g, word);  // -1: build without storing
  if (!cached) {
#pragma unroll 1
    for (int base = 0; base < count; base += 32) {
      const int j = base + lane;
      f3 lo = mk(1e30f, 1e30f, 1e30f), hi = mk(-1e30f, -1e30f, -1e30f);
      if (j < count) {
        StagedFeat s;
        stage(s, featureAtOOL(L, g, j));
        if (e >= 0) entryRecords(cache, uint32_t(e))[j] = s;
        ws.feats[q][j] = s;
        hitBox(unstage(s), lo, hi);
      }
#pragma unroll
      for (int o = 1; o < kRun; o <<= 1) {
        lo = vmin(lo, mk(__shfl_xor_sync(0xffffffffu, lo.x, o), __shfl_xor_sync(0xffffffffu, lo.y, o),
                         __shfl_xor_sync(0xffffffffu, lo.z, o)));
        hi = vmax(hi, mk(__shfl_xor_sync(0xffffffffu, hi.x, o), __shfl_xor_sync(0xffffffffu, hi.y, o),
                         __shfl_xor_sync(0xffffffffu, hi.z, o)));
      }
      if ((lane & (kRun - 1)) == 0 && j < count) {
        const ChunkBox b = ChunkBox{{lo.x, lo.y, lo.z}, {hi.x, hi.y, hi.z}};
        ws.boxes[q][j / kRun] = b;
        if (e >= 0) {
          float* bp = entryBoxes(cache, uint32_t(e)) + (j / kRun) * 6;
          bp[0] = b.lo[0]; bp[1] = b.lo[1]; bp[2] = b.lo[2]; bp[3] = b.hi[0]; bp[4] = b.hi[1]; bp[5] = b.hi[2];
        }
      }
    }
  }
  if (!cached && e >= 0) cachePublish(cache, W, slot, g, count, e);
  return count;
}

// The whole warp traces its 32 rays.  Every lane of the warp must call this
// (inactive lanes with active = false).  `ws` is this warp's shared-memory
// staging area; `cache` is the table's group cache (null base: none).
// kBlockCache: the block's warps share the groups they build through `bc`
// (the drop-in trace); otherwise `bc` is unused.
template <bool kBlockCache = false>
SD TraceResult traceWarp(const float* __restrict__ W, const float4* __restrict__ N, uint32_t o0, uint32_t o2, f3 ro,
                         f3 rd, float cone, bool active, WarpStage& ws, const GroupCache& cache,
                         BlockCache* bc = nullptr) {
  const int lane = int(threadIdx.x & 31);
  CoopRay r;
  coopBegin(r, ro, rd, cone, active);
#pragma unroll 1
  for (;;) {
    coopAdvance(r, W, N, o0, o2);
    unsigned pending = __ballot_sync(0xffffffffu, r.state == kLeafPending);
    if (!pending) break;  // every lane is done (lanes only stop advancing at a leaf or when done)
#if STRATUM_SPEC_LEAVES > 1
    static_assert(kKeys == 1, "queued leaves are served one group at a time");
#pragma unroll 1
    while (pending) {
      const int myKey = (r.slot << 6) | r.pend;
#else
    const int myKey = (r.slot << 6) | r.pend;
#pragma unroll 1
    while (pending) {
#endif
      // up to kKeys distinct keys of the pending lanes (first pending lane's
      // key first), staged one after another
      unsigned batch = 0u;
      int myq = -1, myCount = 0;
      const StagedFeat* myFeats = nullptr;
      const ChunkBox* myBoxes = nullptr;
#pragma unroll
      for (int q = 0; q < kKeys; q++) {
        const unsigned rem = pending & ~batch;
        if (!rem) break;
        const int key = __shfl_sync(0xffffffffu, myKey, __ffs(rem) - 1);
        const unsigned peers = __ballot_sync(0xffffffffu, r.state == kLeafPending && myKey == key);
        batch |= peers;
        if constexpr (kBlockCache) {
          int count;
          const StagedFeat* feats = ws.feats[q];
          const ChunkBox* boxes = ws.boxes[q];
          const int e = blockCacheFind(*bc, key);
          if (e >= 0) {  // built earlier by a warp of this block
            count = bc->count[e];
            feats = bc->feats[e];
            boxes = bc->boxes[e];
          } else {
            count = stageGroup(W, cache, key, ws, q);
            if (q == 0) {
              __syncwarp();
              blockCachePut(*bc, ws, key, count);
            }
          }
          if ((peers >> lane) & 1u) { myq = q; myCount = count; myFeats = feats; myBoxes = boxes; }
        } else {
          const int count = stageGroup(W, cache, key, ws, q);
          if ((peers >> lane) & 1u) { myq = q; myCount = count; }
        }
      }
      __syncwarp();
      // every waiting lane tests its own group's records in index order
      if (myq >= 0) {
        const int g = r.pend;
#pragma unroll 1
        for (int c = 0; c * kRun < myCount; c++) {
          const ChunkBox b = kBlockCache ? myBoxes[c] : ws.boxes[myq][c];
          const Span cr = slabInv(r.lr, r.inv0, mk(b.lo[0], b.lo[1], b.lo[2]), mk(b.hi[0], b.hi[1], b.hi[2]));
          if (cr.hi < fmaxf(0.001f, cr.lo) || cr.lo > r.best) continue;  // no feature of the run can win
          const int kEnd = min(myCount, (c + 1) * kRun);
#pragma unroll 1
          for (int k = c * kRun; k < kEnd; k++) {
            const Feat f = unstage(kBlockCache ? myFeats[k] : ws.feats[myq][k]);
            const bool odd = f.turn % 2 == 1;
            const f3 inv = odd ? inv1Of(r) : r.inv0, p = intoFeature(r.lr - f.p, f.turn);
            const Span rg = featureSlab(f, p, inv);
            if (featureSlabMiss(f, rg)) continue;
            const f3 d = odd ? mk(r.ld.z, r.ld.y, -r.ld.x) : r.ld;
            const float th = featureAfterSlab(f, r.lr, r.ld, p, d, inv, rg, r.cone);
            if (th > 0.001f && th < r.best) {  // index order: the first feature wins ties
              r.best = th; r.fid = g * kMaxFeatures + k; r.wslot = r.slot; r.wcx = r.lcx; r.wcz = r.lcz;
            }
          }
        }
#if STRATUM_SPEC_LEAVES > 1
        // the next queued leaf that can still win (its node tested against
        // the best just found, as the reference tests it when it gets there)
        r.queue >>= 8;
        r.qn--;
#pragma unroll 1
        while (r.qn > 0 && !(nodeEntry(N, r.slot * kNodes + kGroups + int(r.queue & 255u), r.lr, r.inv0, r.best) < r.best)) {
          r.queue >>= 8;
          r.qn--;
        }
        if (r.qn > 0) r.pend = int(r.queue & 255u);
        else r.state = kInLot;  // the walk goes on from where it stopped
      }
      __syncwarp();
      pending = __ballot_sync(0xffffffffu, r.state == kLeafPending);
    }
#else
        r.state = kInLot;
        r.node = popNode(r.stack);
      }
      __syncwarp();
      pending &= ~batch;
    }
#endif
  }
  TraceResult out;
  out.t = r.best; out.fid = r.fid; out.material = 10; out.seed = 0.0f; out.slot = -1;
  out.normal = mk(0.0f, 1.0f, 0.0f);
  if (r.fid >= 0) {  // the winner's record, lot frame and normal (trace.cu:53-54)
    const LotDesc L = loadLot(W, r.wslot);
    const Feat f = winnerFeature(cache, W, r.wslot, r.fid >> 6, r.fid & 63);
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
