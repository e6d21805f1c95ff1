// Group cache: a per-table, lazily filled store of the feature records of the
// (lot, group) pairs that rays evaluate, so that a group's records are built by
// the grammar once and then loaded, instead of rebuilt every time a warp needs
// them.  A frame evaluates each distinct group hundreds of times (one 1600x900
// frame: 10^5-10^6 group evaluations over 10^3-10^5 distinct groups).
//
// Layout of one cache buffer (stratum_groupCacheBytes):
//   header   256 B   next free entry, capacity (entries), resets, fills,
//                    trace launches
//   dir      16,384 x 64 u32: per (slot, group) 0 = empty, kCacheBusy = being
//            filled, else (launch epoch << 24) | (entry index + 1)
//   entries  capacity x 2,192 B: a 64-byte tag (the lot descriptor words the
//            grammar reads, the group, the count), 56 records of 32 bytes and
//            the 14 chunk boxes of runs of 4 records (24 bytes each)
//
// An entry serves a (slot, group) only while its tag equals the slot's current
// descriptor words and the group, so a table refreshed by any path (batched or
// the drop-in prepareLots) never reads a stale entry: a mismatch is a miss.
// Each trace launch has an epoch (its launch count, 8 bits).  A launch reads
// only entries filled by earlier launches: the kernel boundary makes them
// visible, so plain (even read-only-path) loads are correct and no acquire is
// needed.  Entries filled in the current launch are misses for that launch.  A
// warp that misses claims the group (one atomic compare-and-swap on its
// directory word) and fills an entry, or, when another warp holds it or the
// store is full, builds the records with the grammar itself: nothing waits.
// A full store keeps serving the groups it holds; at the start of a launch at
// least kCacheResetInterval launches after its last reset, a full store is
// emptied (directory cleared) and filling starts again, so tables that change
// or need more groups than fit are re-cached from time to time.
#pragma once
#include "grammar_ra.cuh"

namespace st {

struct alignas(16) StagedFeat {
  float px, py, pz, hx;
  float hy, hz;
  int packed;  // shape + 1 | material << 8 | turn << 16
  float seed;
};
SD void stage(StagedFeat& s, const Feat& f) {
  s.px = f.p.x; s.py = f.p.y; s.pz = f.p.z; s.hx = f.h.x; s.hy = f.h.y; s.hz = f.h.z;
  s.packed = (f.shape + 1) | (f.material << 8) | (f.turn << 16);
  s.seed = f.seed;
}
SD Feat unstage(const StagedFeat& s) {
  return Feat{mk(s.px, s.py, s.pz), mk(s.hx, s.hy, s.hz), (s.packed & 255) - 1, (s.packed >> 8) & 255,
              (s.packed >> 16) & 255, s.seed};
}

struct GroupCacheHeader {
  uint32_t next, capacity, resets, fills, launches, resetAt;  // resetAt: launch count of the last reset
  uint32_t pad[58];
};
static_assert(sizeof(GroupCacheHeader) == 256, "group cache header is 256 bytes");
constexpr uint32_t kCacheBusy = 0xFFFFFFFFu;
constexpr uint32_t kCacheResetInterval = 8;  // launches between resets of a full store
constexpr uint32_t kCacheMaxEntries = (1u << 24) - 2u;  // entry index + 1 fits 24 bits and is never 0xFFFFFF
constexpr int kCacheDirWords = kLots * kGroups;
constexpr int kEntryRecords = 56;  // the largest group (group 30 of a building lot)
constexpr int kEntryTagWords = 16;  // 64 bytes, 11 used
constexpr int kEntryBoxes = 14;     // chunk boxes of runs of 4 records, as the trace stages them
constexpr size_t kEntryBoxOffset = size_t(kEntryTagWords) * 4 + size_t(kEntryRecords) * sizeof(StagedFeat);
constexpr size_t kEntryBytes = kEntryBoxOffset + size_t(kEntryBoxes) * 24;
constexpr size_t kCacheDirOffset = sizeof(GroupCacheHeader);
constexpr size_t kCacheEntryOffset = kCacheDirOffset + size_t(kCacheDirWords) * 4;
static_assert(kEntryBytes % 16 == 0 && kCacheEntryOffset % 16 == 0, "entries are 16-byte aligned");

inline size_t groupCacheBytes(int entries) { return kCacheEntryOffset + size_t(entries > 0 ? entries : 0) * kEntryBytes; }

// A cache is its base address alone (kept in two registers through the
// traversal); capacity and epoch are read from the header when needed.  Those
// two header words do not change during a trace launch (the prologue before it
// writes them), so the read-only path may cache them.
struct GroupCache {
  uint32_t* base;  // null: no cache
  SD GroupCacheHeader* hdr() const { return reinterpret_cast<GroupCacheHeader*>(base); }
  SD uint32_t capacity() const { return base ? __ldg(base + 1) : 0u; }
  SD uint32_t epoch() const { return __ldg(base + 4) & 255u; }
  SD uint32_t* dir(int slot, int group) const {
    return reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(base) + kCacheDirOffset) + slot * kGroups + group;
  }
  SD char* entry(uint32_t e) const { return reinterpret_cast<char*>(base) + kCacheEntryOffset + size_t(e) * kEntryBytes; }
};
SD GroupCache groupCache(uint32_t* base) { return GroupCache{base}; }
SD uint32_t* entryTag(const GroupCache& c, uint32_t e) { return reinterpret_cast<uint32_t*>(c.entry(e)); }
SD StagedFeat* entryRecords(const GroupCache& c, uint32_t e) {
  return reinterpret_cast<StagedFeat*>(c.entry(e) + kEntryTagWords * 4);
}
SD float* entryBoxes(const GroupCache& c, uint32_t e) { return reinterpret_cast<float*>(c.entry(e) + kEntryBoxOffset); }

// The entry a directory word names if it was filled by an earlier launch, else -1.
SD int usableEntry(const GroupCache& c, uint32_t d) {
  if (d == 0u || d == kCacheBusy || (d >> 24) == c.epoch()) return -1;
  const uint32_t e = (d & 0xFFFFFFu) - 1u;
  return e < c.capacity() ? int(e) : -1;
}

// Tag word k of (descriptor row, group, count): the nine descriptor words the
// grammar reads (w, d, h, type, material, floors, seed, storey, roofScale),
// then the group and the record count.
SD uint32_t tagWord(const float* row, int group, int count, int k) {
  if (k < 9) return __float_as_uint(__ldg(row + k));
  if (k == 9) return uint32_t(group);
  if (k == 10) return uint32_t(count);
  return 0u;
}

// Warp-collective: claim a fresh entry for (slot, group), or -1 when another
// warp is filling it, filled it in this launch, or the store is full.  `old`
// is the directory word the caller read.  A claimed entry must be published.
SD int cacheClaim(const GroupCache& c, int slot, int group, uint32_t old) {
  if (c.capacity() == 0u || old == kCacheBusy || (old != 0u && (old >> 24) == c.epoch())) return -1;
  int e = -1;
  if ((threadIdx.x & 31) == 0) {
    uint32_t* dp = c.dir(slot, group);
    if (__ldcg(&c.hdr()->next) < c.capacity() && atomicCAS(dp, old, kCacheBusy) == old) {
      const uint32_t i = atomicAdd(&c.hdr()->next, 1u);
      if (i < c.capacity()) e = int(i);
      else atomicExch(dp, old);  // full: leave the word as it was
    }
  }
  return __shfl_sync(0xffffffffu, e, 0);
}

// Warp-collective: publish a claimed entry whose records the lanes have
// written.  Readers use it from the next launch on.
SD void cachePublish(const GroupCache& c, const float* W, int slot, int group, int count, int e) {
  const int lane = int(threadIdx.x & 31);
  if (lane < kEntryTagWords) entryTag(c, uint32_t(e))[lane] = tagWord(W + size_t(slot) * kLotFloats, group, count, lane);
  __syncwarp();
  if (lane == 0) {
    atomicExch(c.dir(slot, group), (c.epoch() << 24) | (uint32_t(e) + 1u));
    atomicAdd(&c.hdr()->fills, 1u);
  }
}

// Record i of a usable entry (filled by an earlier launch: read-only here).
SD StagedFeat cacheRecord(const GroupCache& c, int e, int i) {
  const float4* p = reinterpret_cast<const float4*>(entryRecords(c, uint32_t(e)) + i);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  StagedFeat s;
  s.px = a.x; s.py = a.y; s.pz = a.z; s.hx = a.w;
  s.hy = b.x; s.hz = b.y; s.packed = __float_as_int(b.z); s.seed = b.w;
  return s;
}

}  // namespace st
