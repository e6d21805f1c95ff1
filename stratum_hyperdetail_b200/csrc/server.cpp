// Render server: continuous batching of render requests over resident sessions.
//
// A session is one camera in one seeded world at one resolution.  While it is
// resident its whole device state lives in one allocation: descriptor table,
// tags, the 64 MiB hierarchy, the table's group cache, refresh queue, camera
// state and frame buffers including the 64-sample accumulation buffer.  The
// group cache is not snapshotted on eviction: it refills as the session renders.  Moving or revisiting therefore
// refreshes only the lots whose address changed (prepareLots' tag compare).
//
// Admission is by an HBM budget: a session is admitted when its bytes fit;
// otherwise least recently used sessions that are idle (nothing queued in a
// launched batch) are evicted.  Eviction snapshots what the future needs (camera
// state, table origin, accumulation buffer) to pinned host memory (pinned when
// the session is opened, not while the scheduler holds its lock) and returns
// the device block to the server's arena: device memory taken in 4 GiB chunks
// (only while the budget allows) and divided among sessions by a host-side
// first-fit allocator, so admitting and evicting never call the driver's
// allocator on the request path; re-admission clears only what must start at zero (camera,
// input, table, tags; History when there is no snapshot), restores the
// snapshot and rebuilds the table and hierarchy from the seed, so the session
// continues exactly as if it had never left (the world is a pure function of
// seed and address).  Eviction and admission are ordered on one admission
// stream that batches wait for with an event: the scheduler thread never waits
// on the device for them.
//
// The scheduler thread keeps `streams` batch slots.  Whenever a slot is free it
// takes the oldest pending request of every idle session (up to `max_views`),
// admits sessions as memory allows, and launches one sample of every request in
// the batch -- applyPoses, stepViews, refreshViews, buildViews, renderViews and
// the RGBA8 read-back -- on that slot's stream.  Requests arriving while
// batches run join the next free slot, so their work overlaps on the device.
// A request of k samples rides in k consecutive batches.
//
// A batch whose launch fails after part of its work was queued keeps its slot
// (and its sessions) busy until that work has drained from the slot's stream;
// only then are its requests failed and its sessions released, so no pinned
// staging buffer is rewritten and no session memory is freed under queued
// work.  Sessions of a failed batch restart their sampling on their next
// request (their camera state may have been stepped).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/stratum.h"

namespace {

using Clock = std::chrono::steady_clock;
double nowMs() { return std::chrono::duration<double, std::milli>(Clock::now().time_since_epoch()).count(); }

constexpr int kLots = 16384, kNodes = 128;
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of one session's buffers inside its single allocation.
struct Layout {
  size_t C, Origin, I, World, Tags, Nodes, Queue, Hit, Surface, Linear, History, Pixels, Groups, total;
  int groupEntries;
  static Layout of(int w, int h, int groupEntries) {
    Layout L{};
    size_t o = 0, P = size_t(w) * size_t(h);
    auto take = [&](size_t bytes) { size_t at = o; o += align256(bytes); return at; };
    L.C = take(64 * 4); L.Origin = take(16); L.I = take(32 * 4);
    L.World = take(size_t(kLots) * 64); L.Tags = take(size_t(kLots) * 16); L.Nodes = take(size_t(kLots) * kNodes * 32);
    L.Queue = take(size_t(kLots + 1) * 4);
    L.Hit = take(P * 16); L.Surface = take(P * 16); L.Linear = take(P * 16); L.History = take(P * 16);
    L.Pixels = take(P * 4);
    L.groupEntries = groupEntries;
    L.Groups = groupEntries > 0 ? take(stratum_groupCacheBytes(groupEntries)) : 0;
    L.total = o;
    return L;
  }
};

struct Request {
  long long id;
  int session;
  stratum_pose pose;
  int samples, done = 0;
  unsigned char* out;
  double tSubmit, tStart = -1.0, tDone = -1.0;
  int status = STRATUM_QUEUE_STALLED;
  bool poseApplied = false;
};

struct Session {
  int id, seed, width, height;
  Layout lay;
  char* base = nullptr;
  bool resident = false, inflight = false, started = false, restart = false;
  bool admitQueued = false;  // admission work on the admission stream not yet waited for by a batch
  std::deque<Request*> queue;
  stratum_pose last{};
  double lastUse = 0.0;
  bool hasSnap = false;
  // pinned snapshot while evicted (kept for the next eviction): History (P x 16 B),
  // then C (256 B) and Origin (16 B)
  char* snap = nullptr;
  unsigned char* pinnedOut = nullptr;
  template <class T> T* at(size_t off) const { return reinterpret_cast<T*>(base + off); }
  stratum_view view() const {
    stratum_view v{};
    v.C = at<float>(lay.C); v.Origin = at<unsigned>(lay.Origin); v.I = at<float>(lay.I);
    v.World = at<float>(lay.World); v.Tags = at<unsigned>(lay.Tags); v.Nodes = at<float>(lay.Nodes);
    v.Queue = at<unsigned>(lay.Queue); v.Hit = at<float>(lay.Hit); v.Surface = at<float>(lay.Surface);
    v.Linear = at<float>(lay.Linear); v.History = at<float>(lay.History); v.Pixels = at<unsigned>(lay.Pixels);
    v.Groups = lay.groupEntries > 0 ? at<unsigned>(lay.Groups) : nullptr;
    v.width = width; v.height = height; v.dt = 0.0f;
    return v;
  }
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* scratch = nullptr;
  unsigned long long scratchBytes = 0;
  stratum_view* dViews = nullptr;
  stratum_pose* dPoses = nullptr;
  int* dFlags = nullptr;
  stratum_view* hViews = nullptr;  // pinned staging
  stratum_pose* hPoses = nullptr;
  int* hFlags = nullptr;
  std::vector<Request*> reqs;
  bool busy = false;
  int failStatus = STRATUM_OK;  // a batch that failed after enqueueing: its requests fail on completion
};

bool samePose(const stratum_pose& a, const stratum_pose& b) { return std::memcmp(&a, &b, sizeof a) == 0; }

// Session device memory: chunks of device memory taken with cudaMalloc while
// the budget allows, each divided by first fit over a free list of (offset,
// size) ranges that merges neighbours on release.  Blocks are multiples of
// 2 MiB.  Only the scheduler thread (under the server lock) touches it.
struct Arena {
  struct Chunk {
    char* base;
    size_t size;
    std::map<size_t, size_t> free;  // offset -> size, disjoint, not adjacent
  };
  static constexpr size_t kGrain = size_t(2) << 20;
  static constexpr size_t kChunk = size_t(4) << 30;
  std::vector<Chunk> chunks;
  size_t reserved = 0;  // bytes held in chunks

  static size_t round(size_t n) { return (n + kGrain - 1) / kGrain * kGrain; }
  char* take(size_t need) {
    for (Chunk& c : chunks)
      for (auto it = c.free.begin(); it != c.free.end(); ++it)
        if (it->second >= need) {
          const size_t off = it->first, rest = it->second - need;
          c.free.erase(it);
          if (rest) c.free[off + need] = rest;
          return c.base + off;
        }
    return nullptr;
  }
  // A new chunk of kChunk bytes, or what is left of `limit` if that is less,
  // but never less than `need`.
  int grow(size_t need, size_t limit) {
    if (reserved + need > limit) return STRATUM_QUEUE_STALLED;
    const size_t size = std::max(need, std::min(kChunk, (limit - reserved) / kGrain * kGrain));
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, size);
    if (e != cudaSuccess) { cudaGetLastError(); return -int(e); }
    Chunk c{static_cast<char*>(p), size, {}};
    c.free[0] = size;
    chunks.push_back(std::move(c));
    reserved += size;
    return STRATUM_OK;
  }
  void give(char* p, size_t size) {
    for (Chunk& c : chunks) {
      if (p < c.base || p >= c.base + c.size) continue;
      size_t off = size_t(p - c.base);
      auto next = c.free.lower_bound(off);
      if (next != c.free.end() && off + size == next->first) { size += next->second; next = c.free.erase(next); }
      if (next != c.free.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) { prev->second += size; return; }
      }
      c.free[off] = size;
      return;
    }
  }
  void release() {
    for (Chunk& c : chunks) cudaFree(c.base);
    chunks.clear();
    reserved = 0;
  }
};

}  // namespace

struct stratum_server {
  int device = 0;
  unsigned long long budget = 0;
  int maxViews = 1;
  int groupEntries = 16384;
  stratum_tune tune{64, 1, 1};
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  std::atomic<bool> stop{false};
  cudaStream_t admitStream = nullptr;
  cudaEvent_t admitDone = nullptr;  // recorded after each admission's device work
  Arena arena;                      // session device memory, at most `budget` bytes
  std::unordered_map<int, std::unique_ptr<Session>> sessions;
  int nextSession = 1;
  std::unordered_map<long long, std::unique_ptr<Request>> requests;
  long long nextRequest = 1;
  std::vector<Slot> slots;
  unsigned long long residentBytes = 0;
  long long submitted = 0, completed = 0, failed = 0, batches = 0, admissions = 0, evictions = 0;
  std::vector<double> latencies;
  double rays = 0.0, firstSubmit = -1.0, lastDone = -1.0;
  int injectAllocFail = 0;
  int injectLaunchFail = 0;  // fail launches after refreshViews (work already queued)
};

namespace {

void finish(stratum_server* S, Request* r, int status) {
  r->status = status;
  r->tDone = nowMs();
  if (status == STRATUM_OK) {
    S->completed++;
    S->latencies.push_back(r->tDone - r->tSubmit);
    S->lastDone = r->tDone;
  } else {
    S->failed++;
  }
}

// Snapshot what a session needs to continue, then free its device memory.  All
// of it is ordered on the admission stream (copies, then the free; a later
// re-admission's restore follows on the same stream), so nothing waits here.
// Only idle sessions are evicted: their last batch has completed.
int evict(stratum_server* S, Session& s) {
  size_t P = size_t(s.width) * size_t(s.height);
  if (!s.snap) return STRATUM_EINVAL;  // pinned at open
  cudaError_t e = cudaMemcpyAsync(s.snap + P * 16, s.at<float>(s.lay.C), 64 * 4, cudaMemcpyDeviceToHost, S->admitStream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.snap + P * 16 + 256, s.at<unsigned>(s.lay.Origin), 16, cudaMemcpyDeviceToHost, S->admitStream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.snap, s.at<float>(s.lay.History), P * 16, cudaMemcpyDeviceToHost, S->admitStream);
  if (e != cudaSuccess) return -int(e);
  // the block is reused by admissions queued after these copies on the same stream
  S->arena.give(s.base, Arena::round(s.lay.total));
  s.base = nullptr;
  s.resident = false;
  s.hasSnap = true;
  S->residentBytes -= Arena::round(s.lay.total);
  S->evictions++;
  return STRATUM_OK;
}

bool contains(const std::vector<Session*>& v, const Session* s) { return std::find(v.begin(), v.end(), s) != v.end(); }

// Make `s` resident.  STRATUM_QUEUE_STALLED: no room yet (retry later).
int admit(stratum_server* S, Session& s, const std::vector<Session*>& batch) {
  const size_t need = Arena::round(s.lay.total);
  if (need > S->budget) return STRATUM_BUDGET_EXCEEDED;
  if (S->injectAllocFail > 0) {
    S->injectAllocFail--;
    return -int(cudaErrorMemoryAllocation);
  }
  // A free block that fits; else a new chunk while the budget allows; else
  // evict idle sessions, least recently used first, until a block fits.
  char* p = nullptr;
  while (!(p = S->arena.take(need))) {
    int st = S->arena.grow(need, S->budget);
    if (st == STRATUM_OK) continue;
    if (st != STRATUM_QUEUE_STALLED && S->arena.reserved == 0) return st;
    Session* victim = nullptr;
    for (auto& kv : S->sessions) {
      Session* q = kv.second.get();
      if (q->resident && !q->inflight && !contains(batch, q) && (!victim || q->lastUse < victim->lastUse)) victim = q;
    }
    if (!victim) return STRATUM_QUEUE_STALLED;
    st = evict(S, *victim);
    if (st != STRATUM_OK) return st;
  }
  cudaError_t e = cudaSuccess;
  s.base = p;
  // Only what is read before it is written starts at zero: camera, origin and
  // input, the table and its tags (every lot is then described and its
  // hierarchy built), and History unless a snapshot restores it.  Nodes, the
  // frame buffers and the group cache's entries are written before any read.
  e = cudaMemsetAsync(s.base, 0, s.lay.Nodes, S->admitStream);
  if (e == cudaSuccess && !s.hasSnap)
    e = cudaMemsetAsync(s.base + s.lay.History, 0, size_t(s.width) * s.height * 16, S->admitStream);
  int st = e == cudaSuccess ? STRATUM_OK : -int(e);
  if (st == STRATUM_OK)
    st = stratum_initCamera(s.at<float>(s.lay.C), s.at<unsigned>(s.lay.Origin), s.seed,
                            reinterpret_cast<stratum_stream_t>(S->admitStream));
  if (st == STRATUM_OK && s.lay.groupEntries > 0)
    st = stratum_groupCacheInit(s.at<unsigned>(s.lay.Groups), s.lay.groupEntries,
                                reinterpret_cast<stratum_stream_t>(S->admitStream));
  if (st == STRATUM_OK && s.hasSnap) {  // continue exactly where the session left
    size_t P = size_t(s.width) * size_t(s.height);
    e = cudaMemcpyAsync(s.at<float>(s.lay.C), s.snap + P * 16, 64 * 4, cudaMemcpyHostToDevice, S->admitStream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.at<unsigned>(s.lay.Origin), s.snap + P * 16 + 256, 16, cudaMemcpyHostToDevice, S->admitStream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.at<float>(s.lay.History), s.snap, P * 16, cudaMemcpyHostToDevice, S->admitStream);
    if (e != cudaSuccess) st = -int(e);
  }
  if (st == STRATUM_OK) {  // batches wait for this event on their own streams; the host does not
    e = cudaEventRecord(S->admitDone, S->admitStream);
    if (e != cudaSuccess) st = -int(e);
  }
  if (st != STRATUM_OK) {
    S->arena.give(s.base, need);
    s.base = nullptr;
    return st;
  }
  s.resident = true;
  s.hasSnap = false;
  s.admitQueued = true;
  S->residentBytes += need;
  S->admissions++;
  return STRATUM_OK;
}

int enqueue(stratum_server* S, Slot& sl, const std::vector<Request*>& reqs, int n);
void deferFailure(Slot& sl, const std::vector<Request*>& reqs, int status);

int launch(stratum_server* S, Slot& sl, const std::vector<Request*>& reqs) {
  const int n = int(reqs.size());
  const double t = nowMs();
  for (int i = 0; i < n; i++) {
    Request* r = reqs[i];
    Session& s = *S->sessions[r->session];
    sl.hViews[i] = s.view();
    sl.hPoses[i] = r->pose;
    int flags = 0;
    if (!r->poseApplied) {  // first sample of this request: place the camera
      flags |= 1;
      if (!s.started || s.restart || !samePose(s.last, r->pose)) flags |= 2;
      s.restart = false;
      s.last = r->pose;
      s.started = true;
      r->poseApplied = true;
    }
    sl.hFlags[i] = flags;
    if (r->tStart < 0) r->tStart = t;
  }
  cudaStream_t st = sl.stream;
  // sessions admitted for this batch: their initialisation and restored
  // snapshot are ordered on the admission stream, which this batch then waits
  // for; a batch of sessions that were resident already does not wait on it
  bool admitted = false;
  for (Request* r : reqs) admitted |= S->sessions[r->session]->admitQueued;
  cudaError_t e = admitted ? cudaStreamWaitEvent(st, S->admitDone, 0) : cudaSuccess;
  if (e != cudaSuccess) return -int(e);  // nothing queued yet
  for (Request* r : reqs) S->sessions[r->session]->admitQueued = false;
  int s = enqueue(S, sl, reqs, n);
  if (s != STRATUM_OK) {
    deferFailure(sl, reqs, s);
    return STRATUM_OK;  // the requests fail when the queued work has drained
  }
  e = cudaEventRecord(sl.done, st);
  if (e != cudaSuccess) {
    deferFailure(sl, reqs, -int(e));
    return STRATUM_OK;
  }
  sl.reqs = reqs;
  sl.busy = true;
  S->batches++;
  return STRATUM_OK;
}

// The device work of one batch on its slot's stream.
int enqueue(stratum_server* S, Slot& sl, const std::vector<Request*>& reqs, int n) {
  cudaStream_t st = sl.stream;
  stratum_stream_t ss = reinterpret_cast<stratum_stream_t>(st);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMemcpyAsync(sl.dViews, sl.hViews, sizeof(stratum_view) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sl.dPoses, sl.hPoses, sizeof(stratum_pose) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sl.dFlags, sl.hFlags, sizeof(int) * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return -int(e);
  int s;
  if ((s = stratum_applyPoses(sl.dViews, sl.dPoses, sl.dFlags, n, ss)) != STRATUM_OK) return s;
  if ((s = stratum_stepViews(sl.dViews, n, ss)) != STRATUM_OK) return s;
  if ((s = stratum_refreshViews(sl.dViews, n, ss)) != STRATUM_OK) return s;
  if (S->injectLaunchFail > 0) {  // host-side fault injection: work is already queued on the stream
    S->injectLaunchFail--;
    return -int(cudaErrorLaunchFailure);
  }
  if ((s = stratum_buildViews(sl.dViews, n, ss)) != STRATUM_OK) return s;
  if ((s = stratum_renderViews(sl.dViews, n, sl.scratch, sl.scratchBytes, &S->tune, ss)) != STRATUM_OK) return s;
  for (int i = 0; i < n; i++) {
    Request* r = reqs[i];
    if (r->done + 1 < r->samples) continue;  // not its last sample: no read-back yet
    Session& ses = *S->sessions[r->session];
    e = cudaMemcpyAsync(ses.pinnedOut, ses.at<unsigned>(ses.lay.Pixels), size_t(ses.width) * ses.height * 4,
                        cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return -int(e);
  }
  return STRATUM_OK;
}

// A batch that failed after part of it was queued: hold the slot until that
// work drains (an event on the slot's stream, or a synchronize if even the
// record fails), then fail its requests in complete().
void deferFailure(Slot& sl, const std::vector<Request*>& reqs, int status) {
  sl.reqs = reqs;
  sl.failStatus = status;
  sl.busy = true;
  if (cudaEventRecord(sl.done, sl.stream) != cudaSuccess) {
    cudaStreamSynchronize(sl.stream);
    cudaEventRecord(sl.done, sl.stream);
  }
}

void complete(stratum_server* S, Slot& sl) {
  if (sl.failStatus != STRATUM_OK) {
    for (Request* r : sl.reqs) {
      Session& s = *S->sessions[r->session];
      s.inflight = false;
      s.restart = true;
      s.lastUse = nowMs();
      s.queue.pop_front();
      finish(S, r, sl.failStatus);
    }
    sl.reqs.clear();
    sl.failStatus = STRATUM_OK;
    sl.busy = false;
    return;
  }
  for (Request* r : sl.reqs) {
    Session& s = *S->sessions[r->session];
    s.inflight = false;
    s.lastUse = nowMs();
    r->done++;
    S->rays += double(s.width) * double(s.height);
    if (r->done >= r->samples) {
      if (r->out) std::memcpy(r->out, s.pinnedOut, size_t(s.width) * s.height * 4);
      s.queue.pop_front();
      finish(S, r, STRATUM_OK);
    }
  }
  sl.reqs.clear();
  sl.busy = false;
}

void failQueue(stratum_server* S, Session& s, int status) {
  while (!s.queue.empty()) {
    finish(S, s.queue.front(), status);
    s.queue.pop_front();
  }
}

void schedule(stratum_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (!S->stop.load()) {
    bool progress = false;
    for (Slot& sl : S->slots)
      if (sl.busy && cudaEventQuery(sl.done) == cudaSuccess) {
        complete(S, sl);
        progress = true;
      }
    for (Slot& sl : S->slots) {
      if (sl.busy) continue;
      std::vector<Session*> cand;
      for (auto& kv : S->sessions)
        if (!kv.second->queue.empty() && !kv.second->inflight) cand.push_back(kv.second.get());
      if (cand.empty()) break;
      std::sort(cand.begin(), cand.end(),
                [](Session* a, Session* b) { return a->queue.front()->tSubmit < b->queue.front()->tSubmit; });
      std::vector<Request*> reqs;
      std::vector<Session*> chosen;
      for (Session* s : cand) {
        if (int(reqs.size()) >= S->maxViews) break;
        if (!s->resident) {
          int st = admit(S, *s, chosen);
          if (st == STRATUM_QUEUE_STALLED) continue;  // no room until a batch finishes
          if (st != STRATUM_OK) { failQueue(S, *s, st); progress = true; continue; }
        }
        s->inflight = true;
        chosen.push_back(s);
        reqs.push_back(s->queue.front());
      }
      if (reqs.empty()) break;
      int st = launch(S, sl, reqs);
      if (st != STRATUM_OK) {  // nothing was queued: fail its requests now; the server keeps serving
        for (Request* r : reqs) {
          Session& s = *S->sessions[r->session];
          s.inflight = false;
          s.restart = true;
          s.queue.pop_front();
          finish(S, r, st);
        }
      }
      progress = true;
    }
    if (progress) S->cv.notify_all();
    else S->cv.wait_for(lk, std::chrono::microseconds(100));
  }
}

void freeSession(stratum_server* S, Session& s) {
  if (s.resident) {  // an idle session: nothing of it is queued on a batch stream
    S->arena.give(s.base, Arena::round(s.lay.total));
    S->residentBytes -= Arena::round(s.lay.total);
    s.resident = false;
  }
  if (s.pinnedOut) cudaFreeHost(s.pinnedOut);
  s.pinnedOut = nullptr;
  if (s.snap) cudaFreeHost(s.snap);
  s.snap = nullptr;
}

}  // namespace

extern "C" {

stratum_server* stratum_server_create(unsigned long long budget_bytes, int max_views, int streams,
                                      const stratum_tune* tune) {
  if (max_views <= 0 || streams <= 0 || streams > 8) return nullptr;
  auto S = std::make_unique<stratum_server>();
  cudaGetDevice(&S->device);
  S->budget = budget_bytes;
  S->maxViews = max_views;
  if (tune) S->tune = *tune;
  if (cudaStreamCreateWithFlags(&S->admitStream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&S->admitDone, cudaEventDisableTiming) != cudaSuccess) {
    stratum_server_destroy(S.release());
    return nullptr;
  }
  S->slots.resize(streams);
  for (Slot& sl : S->slots) {
    sl.scratchBytes = stratum_batchScratchBytes(max_views);
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&sl.scratch, sl.scratchBytes) != cudaSuccess ||
        cudaMemset(sl.scratch, 0, sl.scratchBytes) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&sl.dViews), sizeof(stratum_view) * max_views) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&sl.dPoses), sizeof(stratum_pose) * max_views) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&sl.dFlags), sizeof(int) * max_views) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.hViews), sizeof(stratum_view) * max_views) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.hPoses), sizeof(stratum_pose) * max_views) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.hFlags), sizeof(int) * max_views) != cudaSuccess) {
      stratum_server_destroy(S.release());
      return nullptr;
    }
  }
  stratum_server* raw = S.release();
  raw->worker = std::thread(schedule, raw);
  return raw;
}

int stratum_server_set_group_cache(stratum_server* S, int entries) {
  if (!S || entries < 0) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  if (!S->sessions.empty()) return STRATUM_EINVAL;
  S->groupEntries = entries;
  return STRATUM_OK;
}

void stratum_server_destroy(stratum_server* S) {
  if (!S) return;
  S->stop.store(true);
  S->cv.notify_all();
  if (S->worker.joinable()) S->worker.join();
  for (Slot& sl : S->slots) {
    if (sl.busy && sl.done) cudaEventSynchronize(sl.done);
    if (sl.stream) cudaStreamSynchronize(sl.stream);
  }
  for (auto& kv : S->sessions) freeSession(S, *kv.second);
  if (S->admitStream) cudaStreamSynchronize(S->admitStream);
  S->arena.release();
  for (Slot& sl : S->slots) {
    cudaFree(sl.scratch); cudaFree(sl.dViews); cudaFree(sl.dPoses); cudaFree(sl.dFlags);
    cudaFreeHost(sl.hViews); cudaFreeHost(sl.hPoses); cudaFreeHost(sl.hFlags);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  if (S->admitDone) cudaEventDestroy(S->admitDone);
  if (S->admitStream) cudaStreamDestroy(S->admitStream);
  delete S;
}

int stratum_server_open(stratum_server* S, int seed, int width, int height, int* session) {
  if (!S || !session || width <= 0 || height <= 0 || width > STRATUM_MAX_DIM || height > STRATUM_MAX_DIM)
    return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto s = std::make_unique<Session>();
  s->id = S->nextSession++;
  s->seed = seed;
  s->width = width;
  s->height = height;
  s->lay = Layout::of(width, height, S->groupEntries);
  // Host staging is pinned here, not on the scheduler thread: the RGBA8
  // read-back buffer and the eviction snapshot (History, camera, origin).
  const size_t P = size_t(width) * size_t(height);
  if (cudaMallocHost(reinterpret_cast<void**>(&s->pinnedOut), P * 4) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&s->snap), P * 16 + 512) != cudaSuccess) {
    cudaError_t e = cudaGetLastError();
    freeSession(S, *s);
    return -int(e != cudaSuccess ? e : cudaErrorMemoryAllocation);
  }
  *session = s->id;
  S->sessions[s->id] = std::move(s);
  return STRATUM_OK;
}

int stratum_server_close(stratum_server* S, int session) {
  if (!S) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->sessions.find(session);
  if (it == S->sessions.end()) return STRATUM_NOT_FOUND;
  Session& s = *it->second;
  if (s.inflight || !s.queue.empty()) return STRATUM_QUEUE_STALLED;  // busy: close after its requests finish
  freeSession(S, s);
  S->sessions.erase(it);
  return STRATUM_OK;
}

int stratum_server_submit(stratum_server* S, int session, const stratum_pose* pose, int samples, unsigned char* out,
                          long long* request) {
  if (!S || !pose || !request || samples < 1 || samples > 64) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->sessions.find(session);
  if (it == S->sessions.end()) return STRATUM_NOT_FOUND;
  auto r = std::make_unique<Request>();
  r->id = S->nextRequest++;
  r->session = session;
  r->pose = *pose;
  r->samples = samples;
  r->out = out;
  r->tSubmit = nowMs();
  if (S->firstSubmit < 0) S->firstSubmit = r->tSubmit;
  it->second->queue.push_back(r.get());
  *request = r->id;
  S->requests[r->id] = std::move(r);
  S->submitted++;
  S->cv.notify_all();
  return STRATUM_OK;
}

int stratum_server_wait(stratum_server* S, long long request, int timeout_ms, stratum_request_info* info) {
  if (!S) return STRATUM_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->requests.find(request);
  if (it == S->requests.end()) return STRATUM_NOT_FOUND;
  Request* r = it->second.get();
  S->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                 [&] { return r->status != STRATUM_QUEUE_STALLED; });
  int status = r->status;
  if (info) {
    info->status = status;
    info->samples_done = r->done;
    info->latency_ms = r->tDone >= 0 ? r->tDone - r->tSubmit : -1.0;
    info->queue_ms = r->tStart >= 0 ? r->tStart - r->tSubmit : -1.0;
  }
  if (status != STRATUM_QUEUE_STALLED) S->requests.erase(it);
  return status;
}

int stratum_server_stats_get(stratum_server* S, stratum_server_stats* out) {
  if (!S || !out) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  stratum_server_stats st{};
  st.submitted = S->submitted; st.completed = S->completed; st.failed = S->failed; st.batches = S->batches;
  st.admissions = S->admissions; st.evictions = S->evictions;
  for (auto& kv : S->sessions) st.resident_sessions += kv.second->resident ? 1 : 0;
  st.resident_bytes = S->residentBytes;
  st.budget_bytes = S->budget;
  std::vector<double> l = S->latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double p) { return l[std::min(l.size() - 1, size_t(p * double(l.size() - 1) + 0.5))]; };
    st.p50_ms = q(0.5); st.p99_ms = q(0.99); st.max_ms = l.back();
    double sum = 0;
    for (double x : l) sum += x;
    st.mean_ms = sum / double(l.size());
  }
  st.rays = S->rays;
  st.first_submit_s = S->firstSubmit / 1000.0;
  st.last_done_s = S->lastDone / 1000.0;
  *out = st;
  return STRATUM_OK;
}

int stratum_server_inject(stratum_server* S, int kind, int count) {
  if (!S || (kind != 1 && kind != 2) || count < 0) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  if (kind == 1) S->injectAllocFail = count;
  else S->injectLaunchFail = count;
  return STRATUM_OK;
}

int stratum_server_read(stratum_server* S, int session, unsigned char* rgba, float* history) {
  if (!S) return STRATUM_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->sessions.find(session);
  if (it == S->sessions.end()) return STRATUM_NOT_FOUND;
  Session& s = *it->second;
  if (!s.resident || s.inflight) return STRATUM_QUEUE_STALLED;
  size_t P = size_t(s.width) * size_t(s.height);
  cudaError_t e = cudaSuccess;
  if (rgba) e = cudaMemcpyAsync(rgba, s.at<unsigned>(s.lay.Pixels), P * 4, cudaMemcpyDeviceToHost, S->admitStream);
  if (e == cudaSuccess && history)
    e = cudaMemcpyAsync(history, s.at<float>(s.lay.History), P * 16, cudaMemcpyDeviceToHost, S->admitStream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->admitStream);
  return e == cudaSuccess ? STRATUM_OK : -int(e);
}

}  // extern "C"
