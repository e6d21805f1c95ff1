/* stratum.h -- C ABI of the B200 STRATUM frame path.
 *
 * Drop-in for the reference's frame path (stratum-hyperdetail, kernels/*.cu,
 * driven by src/engine.js).  Each reference __global__ entry point becomes one
 * function taking exactly the reference's device buffers and scalars, plus a
 * CUDA stream.  Buffers are owned by the caller and live in device memory;
 * layouts are the reference's (src/engine.js:41-42,58):
 *
 *   World    16,384 x 16 f32   per slot [w,d,h,type,mat,floors,seed,storey,roofScale,
 *                               turn,ox,oz,palette,-,-,valid]  (kernels/world.cu:100-102)
 *   Tags     16,384 x 4 u32    64-bit lot address per slot (xl,xh,zl,zh)
 *   Nodes    16,384 x 128 x 8 f32 = 64 MiB   node = [lo.xyz, count, hi.xyz, group]
 *   Origin   4 u32              64-bit table origin (xl,xh,zl,zh)
 *   C        64 f32             camera/view state (field map in kernels/world.cu:57-91)
 *   I        32 f32             input state (src/app.js:48-57)
 *   Queue    1 + 16,384 u32     refresh count + queued slots
 *   Args     8 x 21 u32         per-chunk dispatch sizes
 *   Hit      W*H x 4 f32        [t, fid, material, seed]; fid -10000 = sky, -1 = ground
 *   Surface  W*H x 4 f32        [n.xyz, slot]
 *   Linear, History  W*H x 4 f32;   Pixels  W*H u32 (RGBA8)
 *
 * Every function returns STRATUM_OK (0) after enqueueing its work on `stream`,
 * STRATUM_EINVAL for a bad argument (nothing is launched), or -(cudaError_t)
 * when the launch itself failed.  Positive values are service statuses.
 * Nothing here allocates or synchronises unless stated.
 */
#ifndef STRATUM_H
#define STRATUM_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* stratum_stream_t; /* a cudaStream_t; NULL = legacy default stream */

#define STRATUM_OK 0
#define STRATUM_EINVAL (-100000)
#define STRATUM_QUEUE_STALLED 1      /* a bounded device wait ran out */
#define STRATUM_BUDGET_EXCEEDED 2    /* admission refused: HBM budget */
#define STRATUM_NOT_FOUND 3          /* unknown session / request */

/* ABI constants (kernels/common.cu:2-16 == src/engine.js:2) */
#define STRATUM_WORLD_SIDE 128
#define STRATUM_WORLD_LOTS 16384
#define STRATUM_LOT_FLOATS 16
#define STRATUM_CLUSTERS 64
#define STRATUM_GROUP_NODES 128
#define STRATUM_MAX_FEATURES 64
#define STRATUM_BUILD_CHUNK 2048
#define STRATUM_BUILD_CHUNKS 8
#define STRATUM_RAY_DISTANCE 2000
#define STRATUM_MAX_DIM 16384

/* ---- camera and world (kernels/world.cu) ---------------------------------- */
/* initCamera(float*C, unsigned*Origin, int seed)          kernels/world.cu:57 */
int stratum_initCamera(float* C, unsigned* Origin, int seed, stratum_stream_t stream);
/* stepCamera(C, Origin, I, dt, width, height)              kernels/world.cu:64 */
int stratum_stepCamera(float* C, unsigned* Origin, const float* I, float dt, int width, int height,
                       stratum_stream_t stream);
/* clearQueue(unsigned*Queue)                               kernels/world.cu:93 */
int stratum_clearQueue(unsigned* Queue, stratum_stream_t stream);
/* prepareLots(Origin, C, World, Tags, Queue)               kernels/world.cu:94
 * Queue order follows device atomics (varies run to run); its set does not. */
int stratum_prepareLots(const unsigned* Origin, const float* C, float* World, unsigned* Tags, unsigned* Queue,
                        stratum_stream_t stream);
/* planBounds(Queue, Args)                                  kernels/world.cu:106 */
int stratum_planBounds(const unsigned* Queue, unsigned* Args, stratum_stream_t stream);

/* ---- bounding hierarchy (kernels/accel.cu) -------------------------------- */
/* buildGroupBounds(Queue, World, Nodes, queueBase)         kernels/accel.cu:2
 * Lots queueBase .. queueBase+2047 of the queue (the reference's indirect
 * dispatch becomes a fixed grid whose surplus blocks exit). */
int stratum_buildGroupBounds(const unsigned* Queue, const float* World, float* Nodes, int queueBase,
                             stratum_stream_t stream);
/* reduceGroupBounds(Queue, Nodes, first, queueBase)         kernels/accel.cu:9
 * first in {32,16,8,4,2,1}. */
int stratum_reduceGroupBounds(const unsigned* Queue, float* Nodes, int first, int queueBase, stratum_stream_t stream);

/* ---- frame (kernels/trace.cu, kernels/shade.cu) --------------------------- */
/* tracePrimary(World, Nodes, Origin, C, Hit, Surface, width, height, rowStart, rowCount)   kernels/trace.cu:29 */
int stratum_tracePrimary(const float* World, const float* Nodes, const unsigned* Origin, const float* C, float* Hit,
                         float* Surface, int width, int height, int rowStart, int rowCount, stratum_stream_t stream);
/* shadePixels(World, Origin, C, Hit, Surface, Linear, width, height, rowStart, rowCount)    kernels/shade.cu:45 */
int stratum_shadePixels(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                        const float* Surface, float* Linear, int width, int height, int rowStart, int rowCount,
                        stratum_stream_t stream);
/* resolveFrame(Linear, History, Pixels, C, Hit, Surface, width, height)                     kernels/shade.cu:104 */
int stratum_resolveFrame(const float* Linear, float* History, unsigned* Pixels, const float* C, const float* Hit,
                         const float* Surface, int width, int height, stratum_stream_t stream);
/* probeGrammar(Inputs[17], Output[16])                      kernels/probe.cu:2 */
int stratum_probeGrammar(const float* Inputs, float* Output, stratum_stream_t stream);

/* ---- page-oriented names of the same roles (legacy names of Stratum.cu) --- */
/* initWorld = initCamera (Stratum.cu:95 role)                                   */
int stratum_initWorld(float* C, unsigned* Origin, int seed, stratum_stream_t stream);
/* schedulePages = clearQueue + prepareLots (Stratum.cu:172 role)                */
int stratum_schedulePages(const unsigned* Origin, const float* C, float* World, unsigned* Tags, unsigned* Queue,
                          stratum_stream_t stream);
/* commitPages = planBounds (Stratum.cu:186 role)                                */
int stratum_commitPages(const unsigned* Queue, unsigned* Args, stratum_stream_t stream);
/* buildBVH = buildGroupBounds + reduceGroupBounds x6 over the whole queue, as
 * one fused kernel (a block per lot; same bits).  Replaces the 8 x 7 indirect
 * dispatches of src/engine.js:71,74. */
int stratum_buildBVH(const unsigned* Queue, const float* World, float* Nodes, stratum_stream_t stream);

/* ---- whole frame (the ordered sequence of src/engine.js:67-83) ------------ */
/* stepCamera, clearQueue, prepareLots, planBounds, buildBVH, then trace and
 * shade in 64-row strips and resolveFrame.  `Args` may be NULL. */
int stratum_frame(float* C, unsigned* Origin, const float* I, float dt, float* World, unsigned* Tags, float* Nodes,
                  unsigned* Queue, unsigned* Args, float* Hit, float* Surface, float* Linear, float* History,
                  unsigned* Pixels, int width, int height, int draw, stratum_stream_t stream);

/* ---- grammar services (test and tooling) ---------------------------------- */
/* Feature records of `pairs` (lot, group) pairs: Lots = pairs x 16 f32 World
 * rows, Groups = pairs i32.  Records = pairs x cap x 10 f32
 * [p.xyz, h.xyz, shape, material, turn, seed]; Counts = pairs i32 (full count,
 * even when above cap).  cap <= 64. */
int stratum_enumerateGroups(const float* Lots, const int* Groups, int pairs, int cap, float* Records, int* Counts,
                            stratum_stream_t stream);
/* Analytic test of n (feature, ray) rows [feature(10), ro(3), rd(3), cone] ->
 * Results n x [t, normal.xyz] (kernels/geometry.cu:33,92). */
int stratum_featureQuery(const float* Queries, int n, float* Results, stratum_stream_t stream);

/* Nearest hit of n arbitrary rays in a view's table (kernels/trace.cu:8-61):
 * Rays n x 7 f32 [ro.xyz, rd.xyz, cone] in the floating-origin frame; Out
 * n x 8 f32 [t, fid, material, seed, normal.xyz, slot].  exhaustive = 1
 * evaluates every group of every visited lot (no hierarchy culling; Nodes may
 * be NULL): the check of the hierarchy (tests/native_harness.cpp:68-79). */
int stratum_traceRays(const float* World, const float* Nodes, const unsigned* Origin, const float* Rays, int n,
                      int exhaustive, float* Out, stratum_stream_t stream);
/* One named feature per ray: Ids n x 2 i32 [slot, fid] (a traced ray's Out[7]
 * and Out[1]) -> Out n x 4 f32 [t, normal.xyz], the feature regenerated from
 * the slot's descriptor and intersected in its lot frame as the trace does
 * (kernels/world.cu:37-56, kernels/sink.cu:21, kernels/geometry.cu:33,92);
 * t = 2000 where the ray misses it.  Two ids of one ray that give the same t bit
 * for bit are an exact tie: either is a correct nearest hit. */
int stratum_retestFeatures(const float* World, const unsigned* Origin, const float* Rays, const int* Ids, int n,
                           float* Out, stratum_stream_t stream);

/* ---- optional material surrogate (kernels/learning.cu; the reference keeps it
 * out of its build) --------------------------------------------------------
 * An 8 -> 24 tanh -> 3 network (291 parameters W, Adam moments M and V) that
 * learns the substrate colour of brick and stone from the frame's hit pixels;
 * Brain[32] holds the step count, validation samples, errors, the gate
 * Brain[4] and the last batch size.  Inputs come from the current buffers:
 * Hit material and seed, Surface normal and slot, lot-frame masonry
 * coordinates. */
#define STRATUM_NN_PARAMS 291
/* learning.cu:5-10: W, M, V (291 each) and Brain (32) from a seed. */
int stratum_initNeural(float* W, float* M, float* V, float* Brain, int seed, stratum_stream_t stream);
/* learning.cu:11-58 fused into one launch: on frames with C[6] % 4 == 0 and
 * C[21] < 0.5, sample 64 brick/stone pixels, score the 8 held-out ones, update
 * the gate and take one Adam step on the other 56.  Work (may be NULL) receives
 * the 64 x 64 sample rows. */
int stratum_materialStep(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                         const float* Surface, float* W, float* M, float* V, float* Brain, float* Work, int width,
                         int height, stratum_stream_t stream);
/* The surrogate's colour for n queries [u, v, seed, material] -> n x 3. */
int stratum_predictSubstrate(const float* W, const float* Queries, int n, float* Out, stratum_stream_t stream);
/* shadePixels with the surrogate for brick and stone when C[16] > 0.5 and
 * Brain[4] > 0.5 (the reference's pre-refactor shade path), else identical. */
int stratum_shadePixelsNeural(const float* World, const unsigned* Origin, const float* C, const float* Hit,
                              const float* Surface, float* Linear, const float* W, const float* Brain, int width,
                              int height, int rowStart, int rowCount, stratum_stream_t stream);

/* ---- batched views (no reference counterpart: B200 multi-view form) ------- */
/* One view of a batch: device pointers to that view's own buffers, in the
 * layouts above, plus its frame size and time step.  A batch is a DEVICE array
 * of these; tileBase/tilesX are written by stratum_renderViews. */
typedef struct stratum_view {
  float* C;
  unsigned* Origin;
  const float* I;
  float* World;
  unsigned* Tags;
  float* Nodes;
  unsigned* Queue;
  float* Hit;
  float* Surface;
  float* Linear;
  float* History;
  unsigned* Pixels;
  unsigned* Groups; /* the table's group cache (stratum_groupCacheInit), or NULL */
  int width, height;
  float dt;
  int tileBase, tilesX, reserved;
} stratum_view;

/* Group cache of one table: the feature records of the (lot, group) pairs the
 * batched trace has evaluated, filled on first use and loaded afterwards
 * instead of being rebuilt by the grammar.  `entries` groups of at most 56
 * records (2,192 bytes each, with their culling boxes) plus a 4 MiB directory.  Entries are checked
 * against the table's current descriptor rows, so the cache never needs
 * invalidating when the table is refreshed (by any entry point); a full cache
 * keeps serving its groups and is emptied at most every 8 batched frames.  A trace launch uses the
 * groups filled by earlier launches (the first frame of a view fills, the
 * following ones reuse; at most 16,777,214 entries).  Results are identical
 * with and without a cache.  Initialise once before use (zeroes the directory,
 * sets the capacity); a zero-filled buffer is a cache of capacity 0. */
unsigned long long stratum_groupCacheBytes(int entries);
int stratum_groupCacheInit(unsigned* Groups, int entries, stratum_stream_t stream);

/* Tunables of the batched trace: block size (64/128/256), tiles a warp claims
 * per queue access (queue depth, 1..16), tile order within a view (bit 0 of
 * order: 0 row-major, 1 Morton-ordered 4x4-tile super-tiles).  Bit 1 of order
 * selects the block-pooled trace, in which the warps of a block serve one
 * another's groups (same results; slower on the benchmark views, so
 * stratum_autotune never chooses it).  Chosen by stratum_autotune. */
typedef struct stratum_tune {
  int threads;
  int grab;
  int order;
} stratum_tune;

/* Device scratch the batched renderer needs for `views` views (work-queue
 * counters and per-view frame constants).  Zero it once before first use; the
 * kernels leave their counters at zero when they finish. */
unsigned long long stratum_batchScratchBytes(int views);
/* stepCamera of every view (dt from the view). */
int stratum_stepViews(stratum_view* views, int n, stratum_stream_t stream);
/* clearQueue + prepareLots of every view, one launch each. */
int stratum_refreshViews(stratum_view* views, int n, stratum_stream_t stream);
/* Every view's queued lots rebuilt in one fused launch. */
int stratum_buildViews(stratum_view* views, int n, stratum_stream_t stream);
/* All views' primary rays through one persistent kernel pulling 8x4-pixel
 * tiles from a device work queue, then one persistent shade+resolve pass. */
int stratum_renderViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                        const stratum_tune* tune, stratum_stream_t stream);
/* The trace half of renderViews alone (Hit, Surface). */
int stratum_traceViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream);
/* The shade + resolve half alone; follows a traceViews of the same views,
 * scratch and tune (it reuses that call's tile bases and frame constants). */
int stratum_shadeViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream);
/* Time every candidate tune (block size x queue depth x tile order) on this
 * batch with CUDA events and return the fastest in *best (and its trace time
 * in *bestMs when not NULL).  Synchronises `stream`. */
int stratum_autotune(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes, stratum_tune* best,
                     float* bestMs, stratum_stream_t stream);
/* renderViews for callers that cannot allocate device memory.  No counterpart
 * in the reference: the reference's engine owns all its buffers, while some
 * callers of this library cannot hand it a scratch buffer -- an embedding that
 * gives every byte of HBM to its own pool (a session server that budgets all
 * memory to per-session tables), a foreign-language binding with no device
 * allocator, or a frame loop that must not allocate.  This variant keeps the
 * renderer's scratch (work-queue counters and per-view frame constants) in a
 * static device array of the library: about 6.9 KB, held by every GPU that
 * loads the library until the process exits.  It allocates nothing and calls
 * no allocating routine.
 * Limits: at most STRATUM_NOALLOC_MAX_VIEWS views per call; more returns
 * STRATUM_ELIMIT and launches nothing.  The first call on each device looks up
 * the array's address (cudaGetSymbolAddress); make that first call before any
 * stream capture on that device.  The address is kept per device context: after
 * a cudaDeviceReset the next call looks it up again, so make that call, too,
 * outside a capture.  All calls share the one array: calls whose
 * work overlaps on the GPU (unordered streams) race and corrupt each other's
 * frames, so order them on one stream or with events.  Each call clears the
 * queue counters and rewrites the per-view constants before using them. */
#define STRATUM_NOALLOC_MAX_VIEWS 64
#define STRATUM_ELIMIT (-100001) /* request exceeds a fixed capacity of the library */
int stratum_renderViewsNoAlloc(stratum_view* views, int n, const stratum_tune* tune, stratum_stream_t stream);
/* The whole batched frame: stepViews, refreshViews, buildViews, renderViews. */
int stratum_frameViews(stratum_view* views, int n, void* scratch, unsigned long long scratchBytes,
                       const stratum_tune* tune, stratum_stream_t stream);

/* ---- measurement ------------------------------------------------------------ */
/* FP32 issue-rate probe: `blocks` x 256 threads, each `iters` iterations of 8
 * independent multiply-add chains (2 ops each).  Lane ops per launch =
 * blocks * 256 * iters * 16.  Used as the roofline denominator of the frame
 * path (its kernels are FP32-issue bound).  `out` receives nothing in practice. */
int stratum_issueProbe(float* out, int blocks, int iters, stratum_stream_t stream);

/* ---- serving (no reference counterpart: the reference renders one view) --- */
/* Absolute camera pose: 64-bit lot address per axis and a position (metres)
 * in that lot's frame, yaw and pitch (radians). */
typedef struct stratum_pose {
  unsigned origin[4];
  float pos[3];
  float yaw, pitch;
} stratum_pose;

/* Per view: flags bit 0 = set the pose (C[0..4], Origin), bit 1 = restart
 * the sample sequence at the next stepCamera (through I[23], the reference's
 * resize-reset input).  Views, poses and flags are device arrays. */
int stratum_applyPoses(stratum_view* views, const stratum_pose* poses, const int* flags, int n, stratum_stream_t stream);

typedef struct stratum_server stratum_server;
typedef struct stratum_server_stats {
  long long submitted, completed, failed, batches, admissions, evictions;
  long long resident_sessions;
  unsigned long long resident_bytes, budget_bytes;
  double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> frame on the host, completed requests */
  double rays;                            /* shaded rays rendered */
  double first_submit_s, last_done_s;     /* wall-clock span of the served requests */
} stratum_server_stats;
typedef struct stratum_request_info {
  int status;          /* STRATUM_OK done, STRATUM_QUEUE_STALLED pending, or an error */
  int samples_done;
  double latency_ms;   /* submit -> done */
  double queue_ms;     /* submit -> first launch */
} stratum_request_info;

/* A render server on the current device: sessions are admitted while their
 * device state fits in `budget_bytes`, least recently used idle sessions are
 * evicted (snapshotted to host memory) to make room, and a scheduler thread
 * batches up to `max_views` requests per launch over `streams` streams, so a
 * batch can be forming and launching while others run.  `tune` may be NULL. */
stratum_server* stratum_server_create(unsigned long long budget_bytes, int max_views, int streams,
                                      const stratum_tune* tune);
void stratum_server_destroy(stratum_server* server);
/* Group cache entries of every session's table (default 16,384: 38 MiB per
 * session, counted in the budget; 0: none).  Only before the first open. */
int stratum_server_set_group_cache(stratum_server* server, int entries);
/* Register a session (not yet resident: admission happens with its first request). */
int stratum_server_open(stratum_server* server, int seed, int width, int height, int* session);
int stratum_server_close(stratum_server* server, int session);
/* Queue `samples` samples of `session` at `pose`.  A pose equal to the
 * session's previous one keeps accumulating toward 64 samples; a new pose
 * restarts the sequence.  When the last sample is done its RGBA8 frame is
 * copied to `out` (width*height*4 bytes, may be NULL). */
int stratum_server_submit(stratum_server* server, int session, const stratum_pose* pose, int samples,
                          unsigned char* out, long long* request);
/* Wait up to timeout_ms for a request: STRATUM_OK when done,
 * STRATUM_QUEUE_STALLED when the time ran out (the request stays queued). */
int stratum_server_wait(stratum_server* server, long long request, int timeout_ms, stratum_request_info* info);
int stratum_server_stats_get(stratum_server* server, stratum_server_stats* stats);
/* Host-side fault injection for tests: kind 1 = the next `count` session
 * admissions fail as if the device allocation had failed; kind 2 = the next
 * `count` batch launches fail after refreshViews, with part of the batch's work
 * already queued (its requests fail once that work has drained; its sessions
 * restart their sampling on their next request). */
int stratum_server_inject(stratum_server* server, int kind, int count);
/* The last frame (RGBA8) and accumulation buffer of a resident session, copied
 * to host memory (test and tooling; synchronises the session). */
int stratum_server_read(stratum_server* server, int session, unsigned char* rgba, float* history);

/* Library version string. */
const char* stratum_version(void);

#ifdef __cplusplus
}
#endif
#endif /* STRATUM_H */
