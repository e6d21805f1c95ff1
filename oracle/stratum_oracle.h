/* Test infrastructure only: the CPU oracle (a restatement of the reference's
 * frame path) used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg.  The product never links it.
 *
 * Buffer layouts are those of the reference entry points:
 *   World   16,384 x 16 f32   [w,d,h,type,mat,floors,seed,storey,roofScale,turn,ox,oz,palette,-,-,valid]
 *   Tags    16,384 x 4  u32   64-bit lot address (xl,xh,zl,zh)
 *   Nodes   16,384 x 128 x 8 f32   node = [lo.xyz, count, hi.xyz, group]
 *   Hit     P x 4 f32  [t, fid, material, seed];  Surface P x 4 f32 [n.xyz, slot]
 *   Linear, History  P x 4 f32;  Pixels P u32 (RGBA8)
 * Feature record (test interface): 10 f32 [p.xyz, h.xyz, shape, material, turn, seed].
 */
#ifndef STRATUM_ORACLE_H
#define STRATUM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Work counters filled by orc_trace / orc_shade (indices). */
enum {
  ORC_RAYS = 0,      /* primary rays traced */
  ORC_DDA = 1,       /* lot DDA cells visited (trace.cu:47) */
  ORC_NODE = 2,      /* nodeNear tests (trace.cu:2) */
  ORC_GROUP = 3,     /* mode-0 group emissions (trace.cu:22) */
  ORC_FEAT = 4,      /* featureHit calls (sink.cu:22) */
  ORC_FOLIAGE = 5,   /* foliage DDA cells (geometry.cu:17) */
  ORC_MASONRY = 6,   /* masonry relief iterations (geometry.cu:87) */
  ORC_SDDA = 7,      /* shadow DDA cells (shade.cu:9) */
  ORC_SHADED = 8,    /* hit pixels shaded (not sky) */
  ORC_SHADED_MASONRY = 9,  /* shaded pixels of brick/stone (materials 0, 1) */
  ORC_PASS_BOX = 10,       /* featureHit calls past the slab test, by shape */
  ORC_PASS_ELLIPSOID = 11,
  ORC_PASS_CYLINDER = 12,
  ORC_PASS_PRISM = 13,
  ORC_PASS_ARCH = 14,      /* shapes 4 and 7 */
  ORC_EMIT = 15,           /* features emitted in mode 0 (same as ORC_FEAT) */
  ORC_COUNTERS = 32
};

/* Sines and cosines of camera, sun and resolve-tap angles: 0 (default) = the C
 * library's float functions, as the reference's CPU build; 1 = double precision
 * rounded once to float, as the CUDA path.  Process-wide. */
void orc_setAngleRounding(int mode);
int orc_angleRounding(void);
/* The camera's forward and right vectors under the current angle mode. */
void orc_cameraBasis(const float* C, float* out6);
void orc_offset_tag(const uint32_t* origin, int dx, int dz, uint32_t* out4);
uint32_t orc_tag_hash(const uint32_t* tag4, int seed);
uint32_t orc_hashU(uint32_t x);
void orc_describe_lot(const uint32_t* tag4, int seed, float* out16);

void orc_initCamera(float* C, uint32_t* Origin, int seed);
void orc_stepCamera(float* C, uint32_t* Origin, const float* I, float dt, int width, int height);
void orc_clearQueue(uint32_t* Queue);
void orc_prepareLots(const uint32_t* Origin, const float* C, float* World, uint32_t* Tags, uint32_t* Queue);
void orc_planBounds(const uint32_t* Queue, uint32_t* Args);
void orc_buildBounds(const uint32_t* Queue, const float* World, float* Nodes, int nthreads);

int orc_enumerate(const float* lot16, int group, float* out10, int cap);
void orc_group_bounds(const float* lot16, int group, float* out7);
float orc_featureHit(const float* f10, const float* ro, const float* rd, float cone);
void orc_featureNormal(const float* f10, const float* point, float* n3);
double orc_featureHit_f64(const float* f10, const double* ro, const double* rd, double cone);
void orc_featureNormal_f64(const float* f10, const double* point, double* n3);
float orc_queryLot(const float* lot16, const float* nodes128, const float* ro, const float* rd, float best,
                   float cone, int* fid, float* f10);
float orc_queryLot_exhaustive(const float* lot16, const float* ro, const float* rd, float best, float cone,
                              int* fid, float* f10);

/* second (may be NULL): per pixel, the second-smallest candidate distance seen
 * by the ray (FAR if none) -- the tie rule for identity comparisons. */
void orc_tracePrimary(const float* World, const float* Nodes, const uint32_t* Origin, const float* C, float* Hit,
                      float* Surface, int width, int height, int rowStart, int rowCount, int nthreads,
                      int64_t* counters, float* second);
void orc_shadePixels(const float* World, const uint32_t* Origin, const float* C, const float* Hit,
                     const float* Surface, float* Linear, int width, int height, int rowStart, int rowCount,
                     int nthreads, int64_t* counters);
void orc_resolveFrame(const float* Linear, float* History, uint32_t* Pixels, const float* C, const float* Hit,
                      const float* Surface, int width, int height, int nthreads);
/* rays: n x 7 [ro.xyz, rd.xyz, cone]; out: n x 8 [t, fid, material, seed, n.xyz, slot] */
void orc_traceRays(const float* World, const float* Nodes, const uint32_t* Origin, const float* rays, int n,
                   int exhaustive, float* out, int nthreads);
void orc_resolveRows(const float* Linear, float* History, uint32_t* Pixels, const float* C, const float* Hit,
                     const float* Surface, int width, int height, int rowStart, int rowCount, int nthreads);
void orc_probeGrammar(const float* Inputs, float* Output);
/* The optional material surrogate (learning.cu): init, one training step
 * (Work: 64 x 64 sample rows, may be NULL), the surrogate colour of n queries
 * [u, v, seed, material] -> n x 3, and shadePixels with the surrogate. */
void orc_initNeural(float* W, float* M, float* V, float* Brain, int seed);
void orc_materialStep(const float* World, const uint32_t* Origin, const float* C, const float* Hit,
                      const float* Surface, float* W, float* M, float* V, float* Brain, float* Work, int width,
                      int height);
void orc_predictSubstrate(const float* W, const float* Queries, int n, float* out);
void orc_shadePixelsNeural(const float* World, const uint32_t* Origin, const float* C, const float* Hit,
                           const float* Surface, float* Linear, const float* W, const float* Brain, int width,
                           int height, int rowStart, int rowCount, int nthreads);
/* trace + shade + resolve of the listed rows (rows[nrows]) only. */
void orc_renderRows(const float* World, const float* Nodes, const uint32_t* Origin, const float* C, float* Hit,
                    float* Surface, float* Linear, float* History, uint32_t* Pixels, int width, int height,
                    const int32_t* rows, int nrows, int nthreads);
/* rays n x 7 as orc_traceRays; ids n x 2 [slot, fid]; out n x 4 [t, n.xyz] of
 * that one feature on that ray (t = 2000 if missed). */
void orc_retestFeatures(const float* World, const uint32_t* Origin, const float* rays, const int32_t* ids, int n,
                        float* out, int nthreads);
/* FP64 re-intersection of every pixel's winning feature, given a frame's
 * World/Origin/C and its Hit/Surface: t64 (P), n64 (P x 6, world frame: the
 * normal at the FP64 hit, then at the frame's own float hit point) and a
 * status per pixel: 0 sky, 1 ground plane, 2 feature, 3 foliage leaf disc,
 * 4 not re-found in FP64, in bits 0-2; the feature's shape in bits 3-6 and
 * its material from bit 8. */
void orc_reintersectF64(const float* World, const uint32_t* Origin, const float* C, const float* Hit,
                        const float* Surface, int width, int height, double* t64, double* n64, int32_t* status,
                        int nthreads);

#ifdef __cplusplus
}
#endif
#endif
