// probeGrammar (kernels/probe.cu:2-14 of the reference) and the grammar
// enumeration service: feature records of many (lot, group) pairs in one launch.
#include "common_api.cuh"
#include "geometry.cuh"

namespace st {

__global__ void probeGrammarK(const float* In, float* Out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  LotDesc l;
  int g = int(In[0]), index = int(In[1]);
  l.w = In[2]; l.d = In[3]; l.h = In[4]; l.type = int(In[5]); l.mat = int(In[6]); l.floors = int(In[7]);
  l.seed = In[8]; l.storey = In[9]; l.roofScale = In[10]; l.turn = 0; l.ox = 0.0f; l.oz = 0.0f; l.palette = 0.0f;
  PickSink pick{index};
  int count = runGroup(l, g, pick);
  const Feat& f = pick.f;
  Out[0] = float(count); Out[1] = float(f.shape); Out[2] = float(f.material); Out[3] = f.seed;
  Out[4] = f.p.x; Out[5] = f.p.y; Out[6] = f.p.z; Out[7] = f.h.x; Out[8] = f.h.y; Out[9] = f.h.z;
  Out[10] = float(f.turn);
  f3 ro = mk(In[11], In[12], In[13]), rd = mk(In[14], In[15], In[16]);
  HitSink s{ro, rd, 0.0f, kFar, -1, Feat{}};
  runGroup(l, g, s);
  Out[11] = s.t; Out[12] = float(s.fid);
  f3 n = mk(0.0f, 0.0f, 0.0f);
  if (s.fid >= 0) n = featureNormal(s.f, ro + rd * s.t);
  Out[13] = n.x; Out[14] = n.y; Out[15] = n.z;
}

// Records are 10 floats [p.xyz, h.xyz, shape, material, turn, seed]; pair i
// writes up to `cap` records at Out + i*cap*10 and its count at Counts[i].
struct StoreSink {
  float* out;
  int cap;
  SD void take(const Feat& f, int id) {
    if (id >= cap) return;
    float* o = out + id * 10;
    o[0] = f.p.x; o[1] = f.p.y; o[2] = f.p.z; o[3] = f.h.x; o[4] = f.h.y; o[5] = f.h.z;
    o[6] = float(f.shape); o[7] = float(f.material); o[8] = float(f.turn); o[9] = f.seed;
  }
};
__global__ void enumerateGroupsK(const float* Lots, const int* Groups, int pairs, int cap, float* Out, int* Counts) {
  int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= pairs) return;
  LotDesc l = loadLotRW(Lots, i);
  StoreSink s{Out + size_t(i) * cap * 10, cap};
  Counts[i] = runGroup(l, Groups[i], s);
}

// featureHit / featureNormal of many (feature, ray) pairs: In rows are
// [feature(10), ro(3), rd(3), cone]; Out rows are [t, n.xyz] at ro + rd*t.
__global__ void featureQueryK(const float* In, int n, float* Out) {
  int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float* r = In + size_t(i) * 17;
  Feat f{mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), int(r[6]), int(r[7]), int(r[8]), r[9]};
  f3 ro = mk(r[10], r[11], r[12]), rd = mk(r[13], r[14], r[15]);
  float t = featureHitCall(f, ro, rd, r[16]);
  f3 nn = mk(0.0f, 0.0f, 0.0f);
  if (t < kFar) nn = featureNormal(f, ro + rd * t);
  float* o = Out + size_t(i) * 4;
  o[0] = t; o[1] = nn.x; o[2] = nn.y; o[3] = nn.z;
}

}  // namespace st

using namespace st;

extern "C" {

int stratum_probeGrammar(const float* Inputs, float* Output, stratum_stream_t stream) {
  if (!Inputs || !Output) return STRATUM_EINVAL;
  probeGrammarK<<<1, 1, 0, asStream(stream)>>>(Inputs, Output);
  return launchStatus();
}
int stratum_enumerateGroups(const float* Lots, const int* Groups, int pairs, int cap, float* Records, int* Counts,
                            stratum_stream_t stream) {
  if (!Lots || !Groups || !Records || !Counts || pairs < 0 || cap < 0 || cap > STRATUM_MAX_FEATURES) return STRATUM_EINVAL;
  if (pairs == 0) return STRATUM_OK;
  enumerateGroupsK<<<(pairs + 127) / 128, 128, 0, asStream(stream)>>>(Lots, Groups, pairs, cap, Records, Counts);
  return launchStatus();
}
int stratum_featureQuery(const float* Queries, int n, float* Results, stratum_stream_t stream) {
  if (!Queries || !Results || n < 0) return STRATUM_EINVAL;
  if (n == 0) return STRATUM_OK;
  featureQueryK<<<(n + 127) / 128, 128, 0, asStream(stream)>>>(Queries, n, Results);
  return launchStatus();
}

}  // extern "C"
