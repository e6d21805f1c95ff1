// Test infrastructure: the device feature grammar (sequential and random
// access) compiled for the HOST, so CPU tests can compare it with the oracle
// bit for bit without a GPU.  Built by tests/test_grammar_host.py.
#include "grammar_ra.cuh"

using namespace st;

namespace {
struct HostStore {
  float* out;
  int cap;
  HD void take(const Feat& f, int id) {
    if (id >= cap) return;
    float* o = out + id * 10;
    o[0] = f.p.x; o[1] = f.p.y; o[2] = f.p.z; o[3] = f.h.x; o[4] = f.h.y; o[5] = f.h.z;
    o[6] = float(f.shape); o[7] = float(f.material); o[8] = float(f.turn); o[9] = f.seed;
  }
};
}  // namespace

extern "C" int hg_sequential(const float* lot16, int group, float* out, int cap) {
  LotDesc L = loadLotRW(lot16, 0);
  HostStore s{out, cap};
  return runGroup(L, group, s);
}

extern "C" int hg_random_access(const float* lot16, int group, float* out, int cap) {
  LotDesc L = loadLotRW(lot16, 0);
  HostStore s{out, cap};
  int n = groupCount(L, group);
  for (int i = 0; i < n; i++) s.take(featureAt(L, group, i), i);
  return n;
}
