// One lot's 127-node bounding hierarchy in one 64-thread block
// (kernels/accel.cu of the reference, fused): thread g runs the grammar of
// group g in bounds mode and writes leaf 64+g, the 63 internal nodes are
// reduced in shared memory, and the block leaves as one coalesced 4 KiB store.
// Min/max and small-integer sums are exact, so this equals the reference's
// two-kernel form bit for bit.  Node 0 of a lot block is never written.
#pragma once
#include "grammar.cuh"

namespace st {

// Queue length clamped to the table, so a stale count never reads past the queue.
SD int queued(const uint32_t* Q) { return int(min(Q[0], uint32_t(kLots))); }

SD void leafBounds(const LotDesc& lot, int g, float* n) {
  BoundsSink s;
  int count = runGroup(lot, g, s);
  n[0] = s.lo.x; n[1] = s.lo.y; n[2] = s.lo.z; n[3] = float(count);
  n[4] = s.hi.x; n[5] = s.hi.y; n[6] = s.hi.z; n[7] = float(g);
}

SD void lotHierarchy(const float* W, float* N, int slot, float (*sm)[8]) {
  const int g = int(threadIdx.x);
  LotDesc lot = loadLotRW(W, slot);
  leafBounds(lot, g, sm[kGroups + g]);
  __syncthreads();
#pragma unroll 1
  for (int first = 32; first >= 1; first >>= 1) {
    if (g < first) {
      int j = first + g;
      float *b = sm[j], *a = sm[2 * j], *c = sm[2 * j + 1];
#pragma unroll
      for (int k = 0; k < 3; k++) { b[k] = fminf(a[k], c[k]); b[4 + k] = fmaxf(a[4 + k], c[4 + k]); }
      b[3] = a[3] + c[3];
      b[7] = 0.0f;
    }
    __syncthreads();
  }
  float4* dst = reinterpret_cast<float4*>(N + size_t(slot) * kNodes * 8);
  const float4* src = reinterpret_cast<const float4*>(&sm[0][0]);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int i = g + 64 * k;  // float4 index within the 4 KiB block; 0 and 1 are node 0
    if (i >= 2) dst[i] = src[i];
  }
  __syncthreads();
}

// Grid-stride over one queue: block b takes queue entries b, b + grid, ...
SD void buildQueue(const uint32_t* Q, const float* W, float* N, int first, int stride, float (*sm)[8]) {
  const int count = queued(Q);
#pragma unroll 1
  for (int q = first; q < count; q += stride) {
    int slot = int(Q[q + 1]);
    if (slot >= 0 && slot < kLots) lotHierarchy(W, N, slot, sm);
  }
}

}  // namespace st
