// Intersection engine: per-type signed triangle counts over the rank-space
// forward CSR.
//
// Reference: count_triangles / merge_intersect / classify
// (MC/tc_serial.cpp:95-170), intersect_signed_ranked
// (MC/tc_merge_sign_enu.cpp:12-44) and the hash probe
// (MC/tc_hash_sign_enu.cpp:125-165).  In rank space every list is sorted and
// every head has a higher rank than its tail, so for the arc u -> v stored at
// position k of N+(u), the third vertex w of a triangle (u, v, w) lies in the
// suffix A' = N+(u)[k+1 ..] and in B = N+(v): the reference's rank filter
// (tc_serial.cpp:126) is implied and half of N+(u) is never looked at.
#include <cuda_runtime.h>

#include "internal.h"
#include "stc_device.cuh"

namespace stc {

namespace {

constexpr int kThreads = 256;

struct Csr {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ nbr;
  const int8_t* __restrict__ sgn;
  const uint32_t* __restrict__ verts;  // rank -> id (per-source counts only)
  uint32_t n;
};

// Per-lane type counters indexed by the number of negative edges.
struct TypeCounts {
  unsigned long long c[4] = {0, 0, 0, 0};
  __device__ __forceinline__ void add(uint32_t neg) {
    c[0] += neg == 0;
    c[1] += neg == 1;
    c[2] += neg == 2;
    c[3] += neg == 3;
  }
};

// First index i in [0, len) with a[i] >= x (len if none).
__device__ __forceinline__ uint32_t lower_bound(const uint32_t* __restrict__ a, uint32_t len,
                                                uint32_t x) {
  uint32_t lo = 0, hi = len;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Block reduction of the four counters and one atomic per counter.
// Slot C_T0 + k receives type Tk = 3 - (negative edges).
__device__ __forceinline__ void flush_counts(TypeCounts& tc, unsigned long long* __restrict__ ctr) {
  __shared__ unsigned long long red[kThreads / 32][4];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const unsigned long long v = warp_sum(tc.c[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long s = 0;
    for (int w = 0; w < kThreads / 32; w++) s += red[w][threadIdx.x];
    if (s) atomicAdd(ctr + C_T0 + (3 - threadIdx.x), s);
  }
}

// Strategy "search": warp per source vertex u; for each arc u -> v the lanes
// take the shorter of A' and B and binary-search each element in the other.
template <bool kVertexCounts>
__global__ void __launch_bounds__(kThreads) k_count_search(Csr g, unsigned long long* __restrict__ ctr,
                                                           unsigned long long* __restrict__ vcounts) {
  TypeCounts tc;
  const unsigned lane = lane_id();
  const uint32_t warps = gridDim.x * (kThreads / 32);
  for (uint32_t u = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); u < g.n; u += warps) {
    const uint64_t ub = g.off[u];
    const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
    TypeCounts vc;
    for (uint32_t k = 0; k + 1 < d; k++) {
      const uint32_t v = g.nbr[ub + k];
      const uint32_t nuv = g.sgn[ub + k] < 0;
      const uint32_t* A = g.nbr + ub + k + 1;
      const int8_t* SA = g.sgn + ub + k + 1;
      const uint32_t alen = d - k - 1;
      const uint64_t vb = g.off[v];
      const uint32_t blen = (uint32_t)(g.off[v + 1] - vb);
      const uint32_t* B = g.nbr + vb;
      const int8_t* SB = g.sgn + vb;
      if (blen == 0) continue;
      if (alen <= blen) {
        for (uint32_t i = lane; i < alen; i += 32) {
          const uint32_t x = A[i];
          const uint32_t j = lower_bound(B, blen, x);
          if (j < blen && B[j] == x) {
            const uint32_t neg = nuv + (SA[i] < 0) + (SB[j] < 0);
            if (kVertexCounts) vc.add(neg); else tc.add(neg);
          }
        }
      } else {
        for (uint32_t j = lane; j < blen; j += 32) {
          const uint32_t y = B[j];
          const uint32_t i = lower_bound(A, alen, y);
          if (i < alen && A[i] == y) {
            const uint32_t neg = nuv + (SA[i] < 0) + (SB[j] < 0);
            if (kVertexCounts) vc.add(neg); else tc.add(neg);
          }
        }
      }
    }
    if (kVertexCounts) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const unsigned long long s = warp_sum(vc.c[k]);
        tc.c[k] += vc.c[k];
        if (lane == 0) vcounts[4ull * g.verts[u] + (3 - k)] = s;
      }
    }
  }
  flush_counts(tc, ctr);
}

}  // namespace

void count_triangles(stc_ctx* c, const DeviceGraph& g, const CountConfig& cfg) {
  if (g.n == 0 || g.m_fwd == 0) return;
  Csr csr{g.off, g.nbr, g.sgn, g.verts, g.n};
  unsigned long long* ctr = (unsigned long long*)counters(c);
  const uint32_t grid = kSMs * 8;
  if (cfg.vertex_counts) {
    k_count_search<true><<<grid, kThreads, 0, c->stream>>>(csr, ctr,
                                                            (unsigned long long*)cfg.vertex_counts);
  } else {
    k_count_search<false><<<grid, kThreads, 0, c->stream>>>(csr, ctr, nullptr);
  }
  c->launches++;
  STC_CUDA(cudaGetLastError());
}

}  // namespace stc
