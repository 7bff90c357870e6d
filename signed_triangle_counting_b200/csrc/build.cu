// Graph build on the GPU: ingest + dedup, degree, (degree, id) rank,
// orientation and the forward CSR with an int8 sign array.
//
// Reference: build_forward_csr (MC/graph_io.h:231-402) followed by
// sort_adj_lists (MC/tc_serial.cpp:33-93), MC = "Signed_TC/Multicore
// Implementations".  The reference sorts 12-byte structs on one thread,
// counting-sorts vertices by degree and scatters arcs with atomics into
// unsorted lists that a second pass sorts.  Here every stage is a sort or a
// streaming pass over HBM:
//
//   1. pack   (min << b | max), sign in bit 63; self-loops -> sentinel keys
//   2. stable radix sort over the 2b id bits; keep the first key of each run
//      (== the reference's "first of equal (u, v)", made deterministic)
//   3. degree = atomics over the unique keys (warp-aggregated on the min id)
//   4. rank   = stable radix sort of (deg << 32 | id) on the degree bits:
//      ties fall back to ascending id exactly like the counting sort at
//      MC/graph_io.h:270-317
//   5. orient + relabel into rank space: arc (rank lo -> rank hi); sorting
//      these keys gives every list already sorted, so no per-list sort
//   6. offsets = exclusive scan of out-degrees.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "internal.h"
#include "radix_sort.cuh"
#include "stc_device.cuh"

namespace stc {

namespace {

constexpr int kThreads = 256;

inline uint32_t grid_for(uint64_t n, uint32_t per_thread = 1) {
  uint64_t g = (n + (uint64_t)kThreads * per_thread - 1) / ((uint64_t)kThreads * per_thread);
  if (g < 1) g = 1;
  if (g > (uint64_t)kSMs * 16) g = kSMs * 16;
  return (uint32_t)g;
}

// Max kept id and self-loop count.
__global__ void k_scan_ids(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                           uint64_t m, unsigned long long* __restrict__ ctr) {
  uint32_t mx = 0;
  uint32_t self = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t a = __ldcs(u + i), b = __ldcs(v + i);
    if (a == b) {
      self++;
    } else {
      mx = max(mx, max(a, b));
    }
  }
  mx = __reduce_max_sync(kFull, mx);
  self = __reduce_add_sync(kFull, self);
  if (lane_id() == 0) {
    atomicMax(ctr + C_MAX_ID, (unsigned long long)mx);
    if (self) atomicAdd(ctr + C_SELF, (unsigned long long)self);
  }
}

// Dedup keys: (min << bits | max) with the negative flag in bit 63; a
// self-loop becomes the all-ones sentinel of the 2*bits window, which sorts
// last and can never equal a real key (real keys have min < max).
__global__ void k_pack_dedup(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                             const int8_t* __restrict__ s, uint64_t m, uint32_t bits,
                             uint64_t* __restrict__ keys) {
  const uint64_t sentinel = (bits * 2 >= 64) ? ~0ull >> 1 : ((1ull << (2 * bits)) - 1);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t a = __ldcs(u + i), b = __ldcs(v + i);
    const int8_t sg = __ldcs(s + i);
    uint64_t k;
    if (a == b) {
      k = sentinel;
    } else {
      const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
      k = (lo << bits) | hi | ((uint64_t)(sg < 0) << 63);
    }
    keys[i] = k;
  }
}

struct UniqueFlag {
  const uint64_t* keys;
  uint64_t mask;
  __device__ uint32_t operator()(uint64_t i) const {
    if (i == 0) return 1u;
    return (keys[i] & mask) != (keys[i - 1] & mask) ? 1u : 0u;
  }
};
struct UniqueEmit {
  const uint64_t* keys;
  uint64_t* out;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t flag) const {
    if (flag) out[pos] = keys[i];
  }
};

// Undirected degree of every vertex from the sorted unique keys
// (min << bits | max).  The min endpoints of consecutive keys repeat, so a
// warp adds each run with one atomic.  The max endpoints are scattered and a
// few hubs may own millions of them, which would serialise on one address; so
// each CTA counts them in a shared-memory table that it flushes every tile of
// kDegTile keys, adding one global atomic per distinct vertex and tile (a
// vertex that finds no free slot within kDegProbes probes is added directly).
constexpr int kDegTile = 1024;
constexpr int kDegSlots = 2048;  // load <= 1/2 per tile
constexpr int kDegProbes = 8;

__global__ void __launch_bounds__(kThreads) k_degree(const uint64_t* __restrict__ keys, uint64_t mu,
                                                     uint32_t bits, uint32_t* __restrict__ deg) {
  __shared__ uint32_t tkey[kDegSlots], tcnt[kDegSlots];
  constexpr uint32_t kFree = 0xFFFFFFFFu;
  for (int i = threadIdx.x; i < kDegSlots; i += kThreads) {
    tkey[i] = kFree;
    tcnt[i] = 0;
  }
  __syncthreads();
  const uint64_t idmask = (1ull << bits) - 1;
  const uint64_t tiles = (mu + kDegTile - 1) / kDegTile;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
#pragma unroll
    for (int r = 0; r < kDegTile / kThreads; r++) {
      const uint64_t i = t * kDegTile + (uint64_t)r * kThreads + threadIdx.x;
      const bool valid = i < mu;
      const uint64_t k = valid ? keys[i] : 0;
      const uint32_t a = valid ? (uint32_t)((k >> bits) & idmask) : kFree;
      const uint32_t b = valid ? (uint32_t)(k & idmask) : kFree;
      const unsigned pa = __match_any_sync(kFull, a);
      if (valid && (pa & lanemask_lt()) == 0) atomicAdd(deg + a, (uint32_t)__popc(pa));
      const unsigned pb = __match_any_sync(kFull, b);
      if (valid && (pb & lanemask_lt()) == 0) {
        const uint32_t add = (uint32_t)__popc(pb);
        uint32_t slot = (b * 0x9E3779B1u) >> (32 - 11);
        bool placed = false;
        for (int p = 0; p < kDegProbes && !placed; p++) {
          uint32_t cur = tkey[slot];
          if (cur == kFree) {  // claim the slot, or see who claimed it first
            const uint32_t old = atomicCAS(&tkey[slot], kFree, b);
            cur = old == kFree ? b : old;
          }
          if (cur == b) {
            atomicAdd(&tcnt[slot], add);
            placed = true;
          }
          slot = (slot + 1) & (kDegSlots - 1);
        }
        if (!placed) atomicAdd(deg + b, add);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kDegSlots; i += kThreads) {
      const uint32_t v = tkey[i];
      if (v != kFree) {
        atomicAdd(deg + v, tcnt[i]);
        tkey[i] = kFree;
        tcnt[i] = 0;
      }
    }
    __syncthreads();
  }
}

// Vertex sort keys (deg << 32 | id) and the max degree.
__global__ void k_vertex_keys(const uint32_t* __restrict__ deg, uint32_t n,
                              uint64_t* __restrict__ vkeys, unsigned long long* __restrict__ ctr) {
  uint32_t mx = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t d = deg[i];
    vkeys[i] = ((uint64_t)d << 32) | i;
    mx = max(mx, d);
  }
  mx = __reduce_max_sync(kFull, mx);
  if (lane_id() == 0) atomicMax(ctr + C_MAX_DEG, (unsigned long long)mx);
}

__global__ void k_rank(const uint64_t* __restrict__ vkeys, uint32_t n, uint32_t* __restrict__ verts,
                       uint32_t* __restrict__ rank) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
    const uint32_t id = (uint32_t)vkeys[r];
    verts[r] = id;
    rank[id] = r;
  }
}

// Orientation + relabelling: arc key (rank lo << bits | rank hi), sign in
// bit 63; out-degree histogram by rank.
__global__ void k_arc_keys(const uint64_t* __restrict__ ukeys, uint64_t mu, uint32_t bits,
                           const uint32_t* __restrict__ rank, uint64_t* __restrict__ akeys,
                           uint32_t* __restrict__ fdeg) {
  const uint64_t idmask = (1ull << bits) - 1;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < mu; i += stride) {
    const uint64_t k = ukeys[i];
    const uint32_t ra = rank[(k >> bits) & idmask], rb = rank[k & idmask];
    const uint32_t lo = min(ra, rb), hi = max(ra, rb);
    akeys[i] = ((uint64_t)lo << bits) | hi | (k & (1ull << 63));
    atomicAdd(fdeg + lo, 1u);
  }
}

struct LoadU32 {
  const uint32_t* a;
  __device__ uint32_t operator()(uint64_t i) const { return a[i]; }
};
struct EmitOffset {
  uint64_t* off;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t) const { off[i] = pos; }
};

// Algorithmic bytes of the arc at position i (tail u, head v) of a sorted
// CSR: the merge model, 5 (d+(u) + d+(v)) + 25, which a merge of both lists
// reads, and the probe model, 5 min(|A'|, |B|) + 30 (A' = the part of N+(u)
// after v, B = N+(v)), which a hash probe that streams the shorter list
// reads, with the arc's own 25 bytes and its entry staged once.
__device__ __forceinline__ void arc_bytes(uint64_t i, uint32_t u, uint32_t v,
                                          const uint64_t* __restrict__ off,
                                          const uint32_t* __restrict__ fdeg,
                                          unsigned long long& merge, unsigned long long& probe) {
  const uint64_t du = fdeg[u], dv = fdeg[v];
  merge += 5ull * (du + dv) + 25ull;
  const uint64_t alen = off[u + 1] - i - 1;
  probe += 5ull * (alen < dv ? alen : dv) + 30ull;
}

// Splits sorted arc keys into the neighbour, sign, tail and signed-head
// arrays (the last two only when given) and accumulates the merge-model and
// probe-model bytes of every arc (arc_bytes).
__global__ void k_csr_fill(const uint64_t* __restrict__ akeys, uint64_t ma, uint32_t bits,
                           const uint32_t* __restrict__ fdeg, const uint64_t* __restrict__ off,
                           uint32_t* __restrict__ nbr, int8_t* __restrict__ sgn,
                           uint32_t* __restrict__ asrc, uint32_t* __restrict__ nkey,
                           unsigned long long* __restrict__ ctr) {
  const uint64_t idmask = (1ull << bits) - 1;
  unsigned long long bytes = 0, probe = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ma; i += stride) {
    const uint64_t k = akeys[i];
    const uint32_t src = (uint32_t)((k >> bits) & idmask), dst = (uint32_t)(k & idmask);
    nbr[i] = dst;
    sgn[i] = (k >> 63) ? (int8_t)-1 : (int8_t)1;
    if (asrc) asrc[i] = src;
    if (nkey) nkey[i] = (dst << 1) | (uint32_t)(k >> 63);
    arc_bytes(i, src, dst, off, fdeg, bytes, probe);
  }
  bytes = warp_sum(bytes);
  probe = warp_sum(probe);
  if (lane_id() == 0 && bytes) {
    atomicAdd(ctr + C_ALG_BYTES, bytes);
    atomicAdd(ctr + C_PROBE_BYTES, probe);
  }
}

// Arc keys of a reference-layout CSR: one warp per vertex.
__global__ void k_csr_arc_keys(const uint64_t* __restrict__ off, const uint32_t* __restrict__ edges,
                               const int8_t* __restrict__ signs, const uint32_t* __restrict__ rank,
                               uint32_t n, uint32_t bits, uint64_t* __restrict__ akeys,
                               uint32_t* __restrict__ fdeg, unsigned long long* __restrict__ ctr) {
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t u = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); u < n; u += warps) {
    const uint64_t b = off[u], e = off[u + 1];
    const uint32_t ru = rank[u];
    for (uint64_t i = b + lane_id(); i < e; i += 32) {
      const uint32_t w = edges[i];
      if (w >= n || rank[w] <= ru) {
        atomicExch(ctr + C_ERROR, 1ull);  // not a forward CSR of this rank order
        continue;
      }
      akeys[i] = ((uint64_t)ru << bits) | rank[w] | ((uint64_t)(signs[i] < 0) << 63);
    }
    if (lane_id() == 0) fdeg[ru] = (uint32_t)(e - b);
  }
}

// Id-space export keys: (source id << bits | head id), sign in bit 63.
__global__ void k_export_keys(const uint64_t* __restrict__ ukeys, uint64_t mu, uint32_t bits,
                              const uint32_t* __restrict__ rank, uint64_t* __restrict__ ekeys,
                              uint32_t* __restrict__ fdeg_id) {
  const uint64_t idmask = (1ull << bits) - 1;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < mu; i += stride) {
    const uint64_t k = ukeys[i];
    const uint32_t a = (uint32_t)((k >> bits) & idmask), b = (uint32_t)(k & idmask);
    const bool fwd = rank[a] < rank[b];
    const uint32_t s = fwd ? a : b, t = fwd ? b : a;
    ekeys[i] = ((uint64_t)s << bits) | t | (k & (1ull << 63));
    atomicAdd(fdeg_id + s, 1u);
  }
}

void read_counters(stc_ctx* c, int first, int count) {
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + first, counters(c) + first, count * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, c->stream));
  STC_CUDA(cudaStreamSynchronize(c->stream));
}

// Rank-space CSR from unique keys: arc keys, sort, offsets, fill.
void finish_csr_from_arc_keys(stc_ctx* c, DeviceGraph& g, uint64_t* akeys, uint64_t* alt) {
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  uint64_t* sorted = radix_sort(akeys, alt, g.m_fwd, 0, 2 * (int)g.bits, sort_counts, c->stream,
                                &c->launches);
  g.off = buffer<uint64_t>(c, B_OFF, (size_t)g.n + 1);
  range_scan(LoadU32{g.fdeg}, EmitOffset{g.off}, g.n, sums, c->stream, &c->launches);
  STC_CUDA(cudaMemcpyAsync(g.off + g.n, sums + range_partition(g.n, kScanTile, kMaxSortGrid).grid,
                           sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
  g.nbr = buffer<uint32_t>(c, B_NBR, g.m_fwd + 4);  // + 4: the engine reads whole int4 chunks
  g.sgn = buffer<int8_t>(c, B_SGN, g.m_fwd + 4);
  g.asrc = buffer<uint32_t>(c, B_ASRC, g.m_fwd);
  g.nkey = buffer<uint32_t>(c, B_NKEY, g.m_fwd + 8);
  k_csr_fill<<<grid_for(g.m_fwd, 4), kThreads, 0, c->stream>>>(sorted, g.m_fwd, g.bits, g.fdeg,
                                                               g.off, g.nbr, g.sgn, g.asrc,
                                                               g.nkey,
                                                               (unsigned long long*)counters(c));
  c->launches += 1;
  STC_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------ batches ----
// A batch of G graphs is counted as one disjoint union: graph g's local id x
// becomes vbase[g] + x, where vbase is the prefix sum of the graphs' id
// spaces.  Edges (and vertices) of one graph are contiguous, so a CTA that
// owns a contiguous range finds the graph of its first element by binary
// search and then only moves a cursor forward.
__device__ __forceinline__ uint32_t first_segment(const uint64_t* __restrict__ bounds, uint32_t G,
                                                  uint64_t i) {
  uint32_t lo = 0, hi = G;  // largest g with bounds[g] <= i
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (bounds[mid] <= i) lo = mid; else hi = mid;
  }
  return lo;
}

// Id space of every graph (max endpoint + 1) and the self-loop count.
__global__ void k_batch_ids(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                            uint64_t m, const uint64_t* __restrict__ eoff, uint32_t G,
                            uint64_t per_cta, unsigned int* __restrict__ gspace,
                            unsigned long long* __restrict__ ctr) {
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < m ? begin + per_cta : m;
  if (begin >= end) return;
  uint32_t g = first_segment(eoff, G, begin);
  uint32_t self = 0;
  for (uint64_t base = begin + (threadIdx.x & ~31u); base < end; base += blockDim.x) {
    const uint64_t i = base + lane_id();
    const bool valid = i < end;
    uint32_t space = 0;
    if (valid) {
      while (eoff[g + 1] <= i) g++;
      const uint32_t a = u[i], b = v[i];
      self += a == b;
      space = max(a, b) + 1;
    }
    const uint32_t key = valid ? g : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(kFull, key);
    const uint32_t mx = __reduce_max_sync(peers, space);
    if (valid && (peers & lanemask_lt()) == 0) atomicMax(gspace + g, mx);
  }
  self = __reduce_add_sync(kFull, self);
  if (lane_id() == 0 && self) atomicAdd(ctr + C_SELF, (unsigned long long)self);
}

// Dedup keys of the union (global ids), as k_pack_dedup.
__global__ void k_batch_pack(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                             const int8_t* __restrict__ s, uint64_t m,
                             const uint64_t* __restrict__ eoff, const uint64_t* __restrict__ vbase,
                             uint32_t G, uint64_t per_cta, uint32_t bits,
                             uint64_t* __restrict__ keys) {
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < m ? begin + per_cta : m;
  if (begin >= end) return;
  const uint64_t sentinel = (bits * 2 >= 64) ? ~0ull >> 1 : ((1ull << (2 * bits)) - 1);
  uint32_t g = first_segment(eoff, G, begin);
  for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    while (eoff[g + 1] <= i) g++;
    const uint32_t a = u[i], b = v[i];
    uint64_t k;
    if (a == b) {
      k = sentinel;
    } else {
      const uint64_t vb = vbase[g];
      const uint64_t lo = vb + (a < b ? a : b), hi = vb + (a < b ? b : a);
      k = (lo << bits) | hi | ((uint64_t)(s[i] < 0) << 63);
    }
    keys[i] = k;
  }
}

// Adds each vertex's graph above its degree in the vertex sort key, so that
// ranks are graph-major and (degree, id) within a graph.
__global__ void k_batch_vertex_graph(uint64_t* __restrict__ vkeys, uint32_t n,
                                     const uint64_t* __restrict__ vbase, uint32_t G,
                                     uint64_t per_cta, uint32_t shift) {
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < n ? begin + per_cta : n;
  if (begin >= end) return;
  uint32_t g = first_segment(vbase, G, begin);
  for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    while (vbase[g + 1] <= i) g++;
    vkeys[i] |= (uint64_t)g << shift;
  }
}

// ------------------------------------------------------- totals path ----
// A count of totals needs an acyclic orientation, not the reference's: every
// total order of the vertices counts each triangle once, from its lowest
// vertex.  So the totals path orders vertices by (degree counted over the
// input's edge copies, id) instead of (unique degree, id), which needs no
// dedup before the orientation: the arc sort that builds the CSR brings the
// copies of an edge together, and the first of each run is kept, the
// dedup's own rule (the sort is stable, so it is the first in input order).
// This removes the dedup sort of all input edges.

// Global ids of input edge i: the edge's own ids, plus the vertex base of
// its graph for a batch (found once per thread by a binary search, then by
// a cursor that only moves forward, as every thread's indices grow).
struct EdgeIds {
  const uint32_t* __restrict__ u;
  const uint32_t* __restrict__ v;
  const uint64_t* __restrict__ eoff;   // G + 1 edge offsets, or null for one graph
  const uint64_t* __restrict__ vbase;  // G + 1 vertex bases
  uint32_t G;
};

struct EdgeCursor {
  uint32_t g = 0;
  __device__ void start(const EdgeIds& e, uint64_t i) {
    if (e.eoff) g = first_segment(e.eoff, e.G, i);
  }
  __device__ void at(const EdgeIds& e, uint64_t i, uint32_t& a, uint32_t& b) {
    a = e.u[i];
    b = e.v[i];
    if (e.eoff) {
      while (e.eoff[g + 1] <= i) g++;
      const uint32_t base = (uint32_t)e.vbase[g];
      a += base;
      b += base;
    }
  }
};

// Degree of every vertex over the input's edge copies (self-loops skipped),
// or over a sample of them: with `shift` > 0, only the copies of the edges
// {a, b} whose hash has its top `shift` bits clear, 1 in 2^shift of the
// distinct edges (every copy of an edge is in or out together).  The order
// only has to be a total order for exact counts; on dense power-law graphs
// a sampled degree orders the vertices nearly as well (at RMAT scale 20 a
// 1/4 sample moves the intersection work by under 0.1%) for a quarter of
// the atomics.  Endpoints are scattered and a few hubs own millions of
// copies, so each CTA first adds them in a shared-memory table per tile of
// kRawTile edges and flushes the slots it used with one global atomic each
// (an endpoint that finds no free slot within kDegProbes probes is added
// directly).
constexpr int kRawTile = 512;
// Edges of the input are taken in chunks of kEdgeChunk, chunk c by CTA
// c mod grid: the CTAs of a launch work on neighbouring edges at any time,
// so for a batch they gather the ranks and degrees of a few neighbouring
// graphs at once, which stay in L2.
constexpr uint64_t kEdgeChunk = 4096;
constexpr int kRawSlots = 2048;  // 2 kRawTile endpoints per tile: load <= 1/2

__device__ __forceinline__ bool sampled_edge(uint32_t a, uint32_t b, uint32_t shift) {
  if (shift == 0) return true;
  const uint32_t lo = min(a, b), hi = max(a, b);
  return ((lo * 0x9E3779B1u) ^ (hi * 0x7FEB352Du) ^ ((lo ^ hi) >> 15)) >> (32 - shift) == 0;
}

__global__ void __launch_bounds__(kThreads) k_degree_raw(EdgeIds e, uint64_t m, uint32_t shift,
                                                         uint32_t n, uint32_t* __restrict__ deg) {
  __shared__ uint32_t tkey[kRawSlots], tcnt[kRawSlots], used[kRawSlots];
  __shared__ uint32_t nused;
  constexpr uint32_t kFree = 0xFFFFFFFFu;
  for (int i = threadIdx.x; i < kRawSlots; i += kThreads) {
    tkey[i] = kFree;
    tcnt[i] = 0;
  }
  if (threadIdx.x == 0) nused = 0;
  __syncthreads();
  for (uint64_t chunk = blockIdx.x; chunk * kEdgeChunk < m; chunk += gridDim.x) {
    const uint64_t begin = chunk * kEdgeChunk;
    const uint64_t end = begin + kEdgeChunk < m ? begin + kEdgeChunk : m;
    EdgeCursor cur;
    cur.start(e, begin);
    for (uint64_t t = begin; t < end; t += kRawTile) {
  #pragma unroll
      for (int r = 0; r < kRawTile / kThreads; r++) {
        const uint64_t i = t + (uint64_t)r * kThreads + threadIdx.x;
        uint32_t a = kFree, b = kFree;
        if (i < end) {
          cur.at(e, i, a, b);
          // Ids at or past n only reach here when a capped build's union
          // outgrew its capacity (flagged by k_batch_bases).
          if (a == b || a >= n || b >= n || !sampled_edge(a, b, shift)) a = b = kFree;
        }
  #pragma unroll
        for (int side = 0; side < 2; side++) {
          const uint32_t x = side ? b : a;
          const unsigned px = __match_any_sync(kFull, x);
          if (x != kFree && (px & lanemask_lt()) == 0) {
            const uint32_t add = (uint32_t)__popc(px);
            uint32_t slot = (x * 0x9E3779B1u) >> (32 - 11);
            bool placed = false;
            for (int p = 0; p < kDegProbes && !placed; p++) {
              uint32_t c = tkey[slot];
              if (c == kFree) {  // claim the slot, or see who claimed it first
                const uint32_t old = atomicCAS(&tkey[slot], kFree, x);
                if (old == kFree) used[atomicAdd(&nused, 1u)] = slot;
                c = old == kFree ? x : old;
              }
              if (c == x) {
                atomicAdd(&tcnt[slot], add);
                placed = true;
              }
              slot = (slot + 1) & (kRawSlots - 1);
            }
            if (!placed) atomicAdd(deg + x, add);
          }
        }
      }
      __syncthreads();
      const uint32_t nu = nused;
      for (uint32_t j = threadIdx.x; j < nu; j += kThreads) {
        const uint32_t slot = used[j];
        atomicAdd(deg + tkey[slot], tcnt[slot]);
        tkey[slot] = kFree;
        tcnt[slot] = 0;
      }
      __syncthreads();
      if (threadIdx.x == 0) nused = 0;
      __syncthreads();
    }
  }
}

// Arc keys of the input's edge copies in rank space: (rank lo << bits |
// rank hi), the negative flag in bit 63; a self-loop becomes the all-ones
// sentinel of the 2 * bits window, which sorts after every real key.  An
// endpoint at or past n (a capped build whose union outgrew its capacity)
// also becomes the sentinel and sets C_OVERFLOW.
__global__ void k_arc_keys_raw(EdgeIds e, const int8_t* __restrict__ sign, uint64_t m,
                               uint32_t bits, uint32_t n, const uint32_t* __restrict__ rank,
                               uint64_t* __restrict__ akeys, unsigned long long* __restrict__ ctr) {
  const uint64_t sentinel = (bits * 2 >= 64) ? ~0ull >> 1 : ((1ull << (2 * bits)) - 1);
  for (uint64_t chunk = blockIdx.x; chunk * kEdgeChunk < m; chunk += gridDim.x) {
    const uint64_t begin = chunk * kEdgeChunk;
    const uint64_t end = begin + kEdgeChunk < m ? begin + kEdgeChunk : m;
    EdgeCursor cur;
    cur.start(e, begin);
    for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
      uint32_t a, b;
      cur.at(e, i, a, b);
      uint64_t k = sentinel;
      if (a == b) {
        // self-loop: the sentinel
      } else if (a >= n || b >= n) {
        atomicExch(ctr + C_OVERFLOW, 1ull);
      } else {
        const uint32_t ra = rank[a], rb = rank[b];
        k = ((uint64_t)min(ra, rb) << bits) | max(ra, rb) | ((uint64_t)(sign[i] < 0) << 63);
      }
      akeys[i] = k;
    }
  }
}

// The first key of each run of equal (lo, hi) in the sorted arc keys becomes
// arc `pos` of the CSR: head, sign, tail and signed head.
struct EmitArc {
  const uint64_t* keys;
  uint32_t bits;
  uint32_t* nbr;
  int8_t* sgn;
  uint32_t* asrc;
  uint32_t* nkey;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t flag) const {
    if (!flag) return;
    const uint64_t k = keys[i];
    const uint64_t idmask = (1ull << bits) - 1;
    const uint32_t head = (uint32_t)(k & idmask);
    nbr[pos] = head;
    sgn[pos] = (k >> 63) ? (int8_t)-1 : (int8_t)1;
    asrc[pos] = (uint32_t)((k >> bits) & idmask);
    nkey[pos] = (head << 1) | (uint32_t)(k >> 63);
  }
};

// Out-degree of every tail from the sorted arcs: lanes take consecutive
// arcs, so a warp adds each run of equal tails with one atomic.  With m_dev,
// m is a capacity and *m_dev the arc count.
__global__ void k_fdeg_count(const uint32_t* __restrict__ asrc, uint64_t m,
                             const unsigned long long* __restrict__ m_dev,
                             uint32_t* __restrict__ fdeg) {
  if (m_dev) m = min(m, (uint64_t)*m_dev);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < m;
       base += stride) {
    const uint64_t p = base + lane_id();
    const uint32_t t = p < m ? asrc[p] : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(kFull, t);
    if (p < m && (peers & lanemask_lt()) == 0) atomicAdd(fdeg + t, (uint32_t)__popc(peers));
  }
}

// The merge-model and probe-model bytes of every arc (arc_bytes); m_dev as
// in k_fdeg_count.
__global__ void k_alg_bytes(const uint32_t* __restrict__ asrc, const uint32_t* __restrict__ nbr,
                            uint64_t m, const unsigned long long* __restrict__ m_dev,
                            const uint64_t* __restrict__ off, const uint32_t* __restrict__ fdeg,
                            unsigned long long* __restrict__ ctr) {
  if (m_dev) m = min(m, (uint64_t)*m_dev);
  unsigned long long bytes = 0, probe = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    arc_bytes(i, asrc[i], nbr[i], off, fdeg, bytes, probe);
  bytes = warp_sum(bytes);
  probe = warp_sum(probe);
  if (lane_id() == 0 && bytes) {
    atomicAdd(ctr + C_ALG_BYTES, bytes);
    atomicAdd(ctr + C_PROBE_BYTES, probe);
  }
}

// Vertex bases of a capped batch build, on the device: vbase = exclusive
// prefix of the graphs' id spaces, vbase[G] = vertices of the union (also
// written to C_BATCH_N); a union larger than the capacity n sets C_OVERFLOW.
// One CTA of 1,024 threads, 1,024 graphs per step.
__global__ void __launch_bounds__(1024) k_batch_bases(const unsigned int* __restrict__ space,
                                                      uint32_t G, uint32_t n,
                                                      uint64_t* __restrict__ vbase,
                                                      unsigned long long* __restrict__ ctr) {
  __shared__ uint64_t warp_incl[32];
  __shared__ uint64_t carry;
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < G; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint64_t x = i < G ? space[i] : 0;
    uint64_t v = x;  // inclusive scan within the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(kFull, v, d);
      if (lane >= (uint32_t)d) v += y;
    }
    if (lane == 31) warp_incl[w] = v;
    __syncthreads();
    if (w == 0) {
      uint64_t t = warp_incl[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = __shfl_up_sync(kFull, t, d);
        if (lane >= (uint32_t)d) t += y;
      }
      warp_incl[lane] = t;
    }
    __syncthreads();
    const uint64_t before = carry + (w ? warp_incl[w - 1] : 0) + v - x;
    if (i < G) vbase[i] = before;
    __syncthreads();
    if (threadIdx.x == 1023) carry = before + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    vbase[G] = carry;
    ctr[C_BATCH_N] = carry;
    if (carry > n) ctr[C_OVERFLOW] = 1;
  }
}

// Vertex sort keys of a capped batch build: graph << (32 + dbits) | degree
// << 32 | id, the keys k_vertex_keys and k_batch_vertex_graph make together;
// vertices past the union (vbase[G] <= i < n) take all-ones graph and
// degree bits and so rank last.  A degree wider than dbits sets C_OVERFLOW.
__global__ void k_batch_vertex_keys(const uint32_t* __restrict__ deg, uint32_t n,
                                    const uint64_t* __restrict__ vbase, uint32_t G,
                                    uint64_t per_cta, uint32_t dbits, uint32_t gbits,
                                    uint64_t* __restrict__ vkeys,
                                    unsigned long long* __restrict__ ctr) {
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < n ? begin + per_cta : n;
  if (begin >= end) return;
  const uint64_t nreal = vbase[G];
  const uint64_t pad = ((1ull << (dbits + gbits)) - 1) << 32;
  uint32_t g = begin < nreal ? first_segment(vbase, G, begin) : 0;
  bool over = false;
  for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    if (i >= nreal) {
      vkeys[i] = pad | i;
      continue;
    }
    while (vbase[g + 1] <= i) g++;
    uint64_t d = deg[i];
    if (d >> dbits) {
      over = true;
      d = (1ull << dbits) - 1;
    }
    vkeys[i] = (gbits ? (uint64_t)g << (32 + dbits) : 0ull) | (d << 32) | i;
  }
  if (over) atomicExch(ctr + C_OVERFLOW, 1ull);
}

// UniqueFlag over all m sorted arc keys, the self-loop sentinels (sorted
// last, all ones in the 2 * bits window) excluded: a capped build does not
// know m_valid on the host.
struct UniqueArcFlag {
  const uint64_t* keys;
  uint64_t mask;
  __device__ uint32_t operator()(uint64_t i) const {
    const uint64_t k = keys[i] & mask;
    if (k == mask) return 0u;
    if (i == 0) return 1u;
    return k != (keys[i - 1] & mask) ? 1u : 0u;
  }
};

// Steps 2-6 of the totals path, after the ids (g.n, g.bits, g.m_valid set):
// degrees over the edge copies (sampled on dense graphs), (degree, id) rank
// (graph-major for a batch with vertex bases d_vbase), arc keys of every
// copy, their sort, the first of each run of equal arcs, offsets.  g.ukeys
// stays null.  With `caps` (a batch whose sizes stay on the device) nothing
// is read back: g.n is the vertex capacity, the degree bits and sample shift
// come from caps, and g.m_fwd is the arc capacity (m) with the arc count in
// C_BATCH_MU (g.m_dev).
void build_totals(stc_ctx* c, const EdgeIds& e, const int8_t* d_sign, uint64_t m, DeviceGraph& g,
                  const uint64_t* d_vbase, uint32_t G, const BatchCaps* caps = nullptr) {
  cudaStream_t st = c->stream;
  unsigned long long* ctr = (unsigned long long*)counters(c);
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  g.ukeys = nullptr;
  g.deg = buffer<uint32_t>(c, B_DEG, g.n);
  g.rank = buffer<uint32_t>(c, B_RANK, g.n);
  g.verts = buffer<uint32_t>(c, B_VERTS, g.n);
  g.fdeg = buffer<uint32_t>(c, B_FDEG, g.n);
  const RangePartition ep = range_partition(m, kSortTile, kMaxSortGrid);
  if (g.n) {
    STC_CUDA(cudaMemsetAsync(g.deg, 0, (size_t)g.n * sizeof(uint32_t), st));
    STC_CUDA(cudaMemsetAsync(g.fdeg, 0, (size_t)g.n * sizeof(uint32_t), st));
  }
  if (g.m_valid) {
    // Sample 1 in 2^shift edges once the average degree reaches 8 (2 m / n
    // >= 8): shift = bit width of m / n, less 2, at most 3.  (From degree 16
    // on the 1,024-graph batch counted 6 ms slower and built 17 ms faster;
    // RMAT scale 24 moved by under 0.5 ms either way.)
    const uint64_t ratio = g.m_valid / std::max<uint64_t>(1, g.n);
    const uint32_t bw = bit_width64(ratio);
    g.shift = caps ? caps->shift : bw > 2 ? std::min<uint32_t>(3, bw - 2) : 0;
    k_degree_raw<<<ep.grid, kThreads, 0, st>>>(e, m, g.shift, g.n, g.deg);
    c->launches++;
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 2);

  if (g.n) {
    uint64_t* va = buffer<uint64_t>(c, B_VKEYS_A, g.n);
    uint64_t* vb = buffer<uint64_t>(c, B_VKEYS_B, g.n);
    const int gbits = d_vbase ? (int)bit_width64(G > 1 ? G - 1 : 0) : 0;
    if (caps) {
      g.dbits = caps->dbits;
      if (32 + (int)g.dbits + gbits > 64)
        fail(STC_ERR_LIMIT, "batch too large for the vertex sort key");
      const RangePartition vp = range_partition(g.n, kSortTile, kMaxSortGrid);
      k_batch_vertex_keys<<<vp.grid, kThreads, 0, st>>>(g.deg, g.n, d_vbase, G, vp.per_cta,
                                                        g.dbits, (uint32_t)gbits, va, ctr);
      c->launches++;
    } else {
      k_vertex_keys<<<grid_for(g.n, 4), kThreads, 0, st>>>(g.deg, g.n, va, ctr);
      c->launches++;
      read_counters(c, C_MAX_DEG, 1);
      g.max_deg = (uint32_t)c->h_pinned[C_MAX_DEG];
      g.dbits = bit_width64(g.max_deg);
      if (32 + (int)g.dbits + gbits > 64)
        fail(STC_ERR_LIMIT, "batch too large for the vertex sort key");
      if (gbits) {
        const RangePartition vp = range_partition(g.n, kSortTile, kMaxSortGrid);
        k_batch_vertex_graph<<<vp.grid, kThreads, 0, st>>>(va, g.n, d_vbase, G, vp.per_cta,
                                                           32 + g.dbits);
        c->launches++;
      }
    }
    uint64_t* vs = radix_sort(va, vb, g.n, 32, 32 + (int)g.dbits + gbits, sort_counts, st,
                              &c->launches);
    k_rank<<<grid_for(g.n, 4), kThreads, 0, st>>>(vs, g.n, g.verts, g.rank);
    c->launches++;
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 3);

  g.m_unique = g.m_fwd = 0;
  if (g.m_valid) {
    uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, m);
    uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, m);
    wait_sign(c);  // a host sign array may still be on its way (stc_count)
    k_arc_keys_raw<<<ep.grid, kThreads, 0, st>>>(e, d_sign, m, g.bits, g.n, g.rank, ka, ctr);
    c->launches++;
    uint64_t* sorted = radix_sort(ka, kb, m, 0, 2 * (int)g.bits, sort_counts, st, &c->launches);
    const uint64_t mask = (1ull << (2 * g.bits)) - 1;
    if (caps) {
      const UniqueArcFlag flag{sorted, mask};
      const uint32_t grid = range_reduce_scan(flag, m, sums, st, &c->launches);
      STC_CUDA(cudaMemcpyAsync(ctr + C_BATCH_MU, sums + grid, sizeof(uint64_t),
                               cudaMemcpyDeviceToDevice, st));
      g.m_unique = g.m_fwd = m;
      g.m_dev = ctr + C_BATCH_MU;
      g.nbr = buffer<uint32_t>(c, B_NBR, m + 4);
      g.sgn = buffer<int8_t>(c, B_SGN, m + 4);
      g.asrc = buffer<uint32_t>(c, B_ASRC, m);
      g.nkey = buffer<uint32_t>(c, B_NKEY, m + 8);
      range_apply(flag, EmitArc{sorted, g.bits, g.nbr, g.sgn, g.asrc, g.nkey}, m, sums, st,
                  &c->launches);
    } else {
      // Self-loops sorted last: the first m_valid keys are the real arcs.
      const UniqueFlag flag{sorted, mask};
      const uint32_t grid = range_reduce_scan(flag, g.m_valid, sums, st, &c->launches);
      STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, sums + grid, sizeof(uint64_t),
                               cudaMemcpyDeviceToHost, st));
      STC_CUDA(cudaStreamSynchronize(st));
      g.m_unique = g.m_fwd = c->h_pinned[C_WORK];
      g.nbr = buffer<uint32_t>(c, B_NBR, g.m_fwd + 4);  // + 4: the engine reads whole int4 chunks
      g.sgn = buffer<int8_t>(c, B_SGN, g.m_fwd + 4);
      g.asrc = buffer<uint32_t>(c, B_ASRC, g.m_fwd);
      g.nkey = buffer<uint32_t>(c, B_NKEY, g.m_fwd + 8);
      range_apply(flag, EmitArc{sorted, g.bits, g.nbr, g.sgn, g.asrc, g.nkey}, g.m_valid, sums,
                  st, &c->launches);
    }
    k_fdeg_count<<<grid_for(g.m_fwd, 4), kThreads, 0, st>>>(g.asrc, g.m_fwd, g.m_dev, g.fdeg);
    c->launches++;
  }
  g.off = buffer<uint64_t>(c, B_OFF, (size_t)g.n + 1);
  if (g.n) {
    range_scan(LoadU32{g.fdeg}, EmitOffset{g.off}, g.n, sums, st, &c->launches);
    STC_CUDA(cudaMemcpyAsync(g.off + g.n, sums + range_partition(g.n, kScanTile, kMaxSortGrid).grid,
                             sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  } else {
    STC_CUDA(cudaMemsetAsync(g.off, 0, sizeof(uint64_t), st));
  }
  if (g.m_fwd) {
    k_alg_bytes<<<grid_for(g.m_fwd, 4), kThreads, 0, st>>>(g.asrc, g.nbr, g.m_fwd, g.m_dev, g.off,
                                                           g.fdeg, ctr);
    c->launches++;
  } else {
    g.nbr = buffer<uint32_t>(c, B_NBR, 4);
    g.sgn = buffer<int8_t>(c, B_SGN, 4);
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 4);
}

// ---------------------------------------------------- dense relabel ----
// Counts of totals accept any 32-bit id: an edge list whose largest id
// reaches 2^31 - 1 (where the engine's signed keys and ranks would not fit)
// is relabelled to dense ids first, the index of each id among the list's
// distinct ids.  The relabelling keeps the ids' order, so the graph, its
// (degree, id) order and its counts are those of the original list.

// Both endpoints of every edge as 64-bit sort keys.
__global__ void k_endpoint_keys(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                                uint64_t m, uint64_t* __restrict__ keys) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    keys[2 * i] = u[i];
    keys[2 * i + 1] = v[i];
  }
}

struct DistinctEmit {
  const uint64_t* keys;
  uint32_t* out;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t flag) const {
    if (flag) out[pos] = (uint32_t)keys[i];
  }
};

__device__ __forceinline__ uint32_t dense_id(const uint32_t* __restrict__ ids, uint32_t nd,
                                             uint32_t x) {
  uint32_t lo = 0, hi = nd;  // first index with ids[index] >= x (x is present)
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (ids[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void k_relabel(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                          uint64_t m, const uint32_t* __restrict__ ids, uint32_t nd,
                          uint32_t* __restrict__ ou, uint32_t* __restrict__ ov) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    ou[i] = dense_id(ids, nd, u[i]);
    ov[i] = dense_id(ids, nd, v[i]);
  }
}

// Relabels the m edges at (*src, *dst) to dense ids in context buffers and
// points *src / *dst at them; returns the number of distinct ids.
uint64_t relabel_dense(stc_ctx* c, const uint32_t** src, const uint32_t** dst, uint64_t m) {
  cudaStream_t st = c->stream;
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, 2 * m);
  uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, 2 * m);
  k_endpoint_keys<<<grid_for(m, 4), kThreads, 0, st>>>(*src, *dst, m, ka);
  c->launches++;
  const uint64_t* sorted = radix_sort(ka, kb, 2 * m, 0, 32, sort_counts, st, &c->launches);
  const UniqueFlag flag{sorted, 0xFFFFFFFFull};
  const uint32_t grid = range_reduce_scan(flag, 2 * m, sums, st, &c->launches);
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, sums + grid, sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  const uint64_t nd = c->h_pinned[C_WORK];
  if (nd >= (1ull << 31) - 1)
    fail(STC_ERR_LIMIT, std::to_string(nd) + " distinct vertex ids >= 2^31 - 1");
  uint32_t* ids = buffer<uint32_t>(c, B_DISTINCT, nd);
  range_apply(flag, DistinctEmit{sorted, ids}, 2 * m, sums, st, &c->launches);
  uint32_t* out = buffer<uint32_t>(c, B_RELABEL, 2 * m);
  k_relabel<<<grid_for(m, 4), kThreads, 0, st>>>(*src, *dst, m, ids, (uint32_t)nd, out, out + m);
  c->launches++;
  STC_CUDA(cudaGetLastError());
  *src = out;
  *dst = out + m;
  return nd;
}

}  // namespace

void build_graph(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst, const int8_t* d_sign,
                 uint64_t m, DeviceGraph& g, bool totals) {
  cudaStream_t st = c->stream;
  unsigned long long* ctr = (unsigned long long*)counters(c);
  g = DeviceGraph{};
  g.m_input = m;
  if (m >= (1ull << 32)) fail(STC_ERR_LIMIT, "edge list has 2^32 or more elements");

  // 1. ids: max kept id and self-loops.
  mark(c, 1);
  if (m) {
    k_scan_ids<<<grid_for(m, 4), kThreads, 0, st>>>(d_src, d_dst, m, ctr);
    c->launches++;
  }
  read_counters(c, C_MAX_ID, 2);
  uint64_t max_id = c->h_pinned[C_MAX_ID];
  const uint64_t self = c->h_pinned[C_SELF];
  // Ids (and ranks) stay below 2^31 - 1: the engine keeps a sign in bit 31.
  // Counts of totals relabel larger ids to dense ones; the other paths
  // report results by id and keep the limit.
  if (max_id >= (1ull << 31) - 1) {
    if (!totals) fail(STC_ERR_LIMIT, "vertex id " + std::to_string(max_id) + " >= 2^31 - 1");
    max_id = relabel_dense(c, &d_src, &d_dst, m) - 1;
  }
  g.n = m ? (uint32_t)max_id + 1 : 0;
  g.m_valid = m - self;
  g.bits = std::max<uint32_t>(1, bit_width64(max_id));
  if (totals) {
    build_totals(c, EdgeIds{d_src, d_dst, nullptr, nullptr, 0}, d_sign, m, g, nullptr, 0);
    return;
  }
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);

  // 2. dedup.
  uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, m);
  uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, m);
  g.ukeys = buffer<uint64_t>(c, B_UKEYS, g.m_valid);
  if (g.m_valid) {
    wait_sign(c);
    k_pack_dedup<<<grid_for(m, 4), kThreads, 0, st>>>(d_src, d_dst, d_sign, m, g.bits, ka);
    c->launches++;
    uint64_t* sorted = radix_sort(ka, kb, m, 0, 2 * (int)g.bits, sort_counts, st, &c->launches);
    const uint64_t mask = (1ull << (2 * g.bits)) - 1;
    range_scan(UniqueFlag{sorted, mask}, UniqueEmit{sorted, g.ukeys}, g.m_valid, sums, st,
               &c->launches);
    const uint32_t grid = range_partition(g.m_valid, kScanTile, kMaxSortGrid).grid;
    STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, sums + grid, sizeof(uint64_t),
                             cudaMemcpyDeviceToHost, st));
    STC_CUDA(cudaStreamSynchronize(st));
    g.m_unique = c->h_pinned[C_WORK];
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 2);

  // 3-4. degree and (degree, id) rank.
  g.deg = buffer<uint32_t>(c, B_DEG, g.n);
  g.rank = buffer<uint32_t>(c, B_RANK, g.n);
  g.verts = buffer<uint32_t>(c, B_VERTS, g.n);
  g.fdeg = buffer<uint32_t>(c, B_FDEG, g.n);
  if (g.n) {
    STC_CUDA(cudaMemsetAsync(g.deg, 0, (size_t)g.n * sizeof(uint32_t), st));
    STC_CUDA(cudaMemsetAsync(g.fdeg, 0, (size_t)g.n * sizeof(uint32_t), st));
    if (g.m_unique) {
      k_degree<<<grid_for(g.m_unique, 16), kThreads, 0, st>>>(g.ukeys, g.m_unique, g.bits, g.deg);
      c->launches++;
    }
    uint64_t* va = buffer<uint64_t>(c, B_VKEYS_A, g.n);
    uint64_t* vb = buffer<uint64_t>(c, B_VKEYS_B, g.n);
    k_vertex_keys<<<grid_for(g.n, 4), kThreads, 0, st>>>(g.deg, g.n, va, ctr);
    c->launches++;
    read_counters(c, C_MAX_DEG, 1);
    g.max_deg = (uint32_t)c->h_pinned[C_MAX_DEG];
    uint64_t* vs = radix_sort(va, vb, g.n, 32, 32 + (int)bit_width64(g.max_deg), sort_counts, st,
                              &c->launches);
    k_rank<<<grid_for(g.n, 4), kThreads, 0, st>>>(vs, g.n, g.verts, g.rank);
    c->launches++;
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 3);

  // 5-6. orientation into rank space and the forward CSR.
  g.m_fwd = g.m_unique;
  if (g.m_fwd) {
    k_arc_keys<<<grid_for(g.m_fwd, 4), kThreads, 0, st>>>(g.ukeys, g.m_fwd, g.bits, g.rank, ka,
                                                          g.fdeg);
    c->launches++;
    finish_csr_from_arc_keys(c, g, ka, kb);
  } else {
    g.off = buffer<uint64_t>(c, B_OFF, (size_t)g.n + 1);
    STC_CUDA(cudaMemsetAsync(g.off, 0, ((size_t)g.n + 1) * sizeof(uint64_t), st));
    g.nbr = buffer<uint32_t>(c, B_NBR, 1);
    g.sgn = buffer<int8_t>(c, B_SGN, 1);
  }
  mark(c, 4);
}

void graph_from_forward_csr(stc_ctx* c, uint32_t n, uint64_t m, const uint64_t* d_off,
                            const uint32_t* d_edges, const int8_t* d_signs, const uint32_t* d_rank,
                            DeviceGraph& g) {
  cudaStream_t st = c->stream;
  unsigned long long* ctr = (unsigned long long*)counters(c);
  g = DeviceGraph{};
  g.n = n;
  g.m_input = g.m_valid = g.m_unique = g.m_fwd = m;
  if (m >= (1ull << 32)) fail(STC_ERR_LIMIT, "forward CSR has 2^32 or more edges");
  if (n >= (1u << 31) - 1) fail(STC_ERR_LIMIT, "forward CSR has 2^31 - 1 or more vertices");
  g.bits = std::max<uint32_t>(1, bit_width64(n ? n - 1 : 0));
  g.rank = const_cast<uint32_t*>(d_rank);
  g.fdeg = buffer<uint32_t>(c, B_FDEG, n);
  mark(c, 1);
  mark(c, 2);
  mark(c, 3);
  if (m) {
    uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, m);
    uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, m);
    k_csr_arc_keys<<<kSMs * 8, kThreads, 0, st>>>(d_off, d_edges, d_signs, d_rank, n, g.bits, ka,
                                                  g.fdeg, ctr);
    c->launches++;
    read_counters(c, C_ERROR, 1);
    if (c->h_pinned[C_ERROR]) {
      fail(STC_ERR_INVALID_ARGUMENT,
           "forward CSR has an edge that does not go from lower to higher rank or an id >= n");
    }
    finish_csr_from_arc_keys(c, g, ka, kb);
  } else {
    g.off = buffer<uint64_t>(c, B_OFF, (size_t)n + 1);
    STC_CUDA(cudaMemsetAsync(g.off, 0, ((size_t)n + 1) * sizeof(uint64_t), st));
    g.nbr = buffer<uint32_t>(c, B_NBR, 1);
    g.sgn = buffer<int8_t>(c, B_SGN, 1);
  }
  mark(c, 4);
}

void build_graph_batch(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst,
                       const int8_t* d_sign, uint64_t m, const uint64_t* h_eoff, uint32_t G,
                       DeviceGraph& g, bool totals) {
  cudaStream_t st = c->stream;
  unsigned long long* ctr = (unsigned long long*)counters(c);
  g = DeviceGraph{};
  g.m_input = m;
  g.G = G;
  if (m >= (1ull << 32)) fail(STC_ERR_LIMIT, "batch has 2^32 or more edges");
  uint64_t* d_eoff = buffer<uint64_t>(c, B_BATCH_META, 2ull * (G + 1));
  uint64_t* d_vbase = d_eoff + (G + 1);
  unsigned int* d_space = reinterpret_cast<unsigned int*>(buffer<uint32_t>(c, B_BATCH_SPACE, G));
  STC_CUDA(cudaMemcpyAsync(d_eoff, h_eoff, (G + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  STC_CUDA(cudaMemsetAsync(d_space, 0, G * sizeof(uint32_t), st));

  // 1. id space per graph -> vertex bases of the union.
  mark(c, 1);
  const RangePartition ep = range_partition(m, kSortTile, kMaxSortGrid);
  if (m) {
    k_batch_ids<<<ep.grid, kThreads, 0, st>>>(d_src, d_dst, m, d_eoff, G, ep.per_cta, d_space, ctr);
    c->launches++;
  }
  std::vector<uint32_t> space(G);
  STC_CUDA(cudaMemcpyAsync(space.data(), d_space, G * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  read_counters(c, C_SELF, 1);
  std::vector<uint64_t> vbase(G + 1, 0);
  for (uint32_t i = 0; i < G; i++) vbase[i + 1] = vbase[i] + space[i];
  const uint64_t ntot = vbase[G];
  if (ntot >= (1ull << 31) - 1)
    fail(STC_ERR_LIMIT, "batch has 2^31 - 1 or more vertices in total");
  STC_CUDA(cudaMemcpyAsync(d_vbase, vbase.data(), (G + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice,
                           st));
  g.n = (uint32_t)ntot;
  g.m_valid = m - c->h_pinned[C_SELF];
  g.bits = std::max<uint32_t>(1, bit_width64(ntot ? ntot - 1 : 0));
  g.gbase = d_vbase;
  if (totals) {
    build_totals(c, EdgeIds{d_src, d_dst, d_eoff, d_vbase, G}, d_sign, m, g, d_vbase, G);
    return;
  }
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);

  // 2. dedup over the union.
  uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, m);
  uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, m);
  g.ukeys = buffer<uint64_t>(c, B_UKEYS, g.m_valid);
  if (g.m_valid) {
    k_batch_pack<<<ep.grid, kThreads, 0, st>>>(d_src, d_dst, d_sign, m, d_eoff, d_vbase, G,
                                                ep.per_cta, g.bits, ka);
    c->launches++;
    uint64_t* sorted = radix_sort(ka, kb, m, 0, 2 * (int)g.bits, sort_counts, st, &c->launches);
    const uint64_t mask = (1ull << (2 * g.bits)) - 1;
    range_scan(UniqueFlag{sorted, mask}, UniqueEmit{sorted, g.ukeys}, g.m_valid, sums, st,
               &c->launches);
    const uint32_t grid = range_partition(g.m_valid, kScanTile, kMaxSortGrid).grid;
    STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, sums + grid, sizeof(uint64_t),
                             cudaMemcpyDeviceToHost, st));
    STC_CUDA(cudaStreamSynchronize(st));
    g.m_unique = c->h_pinned[C_WORK];
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 2);

  // 3-4. degree and graph-major (graph, degree, id) rank.
  g.deg = buffer<uint32_t>(c, B_DEG, g.n);
  g.rank = buffer<uint32_t>(c, B_RANK, g.n);
  g.verts = buffer<uint32_t>(c, B_VERTS, g.n);
  g.fdeg = buffer<uint32_t>(c, B_FDEG, g.n);
  if (g.n) {
    STC_CUDA(cudaMemsetAsync(g.deg, 0, (size_t)g.n * sizeof(uint32_t), st));
    STC_CUDA(cudaMemsetAsync(g.fdeg, 0, (size_t)g.n * sizeof(uint32_t), st));
    if (g.m_unique) {
      k_degree<<<grid_for(g.m_unique, 16), kThreads, 0, st>>>(g.ukeys, g.m_unique, g.bits, g.deg);
      c->launches++;
    }
    uint64_t* va = buffer<uint64_t>(c, B_VKEYS_A, g.n);
    uint64_t* vb = buffer<uint64_t>(c, B_VKEYS_B, g.n);
    k_vertex_keys<<<grid_for(g.n, 4), kThreads, 0, st>>>(g.deg, g.n, va, ctr);
    c->launches++;
    read_counters(c, C_MAX_DEG, 1);
    g.max_deg = (uint32_t)c->h_pinned[C_MAX_DEG];
    const int dbits = (int)bit_width64(g.max_deg);
    const int gbits = (int)bit_width64(G > 1 ? G - 1 : 0);
    if (32 + dbits + gbits > 64) fail(STC_ERR_LIMIT, "batch too large for the vertex sort key");
    if (gbits) {
      const RangePartition vp = range_partition(g.n, kSortTile, kMaxSortGrid);
      k_batch_vertex_graph<<<vp.grid, kThreads, 0, st>>>(va, g.n, d_vbase, G, vp.per_cta, 32 + dbits);
      c->launches++;
    }
    uint64_t* vs = radix_sort(va, vb, g.n, 32, 32 + dbits + gbits, sort_counts, st, &c->launches);
    k_rank<<<grid_for(g.n, 4), kThreads, 0, st>>>(vs, g.n, g.verts, g.rank);
    c->launches++;
  }
  STC_CUDA(cudaGetLastError());
  mark(c, 3);

  // 5-6. orientation and the forward CSR (graphs stay contiguous in rank space).
  g.m_fwd = g.m_unique;
  if (g.m_fwd) {
    k_arc_keys<<<grid_for(g.m_fwd, 4), kThreads, 0, st>>>(g.ukeys, g.m_fwd, g.bits, g.rank, ka,
                                                          g.fdeg);
    c->launches++;
    finish_csr_from_arc_keys(c, g, ka, kb);
  } else {
    g.off = buffer<uint64_t>(c, B_OFF, (size_t)g.n + 1);
    STC_CUDA(cudaMemsetAsync(g.off, 0, ((size_t)g.n + 1) * sizeof(uint64_t), st));
    g.nbr = buffer<uint32_t>(c, B_NBR, 4);
    g.sgn = buffer<int8_t>(c, B_SGN, 4);
  }
  mark(c, 4);
}

void build_graph_batch_capped(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst,
                              const int8_t* d_sign, uint64_t m, uint32_t G, const BatchCaps& caps,
                              DeviceGraph& g) {
  cudaStream_t st = c->stream;
  unsigned long long* ctr = (unsigned long long*)counters(c);
  g = DeviceGraph{};
  g.m_input = m;
  g.G = G;
  if (m >= (1ull << 32)) fail(STC_ERR_LIMIT, "batch has 2^32 or more edges");
  if (caps.n == 0 || caps.n >= (1u << 31) - 1 || caps.bits != std::max<uint32_t>(1, bit_width64(caps.n - 1)))
    fail(STC_ERR_INTERNAL, "inconsistent batch capacities");
  if (!c->h_eoff || c->h_eoff_cap < (size_t)G + 1) fail(STC_ERR_INTERNAL, "edge offsets not staged");
  uint64_t* d_eoff = buffer<uint64_t>(c, B_BATCH_META, 2ull * (G + 1));
  uint64_t* d_vbase = d_eoff + (G + 1);
  unsigned int* d_space = reinterpret_cast<unsigned int*>(buffer<uint32_t>(c, B_BATCH_SPACE, G));
  STC_CUDA(cudaMemcpyAsync(d_eoff, c->h_eoff, (G + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice,
                           st));
  STC_CUDA(cudaMemsetAsync(d_space, 0, G * sizeof(uint32_t), st));

  // 1. id space per graph -> vertex bases of the union, on the device.
  mark(c, 1);
  const RangePartition ep = range_partition(m, kSortTile, kMaxSortGrid);
  if (m) {
    k_batch_ids<<<ep.grid, kThreads, 0, st>>>(d_src, d_dst, m, d_eoff, G, ep.per_cta, d_space, ctr);
    c->launches++;
  }
  k_batch_bases<<<1, 1024, 0, st>>>(d_space, G, caps.n, d_vbase, ctr);
  c->launches++;
  STC_CUDA(cudaGetLastError());
  g.n = caps.n;
  g.m_valid = m;
  g.bits = caps.bits;
  g.gbase = d_vbase;
  build_totals(c, EdgeIds{d_src, d_dst, d_eoff, d_vbase, G}, d_sign, m, g, d_vbase, G, &caps);
}

void export_forward_csr(stc_ctx* c, const DeviceGraph& g, stc_forward_csr* out) {
  cudaStream_t st = c->stream;
  const uint32_t n = g.n;
  const uint64_t mu = g.m_unique;
  uint32_t* fdeg_id = buffer<uint32_t>(c, B_EXPORT_FDEG, n);
  uint64_t* off_id = buffer<uint64_t>(c, B_EXPORT_OFF, (size_t)n + 1);
  uint64_t* ka = buffer<uint64_t>(c, B_KEYS_A, mu);
  uint64_t* kb = buffer<uint64_t>(c, B_KEYS_B, mu);
  uint32_t* sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  uint32_t* edges = buffer<uint32_t>(c, B_NBR, mu);
  int8_t* signs = buffer<int8_t>(c, B_SGN, mu);
  if (n) STC_CUDA(cudaMemsetAsync(fdeg_id, 0, (size_t)n * sizeof(uint32_t), st));
  uint64_t* sorted = ka;
  if (mu) {
    k_export_keys<<<grid_for(mu, 4), kThreads, 0, st>>>(g.ukeys, mu, g.bits, g.rank, ka, fdeg_id);
    sorted = radix_sort(ka, kb, mu, 0, 2 * (int)g.bits, sort_counts, st, &c->launches);
  }
  if (n) {
    range_scan(LoadU32{fdeg_id}, EmitOffset{off_id}, n, sums, st, &c->launches);
    STC_CUDA(cudaMemcpyAsync(off_id + n, sums + range_partition(n, kScanTile, kMaxSortGrid).grid,
                             sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  }
  if (mu) {
    k_csr_fill<<<grid_for(mu, 4), kThreads, 0, st>>>(sorted, mu, g.bits, fdeg_id, off_id, edges,
                                                     signs, nullptr, nullptr,
                                                     (unsigned long long*)counters(c));
  }
  STC_CUDA(cudaGetLastError());
  out->n = n;
  out->m = mu;
  out->offsets = (uint64_t*)malloc(((size_t)n + 1) * sizeof(uint64_t));
  out->edges = (uint32_t*)malloc((mu ? mu : 1) * sizeof(uint32_t));
  out->signs = (int8_t*)malloc(mu ? mu : 1);
  out->fdeg = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  out->rank = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  if (!out->offsets || !out->edges || !out->signs || !out->fdeg || !out->rank) {
    stc_free_forward_csr(out);
    fail(STC_ERR_OUT_OF_MEMORY, "host allocation for the forward CSR failed");
  }
  if (n) {
    STC_CUDA(cudaMemcpyAsync(out->offsets, off_id, ((size_t)n + 1) * sizeof(uint64_t),
                             cudaMemcpyDeviceToHost, st));
    STC_CUDA(cudaMemcpyAsync(out->fdeg, fdeg_id, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    STC_CUDA(cudaMemcpyAsync(out->rank, g.rank, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  } else {
    out->offsets[0] = 0;
  }
  if (mu) {
    STC_CUDA(cudaMemcpyAsync(out->edges, edges, mu * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    STC_CUDA(cudaMemcpyAsync(out->signs, signs, mu, cudaMemcpyDeviceToHost, st));
  }
  STC_CUDA(cudaStreamSynchronize(st));
}

}  // namespace stc
