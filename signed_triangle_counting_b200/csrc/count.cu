// Intersection engine: per-type signed triangle counts over the rank-space
// forward CSR.
//
// Reference: count_triangles / merge_intersect / classify
// (MC/tc_serial.cpp:95-170), intersect_signed_ranked
// (MC/tc_merge_sign_enu.cpp:12-44) and the hash probe
// (MC/tc_hash_sign_enu.cpp:125-165), MC = "Signed_TC/Multicore
// Implementations".  In rank space every list is sorted and every head has a
// higher rank than its tail, so for the arc u -> v stored at position k of
// N+(u), the third vertex w of a triangle lies in the suffix
// A' = N+(u)[k+1 ..] and in B = N+(v); the reference's rank filter
// (tc_serial.cpp:126) is implied, and B is only scanned up to max(A').
//
// Work is grouped by source vertex u, in classes of d = |N+(u)|:
//   tiny   2 <= d <= kTinyMax     one thread per vertex, A in registers,
//                                  monotone binary search of A' in B
//   warp   ..  <= kWarpMax        one warp per vertex, N+(u) staged in the
//                                  warp's shared memory (sorted + hash)
//   block  ..  <= kBlockMax       one CTA per vertex (dynamic queue), staged
//   large  ..  <= large cap       one 512-thread CTA per vertex, staged
//   giant  larger                  one CTA per vertex, A read from global
// Inside warp/block classes a warp takes one arc at a time and a 16x16
// dispatch table indexed by (bucket |A'|, bucket |B|) picks the strategy:
//   MERGE   lanes stream B in 16-byte (int4) chunks, locate each chunk in the
//           staged sorted A' and merge the four keys forward
//   HASH    lanes stream B and probe the shared-memory hash of N+(u)
//   SEARCH  lanes take A' elements and binary-search them in B (global)
// Counters: per-lane u64 by number of negative edges, warp shuffle + block
// reduction, one atomic per counter per CTA.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "stc_device.cuh"

namespace stc {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kWarpCap = 128;  // staged capacity of the warp class

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

__device__ __forceinline__ uint32_t size_bucket(uint32_t x) { return min(15u, 32u - __clz(x)); }

// First index i in [0, len) with a[i] >= x (len if none); `a` may point to
// shared or global memory.
__device__ __forceinline__ uint32_t lower_bound(const uint32_t* a, uint32_t len, uint32_t x) {
  uint32_t lo = 0, hi = len;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t x, uint32_t shift) {
  return (x * 0x9E3779B1u) >> shift;
}

// N+(u) as one team sees it: sorted ids and signs (shared or global memory)
// and, when staged, an open-addressing hash of the same list.
struct Staged {
  const uint32_t* a;
  const int8_t* s;
  const uint32_t* hk;  // nullptr: no hash
  const int8_t* hs;
  uint32_t d;
  uint32_t mask;
  uint32_t shift;
};

struct Arc {
  uint32_t k;    // position of v in N+(u)
  uint32_t nuv;  // 1 if the arc u -> v is negative
  const uint32_t* __restrict__ b;
  const int8_t* __restrict__ sb;
  uint32_t blen;
};

__device__ __forceinline__ void arc_hash(const Staged& L, const Arc& A, uint32_t lane,
                                         TypeCounts& tc) {
  const uint32_t alast = L.a[L.d - 1];
  for (uint32_t j = lane; j < A.blen; j += 32) {
    const uint32_t x = A.b[j];
    if (x > alast) break;
    uint32_t h = hash_slot(x, L.shift);
    while (true) {
      const uint32_t key = L.hk[h];
      if (key == x) {
        tc.add(A.nuv + (L.hs[h] < 0) + (A.sb[j] < 0));
        break;
      }
      if (key == kEmpty) break;
      h = (h + 1) & L.mask;
    }
  }
}

__device__ __forceinline__ void arc_search(const Staged& L, const Arc& A, uint32_t lane,
                                           TypeCounts& tc) {
  for (uint32_t i = A.k + 1 + lane; i < L.d; i += 32) {
    const uint32_t x = L.a[i];
    const uint32_t j = lower_bound(A.b, A.blen, x);
    if (j < A.blen && A.b[j] == x) tc.add(A.nuv + (L.s[i] < 0) + (A.sb[j] < 0));
  }
}

__device__ __forceinline__ void merge_one(const Staged& L, const Arc& A, uint32_t a0, uint32_t alen,
                                          uint32_t j, uint32_t x, TypeCounts& tc) {
  const uint32_t p = lower_bound(L.a + a0, alen, x);
  if (p < alen && L.a[a0 + p] == x) tc.add(A.nuv + (L.s[a0 + p] < 0) + (A.sb[j] < 0));
}

__device__ __forceinline__ void arc_merge(const Staged& L, const Arc& A, uint32_t lane,
                                          TypeCounts& tc) {
  const uint32_t a0 = A.k + 1, alen = L.d - a0;
  const uint32_t alast = L.a[L.d - 1];
  // Scalar head up to 16-byte alignment of B, then int4 chunks, then tail.
  const uint32_t mis = (uint32_t)(((uintptr_t)A.b >> 2) & 3);
  const uint32_t head = min((4 - mis) & 3, A.blen);
  if (lane < head) {
    const uint32_t x = A.b[lane];
    if (x <= alast) merge_one(L, A, a0, alen, lane, x, tc);
  }
  const uint32_t nch = (A.blen - head) >> 2;
  const uint4* b4 = reinterpret_cast<const uint4*>(A.b + head);
  for (uint32_t c = lane; c < nch; c += 32) {
    const uint4 q = b4[c];
    if (q.x > alast) break;
    uint32_t p = lower_bound(L.a + a0, alen, q.x);
    const uint32_t jb = head + 4 * c;
    const uint32_t xs[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const uint32_t x = xs[e];
      while (p < alen && L.a[a0 + p] < x) p++;
      if (p < alen && L.a[a0 + p] == x) tc.add(A.nuv + (L.s[a0 + p] < 0) + (A.sb[jb + e] < 0));
    }
  }
  for (uint32_t j = head + 4 * nch + lane; j < A.blen; j += 32) {
    const uint32_t x = A.b[j];
    if (x <= alast) merge_one(L, A, a0, alen, j, x, tc);
  }
}

// One warp processes arc k of the staged list.
__device__ __forceinline__ void process_arc(const Csr& g, const Staged& L, uint32_t k,
                                            const uint8_t (*table)[16], uint32_t lane,
                                            TypeCounts& tc) {
  Arc A;
  A.k = k;
  const uint32_t v = L.a[k];
  A.nuv = L.s[k] < 0;
  const uint64_t vb = g.off[v];
  A.blen = (uint32_t)(g.off[v + 1] - vb);
  if (A.blen == 0) return;
  A.b = g.nbr + vb;
  A.sb = g.sgn + vb;
  const uint32_t alen = L.d - k - 1;
  uint32_t s = table[size_bucket(alen)][size_bucket(A.blen)];
  if (s == STC_STRATEGY_HASH && L.hk == nullptr) s = STC_STRATEGY_MERGE;
  if (s == STC_STRATEGY_HASH)
    arc_hash(L, A, lane, tc);
  else if (s == STC_STRATEGY_SEARCH)
    arc_search(L, A, lane, tc);
  else
    arc_merge(L, A, lane, tc);
}

// Block reduction of the four counters and one atomic per counter.
// Slot C_T0 + k receives type Tk = 3 - (negative edges).
template <int THREADS>
__device__ __forceinline__ void flush_counts(const TypeCounts& tc, unsigned long long* __restrict__ ctr) {
  __shared__ unsigned long long red[THREADS / 32][4];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const unsigned long long v = warp_sum(tc.c[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long s = 0;
    for (int w = 0; w < THREADS / 32; w++) s += red[w][threadIdx.x];
    if (s) atomicAdd(ctr + C_T0 + (3 - threadIdx.x), s);
  }
}

// Per-source counts: reduce the team's per-vertex counters into
// vcounts[4 * id + type].
template <int THREADS>
__device__ __forceinline__ void block_vertex_flush(const TypeCounts& vc, uint32_t u, const Csr& g,
                                                   unsigned long long* __restrict__ vcounts) {
  __shared__ unsigned long long red[THREADS / 32][4];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const unsigned long long v = warp_sum(vc.c[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long s = 0;
    for (int w = 0; w < THREADS / 32; w++) s += red[w][threadIdx.x];
    vcounts[4ull * g.verts[u] + (3 - threadIdx.x)] = s;
  }
  __syncthreads();
}

// ------------------------------------------------------------ classes ----
struct ClassBounds {
  uint32_t tiny_max, warp_max, block_max, large_max;
  __device__ __forceinline__ uint32_t of(uint32_t d) const {
    if (d < 2) return 5;
    if (d <= tiny_max) return 0;
    if (d <= warp_max) return 1;
    if (d <= block_max) return 2;
    if (d <= large_max) return 3;
    return 4;
  }
};
constexpr int kClasses = 5;

__global__ void k_classify_count(const uint64_t* __restrict__ off, uint32_t n, ClassBounds cb,
                                 unsigned long long* __restrict__ ctr) {
  uint32_t cnt[kClasses] = {0, 0, 0, 0, 0};
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t c = cb.of((uint32_t)(off[u + 1] - off[u]));
#pragma unroll
    for (int i = 0; i < kClasses; i++) cnt[i] += c == (uint32_t)i;
  }
#pragma unroll
  for (int i = 0; i < kClasses; i++) {
    const uint32_t s = __reduce_add_sync(kFull, cnt[i]);
    if (lane_id() == 0 && s) atomicAdd(ctr + C_WORK + i, (unsigned long long)s);
  }
}

// Appends each vertex to its class list (order within a class is free: the
// counts are sums of integers).
__global__ void k_classify_fill(const uint64_t* __restrict__ off, uint32_t n, ClassBounds cb,
                                uint32_t* __restrict__ lists, const uint32_t* __restrict__ starts,
                                unsigned long long* __restrict__ cursor) {
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n;
       base += gridDim.x * blockDim.x) {
    const uint32_t u = base + lane_id();
    const uint32_t c = u < n ? cb.of((uint32_t)(off[u + 1] - off[u])) : 5u;
    const unsigned peers = __match_any_sync(kFull, c);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (c < kClasses && lane_id() == leader) pos = (uint32_t)atomicAdd(cursor + c, (unsigned long long)__popc(peers));
    pos = __shfl_sync(kFull, pos, leader) + __popc(peers & lanemask_lt());
    if (c < kClasses) lists[starts[c] + pos] = u;
  }
}

// Tiny class: one thread per vertex, A in registers, B in global memory.
template <int TMAX, bool kVC>
__global__ void __launch_bounds__(256) k_tiny(Csr g, const uint32_t* __restrict__ list, uint32_t cnt,
                                              unsigned long long* __restrict__ ctr,
                                              unsigned long long* __restrict__ vcounts) {
  TypeCounts tc;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += gridDim.x * blockDim.x) {
    const uint32_t u = list[idx];
    const uint64_t ub = g.off[u];
    const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
    uint32_t a[TMAX];
    uint32_t neg[TMAX];
#pragma unroll
    for (int i = 0; i < TMAX; i++) {
      a[i] = i < (int)d ? g.nbr[ub + i] : kEmpty;
      neg[i] = i < (int)d ? (g.sgn[ub + i] < 0) : 0u;
    }
    TypeCounts vc;
#pragma unroll
    for (int k = 0; k < TMAX - 1; k++) {
      if (k + 1 >= (int)d) break;
      const uint64_t vb = g.off[a[k]];
      const uint32_t blen = (uint32_t)(g.off[a[k] + 1] - vb);
      const uint32_t* b = g.nbr + vb;
      uint32_t pos = 0;
#pragma unroll
      for (int i = k + 1; i < TMAX; i++) {
        if (i >= (int)d || pos >= blen) break;
        pos += lower_bound(b + pos, blen - pos, a[i]);
        if (pos < blen && b[pos] == a[i]) {
          const uint32_t t = neg[k] + neg[i] + (g.sgn[vb + pos] < 0);
          if (kVC) vc.add(t); else tc.add(t);
          pos++;
        }
      }
    }
    if (kVC) {
#pragma unroll
      for (int k = 0; k < 4; k++) vcounts[4ull * g.verts[u] + (3 - k)] = vc.c[k];
    }
  }
  if (!kVC) flush_counts<256>(tc, ctr);
}

// Warp class: one warp per vertex, N+(u) staged in the warp's shared memory.
template <bool kVC>
__global__ void __launch_bounds__(256) k_warp(Csr g, const uint32_t* __restrict__ list, uint32_t cnt,
                                              unsigned long long* __restrict__ ctr,
                                              unsigned long long* __restrict__ vcounts,
                                              const uint8_t* __restrict__ gtable) {
  constexpr int kWarps = 8;
  __shared__ uint32_t sa[kWarps][kWarpCap];
  __shared__ uint32_t hk[kWarps][2 * kWarpCap];
  __shared__ int8_t ss[kWarps][kWarpCap];
  __shared__ int8_t hs[kWarps][2 * kWarpCap];
  __shared__ uint8_t table[16][16];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) (&table[0][0])[i] = gtable[i];
  __syncthreads();
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  TypeCounts tc;
  const uint32_t warps = gridDim.x * kWarps;
  for (uint32_t idx = blockIdx.x * kWarps + w; idx < cnt; idx += warps) {
    const uint32_t u = list[idx];
    const uint64_t ub = g.off[u];
    const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
    uint32_t H = 4;
    while (H < 2 * d) H <<= 1;
    const uint32_t shift = 32 - (31 - __clz(H));
    for (uint32_t i = lane; i < H; i += 32) hk[w][i] = kEmpty;
    for (uint32_t i = lane; i < d; i += 32) {
      sa[w][i] = g.nbr[ub + i];
      ss[w][i] = g.sgn[ub + i];
    }
    __syncwarp();
    for (uint32_t i = lane; i < d; i += 32) {
      const uint32_t x = sa[w][i];
      uint32_t h = hash_slot(x, shift);
      while (atomicCAS(&hk[w][h], kEmpty, x) != kEmpty) h = (h + 1) & (H - 1);
      hs[w][h] = ss[w][i];
    }
    __syncwarp();
    Staged L{sa[w], ss[w], hk[w], hs[w], d, H - 1, shift};
    TypeCounts vc;
    for (uint32_t k = 0; k + 1 < d; k++) process_arc(g, L, k, table, lane, kVC ? vc : tc);
    if (kVC) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const unsigned long long s = warp_sum(vc.c[k]);
        if (lane == 0) vcounts[4ull * g.verts[u] + (3 - k)] = s;
      }
    }
    __syncwarp();
  }
  if (!kVC) flush_counts<256>(tc, ctr);
}

// Block classes: one CTA per vertex from a dynamic queue; `cap` is the
// staged capacity (dynamic shared memory: cap ids, cap signs, 2*cap hash
// keys and signs).  With kStaged == false (giant vertices) A is read from
// global memory and HASH falls back to MERGE.
template <int THREADS, bool kStaged, bool kVC>
__global__ void __launch_bounds__(THREADS) k_block(Csr g, const uint32_t* __restrict__ list,
                                                   uint32_t cnt, uint32_t cap,
                                                   unsigned long long* __restrict__ queue,
                                                   unsigned long long* __restrict__ ctr,
                                                   unsigned long long* __restrict__ vcounts,
                                                   const uint8_t* __restrict__ gtable) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* sa = reinterpret_cast<uint32_t*>(smem);
  uint32_t* hk = sa + cap;
  int8_t* ss = reinterpret_cast<int8_t*>(hk + 2 * cap);
  int8_t* hs = ss + cap;
  __shared__ uint8_t table[16][16];
  __shared__ uint32_t s_item;
  for (int i = threadIdx.x; i < 256; i += THREADS) (&table[0][0])[i] = gtable[i];
  constexpr uint32_t kWarps = THREADS / 32;
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  TypeCounts tc;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (uint32_t)atomicAdd(queue, 1ull);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= cnt) break;
    const uint32_t u = list[item];
    const uint64_t ub = g.off[u];
    const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
    Staged L;
    if (kStaged) {
      uint32_t H = 4;
      while (H < 2 * d) H <<= 1;
      const uint32_t shift = 32 - (31 - __clz(H));
      for (uint32_t i = threadIdx.x; i < H; i += THREADS) hk[i] = kEmpty;
      for (uint32_t i = threadIdx.x; i < d; i += THREADS) {
        sa[i] = g.nbr[ub + i];
        ss[i] = g.sgn[ub + i];
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < d; i += THREADS) {
        const uint32_t x = sa[i];
        uint32_t h = hash_slot(x, shift);
        while (atomicCAS(&hk[h], kEmpty, x) != kEmpty) h = (h + 1) & (H - 1);
        hs[h] = ss[i];
      }
      __syncthreads();
      L = Staged{sa, ss, hk, hs, d, H - 1, shift};
    } else {
      L = Staged{g.nbr + ub, g.sgn + ub, nullptr, nullptr, d, 0, 0};
    }
    TypeCounts vc;
    for (uint32_t k = w; k + 1 < d; k += kWarps) process_arc(g, L, k, table, lane, kVC ? vc : tc);
    if (kVC) block_vertex_flush<THREADS>(vc, u, g, vcounts);
  }
  if (!kVC) flush_counts<THREADS>(tc, ctr);
}

// Fixed degree-threshold dispatch: SEARCH when B is at least 16x longer than
// A', MERGE when both are short, HASH otherwise.
void fixed_table(uint8_t t[16][16]) {
  for (int a = 0; a < 16; a++)
    for (int b = 0; b < 16; b++) {
      uint8_t s = STC_STRATEGY_HASH;
      if (b >= a + 4) s = STC_STRATEGY_SEARCH;
      else if (a <= 3 && b <= 5) s = STC_STRATEGY_MERGE;
      t[a][b] = s;
    }
}

}  // namespace

void count_triangles(stc_ctx* c, const DeviceGraph& g, const CountConfig& cfg) {
  if (g.n == 0 || g.m_fwd == 0) return;
  cudaStream_t st = c->stream;
  Csr csr{g.off, g.nbr, g.sgn, g.verts, g.n};
  unsigned long long* ctr = (unsigned long long*)counters(c);
  const bool vc = cfg.vertex_counts != nullptr;
  unsigned long long* vcounts = (unsigned long long*)cfg.vertex_counts;

  // Dispatch table.
  uint8_t table[16][16];
  if (cfg.strategy == STC_STRATEGY_AUTO) {
    fixed_table(table);
  } else {
    memset(table, (int)cfg.strategy, sizeof(table));
  }
  uint8_t* d_table = buffer<uint8_t>(c, B_WORK2, 256);
  STC_CUDA(cudaMemcpyAsync(d_table, table, 256, cudaMemcpyHostToDevice, st));

  // Vertex classes (a forced strategy disables the tiny class, which only
  // implements the search form).
  ClassBounds cb{cfg.strategy == STC_STRATEGY_AUTO || cfg.strategy == STC_STRATEGY_SEARCH ? 8u : 1u,
                 kWarpCap, 1024u, 8192u};
  k_classify_count<<<kSMs * 4, 256, 0, st>>>(g.off, g.n, cb, ctr);
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, counters(c) + C_WORK, kClasses * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  uint32_t counts[kClasses], starts[kClasses + 1];
  starts[0] = 0;
  for (int i = 0; i < kClasses; i++) {
    counts[i] = (uint32_t)c->h_pinned[C_WORK + i];
    starts[i + 1] = starts[i] + counts[i];
  }
  uint32_t* lists = buffer<uint32_t>(c, B_WORK, (size_t)starts[kClasses] + 8);
  uint32_t* d_starts = lists + starts[kClasses];
  STC_CUDA(cudaMemcpyAsync(d_starts, starts, kClasses * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  // Cursors for the fill and the dynamic queues live in C_WORK + 8 ...
  STC_CUDA(cudaMemsetAsync(counters(c) + C_WORK, 0, 8 * sizeof(uint64_t), st));
  k_classify_fill<<<kSMs * 4, 256, 0, st>>>(g.off, g.n, cb, lists, d_starts, ctr + C_WORK);
  STC_CUDA(cudaMemsetAsync(counters(c) + C_WORK, 0, 8 * sizeof(uint64_t), st));
  c->launches += 2;

  if (counts[0]) {
    const uint32_t grid = std::min<uint32_t>((counts[0] + 255) / 256, kSMs * 8);
    if (vc) k_tiny<8, true><<<grid, 256, 0, st>>>(csr, lists + starts[0], counts[0], ctr, vcounts);
    else k_tiny<8, false><<<grid, 256, 0, st>>>(csr, lists + starts[0], counts[0], ctr, vcounts);
    c->launches++;
  }
  if (counts[1]) {
    const uint32_t grid = std::min<uint32_t>((counts[1] + 7) / 8, kSMs * 8);
    if (vc) k_warp<true><<<grid, 256, 0, st>>>(csr, lists + starts[1], counts[1], ctr, vcounts, d_table);
    else k_warp<false><<<grid, 256, 0, st>>>(csr, lists + starts[1], counts[1], ctr, vcounts, d_table);
    c->launches++;
  }
  if (counts[2]) {
    const uint32_t cap = cb.block_max;
    const size_t smem = (size_t)cap * 15;
    const uint32_t grid = std::min<uint32_t>(counts[2], kSMs * 8);
    auto kern = vc ? k_block<256, true, true> : k_block<256, true, false>;
    kern<<<grid, 256, smem, st>>>(csr, lists + starts[2], counts[2], cap, ctr + C_WORK + 0, ctr,
                                  vcounts, d_table);
    c->launches++;
  }
  if (counts[3]) {
    const uint32_t cap = cb.large_max;
    const size_t smem = (size_t)cap * 15;
    auto kern = vc ? k_block<512, true, true> : k_block<512, true, false>;
    STC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t grid = std::min<uint32_t>(counts[3], kSMs);
    kern<<<grid, 512, smem, st>>>(csr, lists + starts[3], counts[3], cap, ctr + C_WORK + 1, ctr,
                                  vcounts, d_table);
    c->launches++;
  }
  if (counts[4]) {
    auto kern = vc ? k_block<512, false, true> : k_block<512, false, false>;
    const uint32_t grid = std::min<uint32_t>(counts[4], kSMs);
    kern<<<grid, 512, 0, st>>>(csr, lists + starts[4], counts[4], 0, ctr + C_WORK + 2, ctr, vcounts,
                               d_table);
    c->launches++;
  }
  STC_CUDA(cudaGetLastError());
}

}  // namespace stc
