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
// (tc_serial.cpp:126) is implied.
//
// Work is grouped by source vertex u, in classes of d = |N+(u)|:
//   tiny   2 <= d <= 8        one thread per vertex, A in registers,
//                             monotone binary search of A' in B
//   warp   d <= 128           one warp per vertex     } N+(u) staged in
//   block  d <= 1024          one CTA per vertex      } shared memory
//   large  d <= 4096          one 512-thread CTA      }
//   giant  larger             one CTA per vertex, A read from global memory
// A 16x16 dispatch table per class (warp, block, large, giant) indexed by
// (bucket |A'|, bucket |B|) picks each arc's strategy:
//   HASH    B is streamed and every element is looked up in a shared-memory
//           hash of N+(u) whose keys carry the sign, so one 8-byte bucket
//           read answers membership and the A' sign together
//   MERGE   B is streamed and each 16-byte chunk is located in the staged
//           sorted A' by one binary search, its four keys merged forward
//   SEARCH  a warp takes the arc: each lane holds one pivot of B, an A'
//           element finds its segment with five shuffles and is searched in
//           that short segment of B
// HASH and MERGE arcs of one vertex form a single stream of aligned int4
// chunks (prefix sums over the arcs' chunk counts, a per-thread arc cursor),
// so every lane stays busy across arc boundaries and several loads stay in
// flight per thread.  Counters: per-thread packed 16-bit fields by number of
// negative edges, widened into u64 per vertex, then warp shuffle + block
// reduction and one atomic per counter per CTA.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "internal.h"
#include "radix_sort.cuh"
#include "stc_device.cuh"

namespace stc {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kTinyMax = 8;
constexpr uint32_t kWarpCap = 128;    // staged capacity of the warp class
constexpr uint32_t kBlockCap = 1024;  // ... of the block class
constexpr uint32_t kLargeCap = 4096;  // ... of the large class
constexpr int kStreamUnroll = 2;      // int4 chunks in flight per thread
// Device error word value: a list exceeded its staged shared-memory capacity
// (the kernel skipped it instead of overrunning).
constexpr unsigned long long kErrStageCapacity = 3;

struct Csr {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ nbr;  // padded by 4 entries for whole int4 chunks
  const int8_t* __restrict__ sgn;
  const uint32_t* __restrict__ verts;  // rank -> id (per-source counts only)
  uint32_t n;
  // Sign-split heads (same offsets, padded likewise) and positives per
  // vertex; null unless a count uses STC_STRATEGY_SPLIT.
  const uint32_t* __restrict__ nbr_split = nullptr;
  const uint32_t* __restrict__ psplit = nullptr;
  // Heads with their signs, id << 1 | negative (same offsets, padded
  // likewise): what the head side streams, one 16-byte load per chunk.
  const uint32_t* __restrict__ nkey = nullptr;
};

// Per-thread type counters indexed by the number of negative edges.
struct TypeCounts {
  unsigned long long c[4] = {0, 0, 0, 0};
  __device__ __forceinline__ void add(uint32_t neg) {
    c[0] += neg == 0;
    c[1] += neg == 1;
    c[2] += neg == 2;
    c[3] += neg == 3;
  }
};

// Four 16-bit counters packed in one word: one add per triangle; widened
// into TypeCounts before any field can reach 2^16.
struct PackedCounts {
  unsigned long long w = 0;
  __device__ __forceinline__ void add(uint32_t neg) { w += 1ull << (16 * neg); }
  __device__ __forceinline__ void add_if(bool hit, uint32_t neg) {
    w += (unsigned long long)hit << (16 * neg);
  }
  __device__ __forceinline__ void drain(TypeCounts& tc) {
    tc.c[0] += w & 0xFFFF;
    tc.c[1] += (w >> 16) & 0xFFFF;
    tc.c[2] += (w >> 32) & 0xFFFF;
    tc.c[3] += w >> 48;
    w = 0;
  }
};

// Four 8-bit counters packed in one 32-bit word, for the streamed chunks:
// one 32-bit shift and add per triangle; widened into TypeCounts before any
// field can reach 2^8.
struct PackedCounts8 {
  uint32_t w = 0;
  __device__ __forceinline__ void add(uint32_t neg) { w += 1u << (8 * neg); }
  // Branch-free: adds nothing unless `hit`; neg <= 3 either way.
  __device__ __forceinline__ void add_if(bool hit, uint32_t neg) { w += (uint32_t)hit << (8 * neg); }
  __device__ __forceinline__ void drain(TypeCounts& tc) {
    tc.c[0] += w & 0xFFu;
    tc.c[1] += (w >> 8) & 0xFFu;
    tc.c[2] += (w >> 16) & 0xFFu;
    tc.c[3] += w >> 24;
    w = 0;
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

// Multiplicative hash: the top bits of x * an odd constant.
// It hashes 2x, so that a signed key 2x | sign hashes by clearing its sign
// bit (hash_slot_k2) without a shift.
__device__ __forceinline__ uint32_t hash_slot(uint32_t x, uint32_t shift) {
  return ((x << 1) * 0x85EBCA77u) >> shift;
}
__device__ __forceinline__ uint32_t hash_slot_k2(uint32_t k2, uint32_t shift) {
  return (k2 * 0x85EBCA77u) >> shift;
}


// SEARCH for one arc by one warp: each lane holds the pivot B[lane * step];
// an A' element (a[i], i in [i0, d)) finds its segment with five shuffles and
// is searched inside that short segment of B, so a lookup costs about one
// memory latency instead of log2 |B| dependent loads.
template <class Counts>
__device__ __forceinline__ void arc_search(const uint32_t* a, const int8_t* s, uint32_t i0,
                                           uint32_t d, uint32_t nuv, const uint32_t* __restrict__ b,
                                           const int8_t* __restrict__ sb, uint32_t blen,
                                           uint32_t lane, Counts& cnt) {
  const uint32_t step = (blen + 31) >> 5;
  const uint32_t piv = b[min(lane * step, blen - 1)];
  for (uint32_t base = i0; base < d; base += 32) {
    const uint32_t i = base + lane;
    const uint32_t x = i < d ? a[i] : kEmpty;
    uint32_t seg = 0;
#pragma unroll
    for (uint32_t bit = 16; bit; bit >>= 1) {
      const uint32_t p = __shfl_sync(kFull, piv, seg + bit);
      if ((seg + bit) * step < blen && p <= x) seg += bit;
    }
    if (i >= d) continue;
    const uint32_t lo = seg * step;
    const uint32_t j = lo + lower_bound(b + lo, min(step, blen - lo), x);
    if (j < blen && b[j] == x) cnt.add(nuv + (s[i] < 0) + (sb[j] < 0));
  }
}

// MERGE for one arc by one warp over B streamed in int4 chunks (giant lists,
// whose A stays in global memory).
template <class Counts>
__device__ __forceinline__ void arc_merge_global(const uint32_t* a, const int8_t* s, uint32_t a0,
                                                 uint32_t d, uint32_t nuv,
                                                 const uint32_t* __restrict__ b,
                                                 const int8_t* __restrict__ sb, uint32_t blen,
                                                 uint32_t lane, Counts& tc) {
  const uint32_t alen = d - a0;
  const uint32_t alast = a[d - 1];
  for (uint32_t base = 0; base < blen; base += 128) {
    const uint32_t j0 = base + 4 * lane;
    if (__shfl_sync(kFull, j0 < blen ? b[j0] : kEmpty, 0) > alast) return;
    if (j0 >= blen) continue;
    uint32_t p = lower_bound(a + a0, alen, b[j0]);
    for (uint32_t j = j0; j < min(j0 + 4, blen); j++) {
      const uint32_t x = b[j];
      while (p < alen && a[a0 + p] < x) p++;
      if (p < alen && a[a0 + p] == x) tc.add(nuv + (s[a0 + p] < 0) + (sb[j] < 0));
    }
  }
}

// ---------------------------------------------------------- staging ----
// Strategy codes in the per-arc table: STC_STRATEGY_MERGE / _HASH / _SEARCH,
// or kNoArc for the last arc of a list (empty A') and arcs with empty B.
constexpr uint8_t kNoArc = 0xFF;
// Hash keys are id << 1 | (the A' edge is negative).  Ids stay below
// 2^31 - 2, so a key is at most 0xFFFFFFFB: it never equals kEmpty, and no
// key matches kNoId, the id that pads the entries of a chunk outside its arc.
// A query x matches key w exactly when w - 2x is 0 or 1, and that difference
// is the A' sign.
constexpr uint32_t kNoId = 0x7FFFFFFEu;

// Shared-memory image of one staged list of capacity `cap` with `nb` hash
// buckets: the hash (two 32-bit keys per 8-byte bucket), the sorted ids,
// each arc's B extent [lo, hi) as element indices of the CSR, the first
// negative head of a SPLIT arc's B in the split copy, the chunk prefix
// sums, then the byte arrays (list signs, arc strategies).
struct StageMem {
  uint32_t* hk;
  uint32_t* a;
  uint32_t* lo;
  uint32_t* hi;
  uint32_t* sp;
  uint32_t* pre;
  int8_t* s;
  uint8_t* st;
  __host__ __device__ static constexpr size_t bytes(uint32_t cap, uint32_t nb) {
    return 8ull * nb + 22ull * cap + 4;
  }
  __device__ static StageMem carve(unsigned char* p, uint32_t cap, uint32_t nb) {
    StageMem m;
    uint32_t* w = reinterpret_cast<uint32_t*>(p);
    m.hk = w;
    w += 2 * nb;
    m.a = w;
    w += cap;
    m.lo = w;
    w += cap;
    m.hi = w;
    w += cap;
    m.sp = w;
    w += cap;
    m.pre = w;
    w += cap + 1;
    int8_t* b = reinterpret_cast<int8_t*>(w);
    m.s = b;
    b += cap;
    m.st = reinterpret_cast<uint8_t*>(b);
    return m;
  }
};

// Hash geometry for a list of length d: next_pow2(hf d) buckets of two keys
// (hf = 4: load <= 1/8), at most `nb_cap` buckets.
struct Geo {
  uint32_t nb, shift;
  __device__ static Geo of(uint32_t d, uint32_t nb_cap, uint32_t hf) {
    Geo g;
    g.nb = 4;
    while (g.nb < hf * d && g.nb < nb_cap) g.nb <<= 1;
    g.shift = 32 - (31 - __clz(g.nb));
    return g;
  }
};

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Stages N+(u) (d entries at ub) for a team of TS threads (index t): clears
// the hash, copies ids and signs, fetches every arc's B extent, then fills
// the hash and picks each arc's strategy from the table.
template <int TS, class Sync>
__device__ __forceinline__ void stage(const Csr& g, uint64_t ub, uint32_t d, uint32_t t,
                                      const StageMem& m, const Geo& geo,
                                      const uint8_t (*table)[16], Sync sync) {
  for (uint32_t i = t; i < 2 * geo.nb; i += TS) m.hk[i] = kEmpty;
  for (uint32_t i = t; i < d; i += TS) {
    const uint32_t v = g.nbr[ub + i];
    m.a[i] = v;
    m.s[i] = g.sgn[ub + i];
    m.lo[i] = (uint32_t)g.off[v];
    m.hi[i] = (uint32_t)g.off[v + 1];
  }
  sync();
  for (uint32_t i = t; i < d; i += TS) {
    const uint32_t x = m.a[i];
    const uint32_t key = (x << 1) | (uint32_t)(m.s[i] < 0);
    uint32_t b = hash_slot(x, geo.shift);
    while (atomicCAS(&m.hk[2 * b], kEmpty, key) != kEmpty &&
           atomicCAS(&m.hk[2 * b + 1], kEmpty, key) != kEmpty)
      b = (b + 1) & (geo.nb - 1);
    const uint32_t blen = m.hi[i] - m.lo[i];
    uint8_t st = (i + 1 < d && blen) ? table[size_bucket(d - i - 1)][size_bucket(blen)] : kNoArc;
    if (st == STC_STRATEGY_HEAD) st = kNoArc;  // counted by the head-side pass
    m.st[i] = st;
    if (st == STC_STRATEGY_SPLIT) m.sp[i] = m.lo[i] + g.psplit[x];
  }
  sync();
}

// Exact lookup of x from its home bucket on: 0 if x is not in the hash,
// else 1 | (the key's sign flag << 1).
__device__ __noinline__ uint32_t probe_rest(const uint32_t* hk, uint32_t nb, uint32_t shift,
                                            uint32_t x) {
  const uint32_t q = x << 1;
  uint32_t b = hash_slot(x, shift);
  while (true) {
    const uint2 w = *reinterpret_cast<const uint2*>(hk + 2 * b);
    const uint32_t d0 = w.x - q, d1 = w.y - q;
    if (d0 < 2) return 1u | (d0 << 1);
    if (d1 < 2) return 1u | (d1 << 1);
    if (w.y == kEmpty) return 0;
    b = (b + 1) & (nb - 1);
  }
}

// Chunks of arc i's streamed extent: aligned groups of 4 entries (16
// bytes), or of 8 entries (32 bytes) with kWide (the head side's stream).
template <bool kWide = false>
__device__ __forceinline__ uint32_t arc_chunks(const StageMem& m, uint32_t i) {
  const uint8_t st = m.st[i];
  if (st != STC_STRATEGY_HASH && st != STC_STRATEGY_MERGE && st != STC_STRATEGY_SPLIT) return 0;
  return kWide ? ((m.hi[i] + 7) >> 3) - (m.lo[i] >> 3) : ((m.hi[i] + 3) >> 2) - (m.lo[i] >> 2);
}

// pre[i] = chunks of the streamed arcs before arc i; pre[d] = total.
template <bool kWide = false>
__device__ __forceinline__ void warp_chunk_scan(const StageMem& m, uint32_t d, uint32_t lane) {
  uint32_t carry = 0;
  for (uint32_t r = 0; r < d; r += 32) {
    const uint32_t i = r + lane;
    const uint32_t c = i < d ? arc_chunks<kWide>(m, i) : 0;
    const uint32_t inc = warp_inclusive_scan(c);
    if (i < d) m.pre[i] = carry + inc - c;
    carry += __shfl_sync(kFull, inc, 31);
  }
  if (lane == 0) m.pre[d] = carry;
  __syncwarp();
}

template <int THREADS, bool kWide = false>
__device__ __forceinline__ void block_chunk_scan(const StageMem& m, uint32_t d, uint32_t* tmp) {
  uint32_t carry = 0;
  for (uint32_t r = 0; r < d; r += THREADS) {
    const uint32_t i = r + threadIdx.x;
    const uint32_t c = i < d ? arc_chunks<kWide>(m, i) : 0;
    uint32_t total;
    const uint32_t excl = block_exclusive_scan<THREADS>(c, tmp, total);
    if (i < d) m.pre[i] = carry + excl;
    carry += total;
  }
  if (threadIdx.x == 0) m.pre[d] = carry;
  __syncthreads();
}

__device__ __forceinline__ uint32_t pick4(const uint4& q, uint32_t e) {
  const uint32_t lo = (e & 1) ? q.y : q.x;
  const uint32_t hi = (e & 1) ? q.w : q.z;
  return (e & 2) ? hi : lo;
}

// Mask of the entries of int4 chunk ci (elements 4 ci .. 4 ci + 3) that lie
// inside the arc's extent [lo, hi).
__device__ __forceinline__ uint32_t chunk_mask(uint32_t ci, uint32_t lo, uint32_t hi) {
  const uint32_t g0 = 4 * ci;
  const uint32_t first = lo > g0 ? lo - g0 : 0;
  const uint32_t last = min(hi - g0, 4u);
  return ((1u << last) - 1) & ~((1u << first) - 1);
}

// Chunk ci of an arc's B: from the sorted heads with their sign bytes, or,
// for a SPLIT arc, from the sign-split copy, where an element is negative
// exactly when its index is at least `sp` (the sign word is synthesised in
// the layout of the sign bytes: bit 8 e + 7 for element e).
__device__ __forceinline__ void load_chunk(const Csr& g, uint32_t ci, uint32_t st, uint32_t sp,
                                           uint4& q, uint32_t& sw) {
  if (st == STC_STRATEGY_SPLIT) {
    q = reinterpret_cast<const uint4*>(g.nbr_split)[ci];
    const uint32_t g0 = 4 * ci;
    sw = ((uint32_t)(g0 >= sp) << 7) | ((uint32_t)(g0 + 1 >= sp) << 15) |
         ((uint32_t)(g0 + 2 >= sp) << 23) | ((uint32_t)(g0 + 3 >= sp) << 31);
  } else {
    q = reinterpret_cast<const uint4*>(g.nbr)[ci];
    sw = reinterpret_cast<const uint32_t*>(g.sgn)[ci];
  }
}

// One int4 chunk of B for arc k of a staged list: four ids q, their four sign
// bytes sw, and the mask vm (non-zero) of the ids inside the arc.  HASH looks
// every id up in the staged hash (one 8-byte bucket read gives membership and
// the A' sign): ids outside the arc are replaced by kNoId, which matches no
// key, and the rare id whose home bucket is full without a match is looked up
// again past it, once per chunk.  MERGE locates the chunk in the sorted
// A' = a[k+1 ..) by one binary search and merges its ascending ids forward.
// At most four adds per chunk reach any one field of `pc`.  The HASH
// lookups are branch-free: with a few percent of ids hitting, some lane of a
// warp hits at almost every step, so a branch per hit would diverge at
// almost every step.
template <class PC>
__device__ __forceinline__ void process_chunk(const StageMem& m, uint32_t d, const Geo& geo,
                                              const uint4& q, uint32_t sw, uint32_t vm, uint32_t k,
                                              uint32_t nuv, uint32_t st, PC& pc) {
  if (st != STC_STRATEGY_MERGE) {  // HASH or SPLIT
    uint4 x4 = q;
    if (vm != 0xFu) {
      x4.x = (vm & 1u) ? x4.x : kNoId;
      x4.y = (vm & 2u) ? x4.y : kNoId;
      x4.z = (vm & 4u) ? x4.z : kNoId;
      x4.w = (vm & 8u) ? x4.w : kNoId;
    }
    bool again = false;
#pragma unroll
    for (uint32_t e = 0; e < 4; e++) {
      const uint32_t x = pick4(x4, e);
      const uint2 w = *reinterpret_cast<const uint2*>(m.hk + 2 * hash_slot(x, geo.shift));
      const uint32_t d0 = w.x - 2 * x, d1 = w.y - 2 * x;
      const bool hit = d0 < 2 || d1 < 2;
      again |= !hit && w.y != kEmpty;
      pc.add_if(hit, nuv + (d0 < 2 ? d0 : d1 & 1u) + ((sw >> (8 * e + 7)) & 1u));
    }
    if (again) {
#pragma unroll 1
      for (uint32_t e = 0; e < 4; e++) {
        const uint32_t x = pick4(x4, e);
        const uint2 w = *reinterpret_cast<const uint2*>(m.hk + 2 * hash_slot(x, geo.shift));
        if (w.x - 2 * x < 2 || w.y - 2 * x < 2 || w.y == kEmpty) continue;  // settled above
        const uint32_t r = probe_rest(m.hk, geo.nb, geo.shift, x);
        if (r) pc.add(nuv + (r >> 1) + ((sw >> (8 * e + 7)) & 1u));
      }
    }
  } else {  // MERGE
    const uint32_t a0 = k + 1, alen = d - a0;
    const uint32_t* a = m.a + a0;
    const uint32_t e0 = __ffs(vm) - 1;
    uint32_t p = lower_bound(a, alen, pick4(q, e0));
    for (uint32_t e = e0; e < 4 && ((vm >> e) & 1u); e++) {
      const uint32_t x = pick4(q, e);
      while (p < alen && a[p] < x) p++;
      if (p < alen && a[p] == x) pc.add(nuv + (m.s[a0 + p] < 0) + ((sw >> (8 * e + 7)) & 1u));
    }
  }
}

// HASH for an aligned chunk of eight signed heads (id << 1 | negative, the
// head side's stream; a, then b), vm its 8-bit mask: as process_chunk's HASH
// path, with each entry's sign taken from its own low bit instead of a
// separate sign word, one mask test and one overflow test per eight keys.
template <class PC>
__device__ __forceinline__ void process_keyed_chunk8(const StageMem& m, const Geo& geo, uint4 a,
                                                     uint4 b, uint32_t vm, uint32_t nuv,
                                                     PC& pc) {
  constexpr uint32_t kNoKey = kNoId << 1;
  if (vm != 0xFFu) {
    a.x = (vm & 1u) ? a.x : kNoKey;
    a.y = (vm & 2u) ? a.y : kNoKey;
    a.z = (vm & 4u) ? a.z : kNoKey;
    a.w = (vm & 8u) ? a.w : kNoKey;
    b.x = (vm & 16u) ? b.x : kNoKey;
    b.y = (vm & 32u) ? b.y : kNoKey;
    b.z = (vm & 64u) ? b.z : kNoKey;
    b.w = (vm & 128u) ? b.w : kNoKey;
  }
  bool again = false;
#pragma unroll
  for (uint32_t e = 0; e < 8; e++) {
    const uint32_t key = e < 4 ? pick4(a, e) : pick4(b, e - 4);
    const uint32_t k2 = key & ~1u;  // 2 x
    const uint2 w = *reinterpret_cast<const uint2*>(m.hk + 2 * hash_slot_k2(k2, geo.shift));
    const uint32_t d0 = w.x - k2, d1 = w.y - k2;
    const bool hit = d0 < 2 || d1 < 2;
    again |= !hit && w.y != kEmpty;
    pc.add_if(hit, nuv + (d0 < 2 ? d0 : d1 & 1u) + (key & 1u));
  }
  if (again) {
#pragma unroll 1
    for (uint32_t e = 0; e < 8; e++) {
      const uint32_t key = e < 4 ? pick4(a, e) : pick4(b, e - 4), x = key >> 1;
      const uint2 w = *reinterpret_cast<const uint2*>(m.hk + 2 * hash_slot(x, geo.shift));
      if (w.x - (key & ~1u) < 2 || w.y - (key & ~1u) < 2 || w.y == kEmpty) continue;
      const uint32_t r = probe_rest(m.hk, geo.nb, geo.shift, x);
      if (r) pc.add(nuv + (r >> 1) + (key & 1u));
    }
  }
}

// The head side's stream: the staged in-arcs' A' extents of signed heads
// (g.nkey) as one sequence of aligned 8-entry (32-byte) chunks, shared out
// as in stream_pass (warp shares, lanes on consecutive chunks, the last
// eighth claimed from `next`).  A lane loads a chunk with two 16-byte
// loads, UK chunks per round, and the cursor, mask and branch work per
// chunk is spread over eight keys instead of four.  pre[] counts 8-entry
// chunks (block_chunk_scan / warp_chunk_scan with kWide).
template <int UK>
__device__ __forceinline__ void stream_pass_keyed(const Csr& g, const StageMem& m, uint32_t d,
                                                  uint32_t warp, uint32_t warps, uint32_t lane,
                                                  const Geo& geo, TypeCounts& tc,
                                                  uint32_t* next) {
  const uint32_t total = m.pre[d];
  const uint32_t fixed = next ? total - total / 8 : total;
  const uint32_t per = (fixed + warps - 1) / warps;
  uint32_t seg_begin = min(fixed, warp * per), seg_end = min(fixed, seg_begin + per);
  uint32_t k = 0, pk, pk1, cb, mf, ml, anuv;
  auto enter = [&](uint32_t kk) {
    pk = m.pre[kk];
    pk1 = m.pre[kk + 1];
    const uint32_t alo = m.lo[kk], ahi = m.hi[kk];
    cb = (alo >> 3) - pk;
    mf = (0xFFu << (alo & 7u)) & 0xFFu;
    ml = 0xFFu >> (7u - ((ahi - 1u) & 7u));
    anuv = m.s[kk] < 0;
  };
  // 8-bit fields: at most 8 UK adds per field per round.
  constexpr uint32_t kDrainRounds = 255 / (8 * UK);
  constexpr uint32_t kClaim = 32 * UK;  // 8-entry chunks a warp claims at a time (one round)
  const uint4* src = reinterpret_cast<const uint4*>(g.nkey);
  PackedCounts8 p8;
  uint32_t rounds = 0;
  while (true) {
    if (seg_begin < seg_end) {
      {
        uint32_t lo_k = k, hi_k = d;
        const uint32_t c0 = seg_begin + lane;
        while (hi_k - lo_k > 1) {
          const uint32_t mid = (lo_k + hi_k) >> 1;
          if (m.pre[mid] <= c0) lo_k = mid; else hi_k = mid;
        }
        k = lo_k;
        enter(k);
      }
      for (uint32_t base = seg_begin; base < seg_end; base += 32 * UK) {
        uint4 qa[UK], qb[UK];
        uint32_t vm[UK], snuv[UK];
#pragma unroll
        for (int u = 0; u < UK; u++) {
          const uint32_t c = base + 32 * u + lane;
          vm[u] = 0;
          if (c < seg_end) {
            if (c >= pk1) {
              do {
                k++;
              } while (m.pre[k + 1] <= c);
              enter(k);
            }
            const uint32_t ci = cb + c;
            qa[u] = src[2 * ci];
            qb[u] = src[2 * ci + 1];
            vm[u] = (c == pk ? mf : 0xFFu) & (c + 1 == pk1 ? ml : 0xFFu);
            snuv[u] = anuv;
          }
        }
#pragma unroll
        for (int u = 0; u < UK; u++)
          if (vm[u]) process_keyed_chunk8(m, geo, qa[u], qb[u], vm[u], snuv[u], p8);
        if (++rounds == kDrainRounds) {
          p8.drain(tc);
          rounds = 0;
        }
      }
    }
    if (!next) break;
    uint32_t s0 = 0;
    if (lane == 0) s0 = atomicAdd(next, kClaim);
    s0 = fixed + __shfl_sync(kFull, s0, 0);
    if (s0 >= total) break;
    seg_begin = s0;
    seg_end = min(total, s0 + kClaim);
  }
  p8.drain(tc);
}

// The streamed arcs of a staged list as one sequence of aligned int4
// chunks.  Warp w takes a contiguous 1/warps share of the sequence and its
// lanes take consecutive chunks (coalesced); each lane keeps the extent of
// its current arc in registers and moves its cursor only at an arc
// boundary.  With `next` (a shared counter, zero on entry), the shares
// cover the first 7/8 of the sequence and the warps then claim the rest
// 64 U chunks at a time, so that a warp held up by B lists from DRAM or
// by SEARCH arcs takes less of it and the CTA reaches its next barrier
// together.
// Per chunk: the four ids (one 16-byte load) and their four sign bytes (one
// 4-byte load), a 4-bit mask of the ids inside the arc, then for HASH one
// 8-byte bucket read per id answers membership and the A' sign together;
// MERGE chunks are merged against the sorted A' instead.
// kSplit: compiled with the SPLIT path (a split index per arc, a per-chunk
// choice of source); kernels without it stay as lean as before SPLIT.
template <int U, bool kSplit>
__device__ __forceinline__ void stream_pass(const Csr& g, const StageMem& m, uint32_t d,
                                            uint32_t warp, uint32_t warps, uint32_t lane,
                                            const Geo& geo, TypeCounts& tc, uint32_t* next) {
  const uint32_t total = m.pre[d];
  const uint32_t fixed = next ? total - total / 8 : total;
  const uint32_t per = (fixed + warps - 1) / warps;
  uint32_t seg_begin = min(fixed, warp * per), seg_end = min(fixed, seg_begin + per);
  // Arc cursor k and, per arc: chunk index = cb + flattened index; the masks
  // of its first and last chunk (every chunk between is whole).
  uint32_t k = 0, pk, pk1, cb, mf, ml, ast, anuv, asp = 0;
  auto enter = [&](uint32_t kk) {
    pk = m.pre[kk];
    pk1 = m.pre[kk + 1];
    const uint32_t alo = m.lo[kk], ahi = m.hi[kk];
    cb = (alo >> 2) - pk;
    mf = (0xFu << (alo & 3u)) & 0xFu;
    ml = 0xFu >> (3u - ((ahi - 1u) & 3u));
    ast = m.st[kk];
    anuv = m.s[kk] < 0;
    if (kSplit) asp = m.sp[kk];
  };
  // 8-bit fields: at most 4 U adds per field per round.
  constexpr uint32_t kDrainRounds = 255 / (4 * U);
  constexpr uint32_t kClaim = 64 * U;  // chunks a warp claims at a time
  PackedCounts8 p8;
  uint32_t rounds = 0;
  while (true) {
    if (seg_begin < seg_end) {
      // Forward to the last arc with pre[k] <= the lane's first chunk (the
      // chunks of a lane only grow, and pre[d] = total exceeds every chunk).
      {
        uint32_t lo_k = k, hi_k = d;
        const uint32_t c0 = seg_begin + lane;
        while (hi_k - lo_k > 1) {
          const uint32_t mid = (lo_k + hi_k) >> 1;
          if (m.pre[mid] <= c0) lo_k = mid; else hi_k = mid;
        }
        k = lo_k;
        enter(k);
      }
      for (uint32_t base = seg_begin; base < seg_end; base += 32 * U) {
        uint4 q[U];
        uint32_t sw[U], vm[U], sk[U], snuv[U], sst[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t c = base + 32 * u + lane;
          vm[u] = 0;
          if (c < seg_end) {
            if (c >= pk1) {
              do {
                k++;
              } while (m.pre[k + 1] <= c);
              enter(k);
            }
            const uint32_t ci = cb + c;
            load_chunk(g, ci, kSplit ? ast : (uint32_t)STC_STRATEGY_HASH, asp, q[u], sw[u]);
            vm[u] = (c == pk ? mf : 0xFu) & (c + 1 == pk1 ? ml : 0xFu);
            sk[u] = k;
            snuv[u] = anuv;
            sst[u] = ast;
          }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
          if (vm[u]) process_chunk(m, d, geo, q[u], sw[u], vm[u], sk[u], snuv[u], sst[u], p8);
        if (++rounds == kDrainRounds) {
          p8.drain(tc);
          rounds = 0;
        }
      }
    }
    if (!next) break;
    uint32_t s0 = 0;
    if (lane == 0) s0 = atomicAdd(next, kClaim);
    s0 = fixed + __shfl_sync(kFull, s0, 0);
    if (s0 >= total) break;
    seg_begin = s0;
    seg_end = min(total, s0 + kClaim);
  }
  p8.drain(tc);
}

// SEARCH arcs of a staged list, one arc per warp.
__device__ __forceinline__ void search_pass(const Csr& g, const StageMem& m, uint32_t d,
                                            uint32_t warp, uint32_t warps, uint32_t lane,
                                            PackedCounts& pc, TypeCounts& tc) {
  for (uint32_t k = warp; k + 1 < d; k += warps) {
    if (m.st[k] != STC_STRATEGY_SEARCH) continue;
    const uint32_t lo = m.lo[k];
    arc_search(m.a, m.s, k + 1, d, m.s[k] < 0, g.nbr + lo, g.sgn + lo, m.hi[k] - lo, lane, pc);
    pc.drain(tc);
  }
}

// ------------------------------------------------------ arc timing ----
// Timing recorder (CountConfig::arc_cycles): per dispatch cell
// (class, bucket |A'|, bucket |B|), the SM cycles spent on its arcs and the
// number of arcs.  In this mode every arc is processed alone by one warp,
// timed from the first load of its B to the last count it adds, so three runs
// with the strategy forced give every cell's cost under every strategy: the
// training data of the learned dispatcher and the measure of a dispatch
// table's regret.  The counting kernels proper pack the int4 chunks of all
// HASH and MERGE arcs of a list into one stream that keeps every lane busy,
// so such an arc of c chunks is charged its share of the lanes it would
// occupy there, c / (32 ceil(c / 32)) of the warp's time; a SEARCH arc holds
// a whole warp in both modes and is charged the warp's time.
struct ArcTimes {
  unsigned long long* cycles;  // kTableClasses * 256 cells
  unsigned long long* arcs;
};

// SM clock read that the compiler cannot hoist above the computation of
// `dep` (an input operand of the read).
__device__ __forceinline__ long long clock_after(unsigned long long dep) {
  long long t;
  asm volatile("mov.u64 %0, %%clock64;" : "=l"(t) : "l"(dep) : "memory");
  return t;
}

__device__ __forceinline__ void record_arc(const ArcTimes& at, uint32_t tclass, uint32_t alen,
                                           uint32_t blen, unsigned cycles) {
  const uint32_t cell = tclass * 256 + size_bucket(alen) * 16 + size_bucket(blen);
  atomicAdd(at.cycles + cell, (unsigned long long)cycles);
  atomicAdd(at.arcs + cell, 1ull);
}

// HASH or MERGE for arc k alone: the warp's lanes take consecutive int4
// chunks of B.
__device__ __forceinline__ void arc_stream(const Csr& g, const StageMem& m, uint32_t d, uint32_t k,
                                           uint32_t lane, const Geo& geo, PackedCounts& pc) {
  const uint32_t lo = m.lo[k], hi = m.hi[k], st = m.st[k], nuv = m.s[k] < 0;
  const uint32_t sp = st == STC_STRATEGY_SPLIT ? m.sp[k] : 0u;
  const uint32_t c1 = (hi + 3) >> 2;
  for (uint32_t ci = (lo >> 2) + lane; ci < c1; ci += 32) {
    uint4 q;
    uint32_t sw;
    load_chunk(g, ci, st, sp, q, sw);
    process_chunk(m, d, geo, q, sw, chunk_mask(ci, lo, hi), k, nuv, st, pc);
  }
}

// All arcs of a staged list, one arc per warp at a time, each timed.
__device__ __forceinline__ void timed_pass(const Csr& g, const StageMem& m, uint32_t d,
                                           uint32_t warp, uint32_t warps, uint32_t lane,
                                           const Geo& geo, PackedCounts& pc, TypeCounts& tc,
                                           const ArcTimes& at, uint32_t tclass) {
  for (uint32_t k = warp; k + 1 < d; k += warps) {
    const uint32_t st = m.st[k];
    if (st == kNoArc) continue;
    const uint32_t lo = m.lo[k], hi = m.hi[k], blen = hi - lo;
    __syncwarp();
    const long long t0 = clock_after(0);
    if (st == STC_STRATEGY_SEARCH)
      arc_search(m.a, m.s, k + 1, d, m.s[k] < 0, g.nbr + lo, g.sgn + lo, blen, lane, pc);
    else
      arc_stream(g, m, d, k, lane, geo, pc);
    // The arc's time is the latest lane's (each lane stops its clock once its
    // own counts are in).
    unsigned dt = __reduce_max_sync(kFull, (unsigned)(clock_after(pc.w) - t0));
    if (st != STC_STRATEGY_SEARCH) {  // lane share in the packed stream
      const uint32_t chunks = ((hi + 3) >> 2) - (lo >> 2);
      dt = (unsigned)((unsigned long long)dt * chunks / (32ull * ((chunks + 31) >> 5)));
    }
    pc.drain(tc);
    if (lane == 0) record_arc(at, tclass, d - k - 1, blen, max(dt, 1u));
  }
}

// ------------------------------------------------------- reductions ----
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

// Where per-vertex totals go when a kernel reports per vertex.
struct TotalSink {  // only the four global counters
  static constexpr bool kPerVertex = false;
  __device__ void put(uint32_t, const unsigned long long*) const {}
  __device__ uint32_t key(uint32_t) const { return 0; }
  __device__ void put_key(uint32_t, const unsigned long long*) const {}
};
struct VertexSink {  // per-source counts by original id: vcounts[4 * id + type]
  static constexpr bool kPerVertex = true;
  unsigned long long* vcounts;
  const uint32_t* verts;
  __device__ void put(uint32_t u, const unsigned long long* c) const {
#pragma unroll
    for (int k = 0; k < 4; k++) vcounts[4ull * verts[u] + (3 - k)] = c[k];
  }
  // Keyed form (the head side adds up the items of one key): the vertex.
  __device__ uint32_t key(uint32_t u) const { return u; }
  __device__ void put_key(uint32_t u, const unsigned long long* c) const {
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (c[k]) atomicAdd(vcounts + 4ull * verts[u] + (3 - k), c[k]);
  }
};
struct GraphSink {  // per-graph counts of a batch: gcounts[4 * graph + type]
  static constexpr bool kPerVertex = true;
  unsigned long long* gcounts;
  const uint64_t* gbase;  // G + 1 rank boundaries (graphs are contiguous in rank space)
  uint32_t G;
  __device__ uint32_t graph_of(uint32_t u) const {
    uint32_t lo = 0, hi = G;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (gbase[mid] <= u) lo = mid; else hi = mid;
    }
    return lo;
  }
  __device__ void put(uint32_t u, const unsigned long long* c) const { put_key(graph_of(u), c); }
  // Keyed form (the head side adds up the items of one key): the graph.
  __device__ uint32_t key(uint32_t u) const { return graph_of(u); }
  __device__ void put_key(uint32_t g, const unsigned long long* c) const {
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (c[k]) atomicAdd(gcounts + 4ull * g + (3 - k), c[k]);
  }
};

// Reduces one vertex's counters over the CTA and hands them to the sink.
template <int THREADS, class Sink>
__device__ __forceinline__ void block_vertex_flush(const TypeCounts& vc, uint32_t u, const Sink& sink) {
  __shared__ unsigned long long red[THREADS / 32][4];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const unsigned long long v = warp_sum(vc.c[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s[4] = {0, 0, 0, 0};
    for (int w = 0; w < THREADS / 32; w++)
      for (int k = 0; k < 4; k++) s[k] += red[w][k];
    sink.put(u, s);
  }
  __syncthreads();
}

// Reduces a key's counters over the CTA and hands them to the sink's keyed
// form (every thread calls it, with the same key).
template <int THREADS, class Sink>
__device__ __forceinline__ void block_key_flush(const TypeCounts& vc, uint32_t key,
                                                const Sink& sink) {
  __shared__ unsigned long long red[THREADS / 32][4];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const unsigned long long v = warp_sum(vc.c[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s[4] = {0, 0, 0, 0};
    for (int w = 0; w < THREADS / 32; w++)
      for (int k = 0; k < 4; k++) s[k] += red[w][k];
    sink.put_key(key, s);
  }
  __syncthreads();
}

template <class Sink>
__device__ __forceinline__ void warp_vertex_flush(const TypeCounts& vc, uint32_t u, uint32_t lane,
                                                  const Sink& sink) {
  unsigned long long s[4];
#pragma unroll
  for (int k = 0; k < 4; k++) s[k] = warp_sum(vc.c[k]);
  if (lane == 0) sink.put(u, s);
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
// Device plan of a persistent count: plan[c] = first list entry of class c
// (plan[kClasses] = total), plan[kPlanCounts + c] = its vertex count.
constexpr uint32_t kPlanCounts = 8;
constexpr uint32_t kPlanWords = kPlanCounts + kClasses;

// Source vertices [range[0], range[1]) of rank space, or all n when `range`
// is null (a sharded count reads its range from the counters).
__device__ __forceinline__ void source_range(const unsigned long long* range, uint32_t n,
                                             uint32_t& u0, uint32_t& u1) {
  u0 = range ? (uint32_t)range[0] : 0u;
  u1 = range ? (uint32_t)range[1] : n;
}

// `need` (optional): a vertex whose flag is 0 has no arc for the tail side
// (the head-side pass counts all of them) and joins no class.
__global__ void k_classify_count(const uint64_t* __restrict__ off, uint32_t n, ClassBounds cb,
                                 unsigned long long* __restrict__ ctr,
                                 const unsigned long long* __restrict__ range,
                                 const uint8_t* __restrict__ need = nullptr) {
  uint32_t cnt[kClasses] = {0, 0, 0, 0, 0};
  uint32_t dmax = 0;
  uint32_t u0, u1;
  source_range(range, n, u0, u1);
  for (uint32_t u = u0 + blockIdx.x * blockDim.x + threadIdx.x; u < u1; u += gridDim.x * blockDim.x) {
    const uint32_t d = (uint32_t)(off[u + 1] - off[u]);
    const uint32_t c = (need && !need[u]) ? 5u : cb.of(d);
    dmax = max(dmax, d);
#pragma unroll
    for (int i = 0; i < kClasses; i++) cnt[i] += c == (uint32_t)i;
  }
  dmax = __reduce_max_sync(kFull, dmax);
  if (lane_id() == 0) atomicMax(ctr + C_MAX_FDEG, (unsigned long long)dmax);
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
                                unsigned long long* __restrict__ cursor,
                                const unsigned long long* __restrict__ range,
                                const uint8_t* __restrict__ need = nullptr) {
  uint32_t u0, u1;
  source_range(range, n, u0, u1);
  for (uint32_t base = u0 + blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < u1;
       base += gridDim.x * blockDim.x) {
    const uint32_t u = base + lane_id();
    const uint32_t c = (u >= u1 || (need && !need[u])) ? 5u : cb.of((uint32_t)(off[u + 1] - off[u]));
    const unsigned peers = __match_any_sync(kFull, c);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (c < kClasses && lane_id() == leader) pos = (uint32_t)atomicAdd(cursor + c, (unsigned long long)__popc(peers));
    pos = __shfl_sync(kFull, pos, leader) + __popc(peers & lanemask_lt());
    if (c < kClasses) lists[starts[c] + pos] = u;
  }
}

// Tiny class: one thread per vertex, A in registers, B in global memory.
// One tiny list (one thread): A in registers, a monotone binary search of
// each later A' element in B; arcs whose cell in `table` (the warp class's)
// is HEAD are left to the head-side pass.
template <int TMAX, class Sink>
__device__ __forceinline__ void tiny_vertex(const Csr& g, uint32_t u, const Sink& sink,
                                            const uint8_t (*table)[16], TypeCounts& tc) {
  constexpr bool kVC = Sink::kPerVertex;
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
    if (table[size_bucket(d - k - 1)][size_bucket(blen)] == STC_STRATEGY_HEAD) continue;
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
  if (kVC) sink.put(u, vc.c);
}

// Tiny class: one thread per vertex, A in registers, B in global memory.
template <int TMAX, class Sink>
__global__ void __launch_bounds__(256) k_tiny(Csr g, const uint32_t* __restrict__ list, uint32_t cnt,
                                              unsigned long long* __restrict__ ctr, Sink sink,
                                              const uint8_t* __restrict__ gtable) {
  __shared__ uint8_t table[16][16];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) (&table[0][0])[i] = gtable[i];
  __syncthreads();
  TypeCounts tc;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += gridDim.x * blockDim.x)
    tiny_vertex<TMAX>(g, list[idx], sink, table, tc);
  if (!Sink::kPerVertex) flush_counts<256>(tc, ctr);
}

// Warp class: one warp per vertex, staged in the warp's slice of shared
// memory (256 hash buckets).
constexpr uint32_t kWarpBuckets = 2 * kWarpCap;
constexpr size_t kWarpStageBytes = (StageMem::bytes(kWarpCap, kWarpBuckets) + 15) & ~size_t(15);

// One warp-class list, staged in the warp's shared-memory slice `m` with
// up to hf hash buckets per element; U int4 chunks in flight per lane.
template <class Sink, bool kTime, int U, bool kSplit>
__device__ __forceinline__ void warp_vertex(const Csr& g, uint32_t u, uint32_t lane,
                                            const StageMem& m, const uint8_t (*table)[16],
                                            uint32_t hf, unsigned long long* __restrict__ ctr,
                                            const Sink& sink, const ArcTimes& at, TypeCounts& tc) {
  constexpr bool kVC = Sink::kPerVertex;
  const uint64_t ub = g.off[u];
  const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
  if (d > kWarpCap) {  // uniform over the warp
    if (lane == 0) atomicExch(ctr + C_ERROR, kErrStageCapacity);
    return;
  }
  const Geo geo = Geo::of(d, kWarpBuckets, hf);
  stage<32>(g, ub, d, lane, m, geo, table, WarpSync{});
  TypeCounts vc;
  TypeCounts& out = kVC ? vc : tc;
  PackedCounts pc;
  if (kTime) {
    timed_pass(g, m, d, 0, 1, lane, geo, pc, out, at, kTableWarp);
  } else {
    warp_chunk_scan(m, d, lane);
    stream_pass<U, kSplit>(g, m, d, 0, 1, lane, geo, out, nullptr);
    search_pass(g, m, d, 0, 1, lane, pc, out);
  }
  pc.drain(out);
  if (kVC) warp_vertex_flush(vc, u, lane, sink);
  __syncwarp();
}

template <class Sink, bool kTime, int U, bool kSplit>
__global__ void __launch_bounds__(256, U >= 4 ? 3 : 4) k_warp(Csr g, const uint32_t* __restrict__ list, uint32_t cnt,
                                              unsigned long long* __restrict__ ctr, Sink sink,
                                              const uint8_t* __restrict__ gtable, ArcTimes at,
                                              uint32_t hf) {
  constexpr bool kVC = Sink::kPerVertex;
  constexpr int kWarps = 8;
  __shared__ __align__(16) unsigned char smem[kWarps * kWarpStageBytes];
  __shared__ uint8_t table[16][16];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) (&table[0][0])[i] = gtable[i];
  __syncthreads();
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const StageMem m = StageMem::carve(smem + w * kWarpStageBytes, kWarpCap, kWarpBuckets);
  TypeCounts tc;
  const uint32_t warps = gridDim.x * kWarps;
  for (uint32_t idx = blockIdx.x * kWarps + w; idx < cnt; idx += warps)
    warp_vertex<Sink, kTime, U, kSplit>(g, list[idx], lane, m, table, hf, ctr, sink, at, tc);
  if (!kVC) flush_counts<256>(tc, ctr);
}

// Block classes: one CTA per vertex from a dynamic queue, the list staged in
// dynamic shared memory of capacity `cap` with `nb` hash buckets
// (nb >= 2 * cap, powers of two).
inline size_t block_stage_bytes(uint32_t cap, uint32_t nb) { return StageMem::bytes(cap, nb); }
constexpr size_t kMaxStageSmem = 220 * 1024;  // dynamic shared memory a staged CTA may use

// One block-class list (the whole CTA), staged in `m` of capacity `cap`
// with `nb` hash buckets.  scan_tmp has THREADS / 32 + 2 words: the chunk
// scan's and the stream's claim counter.
template <int THREADS, class Sink, bool kTime, int U, bool kSplit>
__device__ __forceinline__ void block_vertex(const Csr& g, uint32_t u, uint32_t cap, uint32_t nb,
                                             uint32_t hf, const StageMem& m,
                                             const uint8_t (*table)[16],
                                             uint32_t* scan_tmp, unsigned long long* __restrict__ ctr,
                                             const Sink& sink, const ArcTimes& at, uint32_t tclass,
                                             TypeCounts& tc) {
  constexpr bool kVC = Sink::kPerVertex;
  constexpr uint32_t kWarps = THREADS / 32;
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const uint64_t ub = g.off[u];
  const uint32_t d = (uint32_t)(g.off[u + 1] - ub);
  if (d > cap) {  // uniform over the CTA
    if (threadIdx.x == 0) atomicExch(ctr + C_ERROR, kErrStageCapacity);
    return;
  }
  const Geo geo = Geo::of(d, nb, hf);
  // The stream's claim counter: the CTA passed a barrier since the last list
  // used it, and stage() passes another before this one does.
  uint32_t* next = scan_tmp + kWarps + 1;
  if (threadIdx.x == 0) *next = 0;
  stage<THREADS>(g, ub, d, threadIdx.x, m, geo, table, BlockSync{});
  TypeCounts vc;
  TypeCounts& out = kVC ? vc : tc;
  PackedCounts pc;
  if (kTime) {
    timed_pass(g, m, d, w, kWarps, lane, geo, pc, out, at, tclass);
  } else {
    block_chunk_scan<THREADS>(m, d, scan_tmp);
    search_pass(g, m, d, w, kWarps, lane, pc, out);
    stream_pass<U, kSplit>(g, m, d, w, kWarps, lane, geo, out, next);
  }
  pc.drain(out);
  if (kVC) block_vertex_flush<THREADS>(vc, u, sink);
}

template <int THREADS, class Sink, bool kTime, int U, bool kSplit>
__global__ void __launch_bounds__(THREADS) k_block(Csr g, const uint32_t* __restrict__ list,
                                                   uint32_t cnt, uint32_t cap, uint32_t nb, uint32_t hf,
                                                   unsigned long long* __restrict__ queue,
                                                   unsigned long long* __restrict__ ctr, Sink sink,
                                                   const uint8_t* __restrict__ gtable, ArcTimes at,
                                                   uint32_t tclass, const uint32_t* __restrict__ plan,
                                                   uint32_t pclass) {
  constexpr bool kVC = Sink::kPerVertex;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint8_t table[16][16];
  __shared__ uint32_t scan_tmp[THREADS / 32 + 2];
  __shared__ uint32_t s_item;
  for (int i = threadIdx.x; i < 256; i += THREADS) (&table[0][0])[i] = gtable[i];
  if (plan) {  // list and count planned on the device
    list += plan[pclass];
    cnt = plan[kPlanCounts + pclass];
  }
  const StageMem m = StageMem::carve(smem, cap, nb);
  TypeCounts tc;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (uint32_t)atomicAdd(queue, 1ull);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= cnt) break;
    block_vertex<THREADS, Sink, kTime, U, kSplit>(g, list[item], cap, nb, hf, m, table, scan_tmp,
                                                  ctr, sink, at, tclass, tc);
  }
  if (!kVC) flush_counts<THREADS>(tc, ctr);
}

// Giant lists (d > kLargeCap): one CTA per vertex, A read from global memory,
// one arc per warp; HASH falls back to MERGE (no staged hash).
template <int THREADS, class Sink, bool kTime>
__global__ void __launch_bounds__(THREADS) k_giant(Csr g, const uint32_t* __restrict__ list,
                                                   uint32_t cnt, unsigned long long* __restrict__ queue,
                                                   unsigned long long* __restrict__ ctr, Sink sink,
                                                   const uint8_t* __restrict__ gtable, ArcTimes at,
                                                   const uint32_t* __restrict__ plan, uint32_t pclass) {
  constexpr bool kVC = Sink::kPerVertex;
  __shared__ uint8_t table[16][16];
  __shared__ uint32_t s_item;
  for (int i = threadIdx.x; i < 256; i += THREADS) (&table[0][0])[i] = gtable[i];
  if (plan) {  // list and count planned on the device
    list += plan[pclass];
    cnt = plan[kPlanCounts + pclass];
  }
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
    const uint32_t* a = g.nbr + ub;
    const int8_t* s = g.sgn + ub;
    TypeCounts vc;
    TypeCounts& out = kVC ? vc : tc;
    for (uint32_t k = w; k + 1 < d; k += kWarps) {
      const uint32_t v = a[k];
      const uint64_t vb = g.off[v];
      const uint32_t blen = (uint32_t)(g.off[v + 1] - vb);
      if (blen == 0) continue;
      const uint32_t st = table[size_bucket(d - k - 1)][size_bucket(blen)];
      if (st == STC_STRATEGY_HEAD) continue;  // counted by the head-side pass
      long long t0 = 0;
      if (kTime) {
        __syncwarp();
        t0 = clock_after(0);
      }
      // 64-bit counters: a giant list may be long enough to overflow the
      // packed 16-bit fields within one arc.
      if (st == STC_STRATEGY_SEARCH)
        arc_search(a, s, k + 1, d, s[k] < 0, g.nbr + vb, g.sgn + vb, blen, lane, out);
      else
        arc_merge_global(a, s, k + 1, d, s[k] < 0, g.nbr + vb, g.sgn + vb, blen, lane, out);
      if (kTime) {
        const unsigned long long dep = out.c[0] + out.c[1] + out.c[2] + out.c[3];
        const unsigned dt = __reduce_max_sync(kFull, (unsigned)(clock_after(dep) - t0));
        if (lane == 0) record_arc(at, kTableGiant, d - k - 1, blen, dt);
      }
    }
    if (kVC) block_vertex_flush<THREADS>(vc, u, sink);
  }
  if (!kVC) flush_counts<THREADS>(tc, ctr);
}

// Compile-time choices of the tuned kernels, selected at run time.
template <int V> struct Int { static constexpr int value = V; };
template <class F> void with_unroll(uint32_t u, F&& f) {
  if (u == 1) f(Int<1>{});
  else if (u == 4) f(Int<4>{});
  else f(Int<2>{});
}
template <class F> void with_split(bool split, F&& f) {
  if (split) f(std::true_type{});
  else f(std::false_type{});
}
template <class F> void with_block_threads(uint32_t t, F&& f) {
  if (t == 128) f(Int<128>{});
  else if (t == 512) f(Int<512>{});
  else f(Int<256>{});
}

// Largest hash factor whose staged image of `cap` entries fits the
// shared memory of one CTA.
inline uint32_t fit_hash_factor(uint32_t hf, uint32_t cap) {
  while (hf > 1 && StageMem::bytes(cap, hf * cap) > kMaxStageSmem) hf >>= 1;
  return hf;
}

// Launches the class kernels for one sink kind.  `d_tables` holds one
// 256-byte table per TableClass; `tu` gives the tuned block size, hash
// factors and stream widths; classes outside `mask` are skipped.  The timing
// recorder (kTime) uses the default widths and block size, which its
// per-arc passes do not depend on.
template <class Sink, bool kTime>
void launch_classes(cudaStream_t st, const Csr& csr, const uint32_t* lists, const uint32_t* counts,
                    const uint32_t* starts, uint32_t max_fdeg, unsigned long long* ctr,
                    const uint8_t* d_tables, const Sink& sink, const ArcTimes& at,
                    const Tuning& tu, uint32_t mask, int& launches) {
  if (counts[0] && (mask & 1u)) {
    const uint32_t grid = std::min<uint32_t>((counts[0] + 255) / 256, kSMs * 8);
    k_tiny<kTinyMax, Sink><<<grid, 256, 0, st>>>(csr, lists + starts[0], counts[0], ctr, sink,
                                                  d_tables + 256 * kTableWarp);
    launches++;
  }
  if (counts[1] && (mask & 2u)) {
    const uint32_t grid = std::min<uint32_t>((counts[1] + 7) / 8, kSMs * 8);
    const uint32_t u = kTime ? kStreamUnroll : tu.unroll[0];
    with_split(!kTime && csr.nbr_split != nullptr, [&](auto S) {
      with_unroll(u, [&](auto U) {
        if constexpr (!kTime || (decltype(U)::value == kStreamUnroll && !decltype(S)::value))
          k_warp<Sink, kTime, decltype(U)::value, decltype(S)::value><<<grid, 256, 0, st>>>(
              csr, lists + starts[1], counts[1], ctr, sink, d_tables + 256 * kTableWarp, at,
              tu.hash_factor[0]);
      });
    });
    launches++;
  }
  if (counts[2] && (mask & 4u)) {
    const uint32_t cap = kBlockCap;
    const uint32_t hf = fit_hash_factor(tu.hash_factor[1], cap);
    const uint32_t nb = hf * cap;
    const size_t smem = block_stage_bytes(cap, nb);
    const uint32_t threads = kTime ? 256 : tu.block_threads;
    const uint32_t u = kTime ? kStreamUnroll : tu.unroll[1];
    with_split(!kTime && csr.nbr_split != nullptr, [&](auto S) {
      with_block_threads(threads, [&](auto T) {
        with_unroll(u, [&](auto U) {
          constexpr int kT = decltype(T)::value, kU = decltype(U)::value;
          constexpr bool kS = decltype(S)::value;
          if constexpr (!kTime || (kT == 256 && kU == kStreamUnroll && !kS)) {
            STC_CUDA(cudaFuncSetAttribute(k_block<kT, Sink, kTime, kU, kS>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const uint32_t grid = std::min<uint32_t>(counts[2], kSMs * 8);
            k_block<kT, Sink, kTime, kU, kS><<<grid, kT, smem, st>>>(
                csr, lists + starts[2], counts[2], cap, nb, hf, ctr + C_WORK + 0, ctr, sink,
                d_tables + 256 * kTableBlock, at, kTableBlock, nullptr, 0);
          }
        });
      });
    });
    launches++;
  }
  if (counts[3] && (mask & 8u)) {
    // Capacity: the class's largest list rounded up to a power of two.
    uint32_t cap = kBlockCap;
    while (cap < std::min<uint32_t>(max_fdeg, kLargeCap)) cap <<= 1;
    const uint32_t hf = fit_hash_factor(tu.hash_factor[2], cap);
    const uint32_t nb = hf * cap;
    const size_t smem = block_stage_bytes(cap, nb);
    const uint32_t u = kTime ? kStreamUnroll : tu.unroll[2];
    with_split(!kTime && csr.nbr_split != nullptr, [&](auto S) {
      with_unroll(u, [&](auto U) {
        constexpr int kU = decltype(U)::value;
        constexpr bool kS = decltype(S)::value;
        if constexpr (!kTime || (kU == kStreamUnroll && !kS)) {
          STC_CUDA(cudaFuncSetAttribute(k_block<512, Sink, kTime, kU, kS>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          const uint32_t grid = std::min<uint32_t>(counts[3], kSMs * 2);
          k_block<512, Sink, kTime, kU, kS><<<grid, 512, smem, st>>>(
              csr, lists + starts[3], counts[3], cap, nb, hf, ctr + C_WORK + 1, ctr, sink,
              d_tables + 256 * kTableLarge, at, kTableLarge, nullptr, 0);
        }
      });
    });
    launches++;
  }
  if (counts[4] && (mask & 16u)) {
    const uint32_t grid = std::min<uint32_t>(counts[4], kSMs * 2);
    k_giant<512, Sink, kTime><<<grid, 512, 0, st>>>(csr, lists + starts[4], counts[4],
                                                     ctr + C_WORK + 2, ctr, sink,
                                                     d_tables + 256 * kTableGiant, at, nullptr, 0);
    launches++;
  }
}

// ------------------------------------------------------- head side ----
// Arcs whose dispatch cell says STC_STRATEGY_HEAD are counted from their
// head.  For the arc u -> v, the third vertex w of a triangle lies in
// A' = the part of N+(u) after v and in B = N+(v).  The tail side (the
// kernels above) stages N+(u) and streams B; the head side stages N+(v) as
// the shared-memory hash and streams A' through it, so an arc costs |A'|
// probes instead of |B|.  Over a power-law graph in (degree, id) order,
// A' is the shorter list for almost every arc (the reference's hash
// program iterates the shorter of its two lists for the same reason,
// MC/tc_hash_sign_enu.cpp:146-160).
//
// The head side finds each vertex's in-arcs by a sort: every HEAD arc i
// (its index in the CSR) is appended as the key v << 32 | i (a warp adds its
// keys with one atomic, so their order varies from run to run; the counts
// are sums and do not depend on it), a radix sort over the vertex bits of
// the appended keys, their number known on the device only, groups each
// head's in-arcs, and the runs of equal v are its in-arc ranges.  Head vertices are classed by
// |N+(v)|, the list they stage: warp (<= 128), block (<= 1024) and large
// (<= 4095).  A work item is a piece of one head's run that does not cross
// a multiple of its class's item size (a hub with millions of in-arcs
// becomes thousands of items, each staging its small N+(v) again), so no
// warp or CTA is left with one huge run.  Each in-arc is one "arc" of the
// staged tile with extent
// [i + 1, end of u's list), its sign s(u, v), strategy HASH: the tail
// side's stream pass then runs unchanged, with the hash keys carrying
// s(v, w), the streamed sign bytes s(u, w) and the arc's sign s(u, v).
constexpr uint32_t kHeadMaxB = kLargeCap - 1;  // |N+(v)| of a HEAD arc: bucket <= 12
static_assert(32 - __builtin_clz(kHeadMaxB) == 12 && 32 - __builtin_clz(kHeadMaxB + 1) == 13,
              "HEAD cells (bucket |B| <= 12) are exactly the arcs whose head fits the large class");
constexpr int kHeadClasses = 3;
// Head list buffer: plan words first (start of class c's list, then from
// kHeadPlanCount its count), the class lists after them, then one byte per
// vertex: whether it keeps arcs for the tail side.
constexpr uint32_t kHeadPlanCount = 4;
constexpr uint32_t kHeadPlanWords = 8;
constexpr uint32_t kHeadItemMin = 2048;  // the smallest class item size

// In-arcs per work item of head class c (powers of two).
__host__ __device__ __forceinline__ uint32_t head_item(uint32_t c) {
  return c == 0 ? kHeadItemMin : c == 1 ? 8192u : 16384u;
}

// Table class of a list of d arcs (tiny lists use the warp class's table).
__device__ __forceinline__ uint32_t table_class(uint32_t d) {
  return d <= kWarpCap ? kTableWarp : d <= kBlockCap ? kTableBlock
                                    : d <= kLargeCap ? kTableLarge : kTableGiant;
}
// Head class of a head vertex with d = |N+(v)| in [1, kHeadMaxB].
__device__ __forceinline__ uint32_t head_class(uint32_t d) {
  return d <= kWarpCap ? 0u : d <= kBlockCap ? 1u : 2u;
}

struct HeadArcs {
  const uint64_t* __restrict__ keys;  // sorted: v << 32 | arc index
  const uint32_t* __restrict__ aend;  // per arc: end of its tail's list in the CSR
  const uint32_t* __restrict__ end;   // per head vertex: one past its last in-arc entry
  const uint32_t* __restrict__ asrc;  // per arc: its tail (timing recorder only)
  // Work item starting at entry j0 of head class c: its head and its end.
  __device__ __forceinline__ void item(uint32_t j0, uint32_t c, uint32_t& v, uint32_t& j1) const {
    v = (uint32_t)(keys[j0] >> 32);
    j1 = min(end[v], (j0 | (head_item(c) - 1)) + 1);
  }
};

// Appends the keys of the HEAD arcs (count in ctr[C_HEAD_NKEYS]), records
// the list end of each HEAD arc, and sets need[u] = 1 for each tail u with
// an arc left to the tail side (the array starts at 0; tails without such
// arcs are not staged there).  `range` (a sharded count) keeps only tails
// in [range[0], range[1]).
// Size bucket of every vertex's out-degree, one byte each: the head keys
// gather it for every arc's head, from an array a quarter the size of the
// out-degrees (more of it stays in L2).
__global__ void k_fdeg_bucket(const uint32_t* __restrict__ fdeg, uint32_t n,
                              uint8_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (uint8_t)size_bucket(fdeg[i]);
}

__global__ void __launch_bounds__(256) k_head_keys(Csr g, const uint32_t* __restrict__ asrc,
                                                   const uint8_t* __restrict__ fbkt, uint64_t m,
                                                   const unsigned long long* __restrict__ m_dev,
                                                   const uint8_t* __restrict__ gtables,
                                                   const unsigned long long* __restrict__ range,
                                                   uint64_t* __restrict__ keys,
                                                   uint32_t* __restrict__ aend,
                                                   uint8_t* __restrict__ need,
                                                   unsigned long long* __restrict__ ctr) {
  constexpr int kItems = 4;  // arcs per lane with their gathers in flight together
  __shared__ uint8_t tab[kTableBytes];
  if (m_dev) m = min(m, (uint64_t)*m_dev);  // m a capacity, *m_dev the arc count
  for (uint32_t i = threadIdx.x; i < kTableBytes; i += blockDim.x) tab[i] = gtables[i];
  __syncthreads();
  const uint32_t r0 = range ? (uint32_t)range[0] : 0u;
  const uint32_t r1 = range ? (uint32_t)range[1] : 0xFFFFFFFFu;
  const uint32_t lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * kItems;
  for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) * kItems;
       base < m; base += stride) {
    uint32_t u[kItems], v[kItems], blen[kItems];
    uint64_t ub[kItems], ue[kItems];
#pragma unroll
    for (int q = 0; q < kItems; q++) {
      const uint64_t i = base + 32 * q + lane;
      u[q] = i < m ? asrc[i] : 0u;
      v[q] = i < m ? g.nbr[i] : 0u;
    }
#pragma unroll
    for (int q = 0; q < kItems; q++) {
      const uint64_t i = base + 32 * q + lane;
      ub[q] = i < m ? g.off[u[q]] : 0;
      ue[q] = i < m ? g.off[u[q] + 1] : 0;
      blen[q] = i < m ? fbkt[v[q]] : 0u;
    }
#pragma unroll
    for (int q = 0; q < kItems; q++) {
      const uint64_t i = base + 32 * q + lane;
      bool head = false;
      if (i < m) {
        const uint32_t alen = (uint32_t)(ue[q] - i - 1);
        if (alen && blen[q] && u[q] >= r0 && u[q] < r1) {
          head = tab[256 * table_class((uint32_t)(ue[q] - ub[q])) + 16 * size_bucket(alen) +
                     blen[q]] == STC_STRATEGY_HEAD;
          if (!head) need[u[q]] = 1;  // u keeps an arc for the tail side
        }
      }
      const unsigned hb = __ballot_sync(kFull, head);
      uint32_t at = 0;
      if (lane == 0 && hb)
        at = (uint32_t)atomicAdd(ctr + C_HEAD_NKEYS, (unsigned long long)__popc(hb));
      at = __shfl_sync(kFull, at, 0);
      if (head) {
        keys[at + __popc(hb & lanemask_lt())] = ((uint64_t)v[q] << 32) | i;
        aend[i] = (uint32_t)ue[q];
      }
    }
  }
}

// Work items in the sorted keys: an entry starts one where its head's run
// starts or where it is a multiple of its class's item size.  Without
// kFill: counts the items of each class.  With kFill: appends each item's
// first entry to its class list and records the end of every run.
template <bool kFill>
__global__ void __launch_bounds__(256) k_head_runs(const uint64_t* __restrict__ keys,
                                                   const uint64_t* __restrict__ off,
                                                   unsigned long long* __restrict__ ctr,
                                                   uint32_t* __restrict__ hl,
                                                   uint32_t* __restrict__ end) {
  const uint64_t m = ctr[C_HEAD_NKEYS];
  const uint32_t lane = lane_id();
  uint32_t cnt[kHeadClasses] = {0, 0, 0};
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < m;
       base += stride) {
    const uint64_t j = base + lane;
    uint32_t c = kHeadClasses;  // not an item start
    if (j < m) {
      const uint64_t kv = keys[j] >> 32;
      const uint32_t v = (uint32_t)kv;
      const uint32_t hc = head_class((uint32_t)(off[v + 1] - off[v]));
      if (j == 0 || (keys[j - 1] >> 32) != kv || (j & (head_item(hc) - 1)) == 0) c = hc;
      if (kFill && (j + 1 == m || (keys[j + 1] >> 32) != kv)) end[v] = (uint32_t)(j + 1);
    }
    if (!kFill) {
#pragma unroll
      for (int k = 0; k < kHeadClasses; k++) cnt[k] += c == (uint32_t)k;
    } else {
      // Item starts are rare (about one entry in fifty): one ballot per
      // class, and an atomic only where the warp holds some.
#pragma unroll
      for (uint32_t k = 0; k < (uint32_t)kHeadClasses; k++) {
        const unsigned peers = __ballot_sync(kFull, c == k);
        if (peers == 0) continue;
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t pos = 0;
        if (lane == leader)
          pos = (uint32_t)atomicAdd(ctr + C_HEAD_CURSOR + k, (unsigned long long)__popc(peers));
        pos = __shfl_sync(kFull, pos, leader) + __popc(peers & lanemask_lt());
        if (c == k) hl[kHeadPlanWords + hl[k] + pos] = (uint32_t)j;
      }
    }
  }
  if (!kFill) {
#pragma unroll
    for (int k = 0; k < kHeadClasses; k++) {
      const uint32_t s = __reduce_add_sync(kFull, cnt[k]);
      if (lane == 0 && s) atomicAdd(ctr + C_HEAD_COUNT + k, (unsigned long long)s);
    }
  }
}

// Class list starts from the counts; clears the fill cursors and queues.
__global__ void k_head_plan(unsigned long long* __restrict__ ctr, uint32_t* __restrict__ hl) {
  if (threadIdx.x != 0) return;
  uint32_t start = 0;
  for (int c = 0; c < kHeadClasses; c++) {
    const uint32_t n = (uint32_t)ctr[C_HEAD_COUNT + c];
    hl[c] = start;
    hl[kHeadPlanCount + c] = n;
    start += n;
    ctr[C_HEAD_CURSOR + c] = 0;
    ctr[C_HEAD_QUEUE + c] = 0;
  }
}

// N+(v) (d entries from vb) as the staged hash of a team of TS threads.
template <int TS, class Sync>
__device__ __forceinline__ void stage_hash(const Csr& g, uint64_t vb, uint32_t d, uint32_t t,
                                           const StageMem& m, const Geo& geo, Sync sync) {
  for (uint32_t i = t; i < 2 * geo.nb; i += TS) m.hk[i] = kEmpty;
  sync();
  for (uint32_t i = t; i < d; i += TS) {
    const uint32_t x = g.nbr[vb + i];
    const uint32_t key = (x << 1) | (uint32_t)(g.sgn[vb + i] < 0);
    uint32_t b = hash_slot(x, geo.shift);
    while (atomicCAS(&m.hk[2 * b], kEmpty, key) != kEmpty &&
           atomicCAS(&m.hk[2 * b + 1], kEmpty, key) != kEmpty)
      b = (b + 1) & (geo.nb - 1);
  }
  sync();
}

// In-arcs [j0, j0 + tn) of a head vertex as the arcs of the staged tile.
template <int TS, class Sync>
__device__ __forceinline__ void stage_in_arcs(const Csr& g, const HeadArcs& h, uint32_t j0,
                                              uint32_t tn, uint32_t t, const StageMem& m,
                                              Sync sync) {
  for (uint32_t k = t; k < tn; k += TS) {
    const uint32_t i = (uint32_t)h.keys[j0 + k];
    m.lo[k] = i + 1;
    m.hi[k] = h.aend[i];  // > i + 1: a HEAD arc has a non-empty A'
    m.s[k] = g.sgn[i];
    m.st[k] = STC_STRATEGY_HASH;
  }
  sync();
}

// Timing recorder, head side: each in-arc of the tile alone on one warp,
// timed and charged as a streamed arc is; its cell is that of the arc
// u -> v (class of N+(u), bucket |A'|, bucket |B| = |N+(v)|).
__device__ __forceinline__ void timed_head_pass(const Csr& g, const HeadArcs& h, const StageMem& m,
                                                uint32_t tn, uint32_t dv, uint32_t warp,
                                                uint32_t warps, uint32_t lane, const Geo& geo,
                                                PackedCounts& pc, TypeCounts& tc,
                                                const ArcTimes& at) {
  for (uint32_t k = warp; k < tn; k += warps) {
    const uint32_t lo = m.lo[k], hi = m.hi[k];
    __syncwarp();
    const long long t0 = clock_after(0);
    arc_stream(g, m, tn, k, lane, geo, pc);
    unsigned dt = __reduce_max_sync(kFull, (unsigned)(clock_after(pc.w) - t0));
    const uint32_t chunks = ((hi + 3) >> 2) - (lo >> 2);
    dt = (unsigned)((unsigned long long)dt * chunks / (32ull * ((chunks + 31) >> 5)));
    pc.drain(tc);
    if (lane == 0) {
      const uint32_t u = h.asrc[lo - 1];
      record_arc(at, table_class((uint32_t)(hi - g.off[u])), hi - lo, dv, max(dt, 1u));
    }
  }
}

// Head vertices of the warp class: one warp per vertex from a dynamic
// queue, N+(v) and up to kWarpCap in-arcs at a time staged in the warp's
// slice of shared memory.
template <class Sink, bool kTime, int U>
__global__ void __launch_bounds__(256) k_head_warp(Csr g, HeadArcs h, const uint32_t* __restrict__ hl,
                                                   unsigned long long* __restrict__ ctr, Sink sink,
                                                   ArcTimes at, uint32_t hf) {
  constexpr bool kVC = Sink::kPerVertex;
  constexpr int kWarps = 8;
  __shared__ __align__(16) unsigned char smem[kWarps * kWarpStageBytes];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const StageMem m = StageMem::carve(smem + w * kWarpStageBytes, kWarpCap, kWarpBuckets);
  const uint32_t* list = hl + kHeadPlanWords + hl[0];
  const uint32_t cnt = hl[kHeadPlanCount + 0];
  TypeCounts tc;
  // Per-key counts (a sink that reports per graph): a warp's items come in
  // increasing order of their heads, so the counts of one key are added up
  // and handed to the sink once, when the key changes.
  uint32_t cur = 0xFFFFFFFFu;
  auto flush = [&]() {
    if (kVC && cur != 0xFFFFFFFFu) {
      unsigned long long s[4];
#pragma unroll
      for (int k = 0; k < 4; k++) s[k] = warp_sum(tc.c[k]);
      if (lane == 0) sink.put_key(cur, s);
      tc = TypeCounts{};
    }
  };
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = (uint32_t)atomicAdd(ctr + C_HEAD_QUEUE + 0, 1ull);
    item = __shfl_sync(kFull, item, 0);
    if (item >= cnt) break;
    uint32_t v, j1;
    const uint32_t j00 = list[item];
    h.item(j00, 0, v, j1);
    const uint64_t vb = g.off[v];
    const uint32_t d = (uint32_t)(g.off[v + 1] - vb);
    if (d > kWarpCap) {  // uniform over the warp
      if (lane == 0) atomicExch(ctr + C_ERROR, kErrStageCapacity);
      continue;
    }
    if (kVC) {
      const uint32_t key = sink.key(v);
      if (key != cur) {
        flush();
        cur = key;
      }
    }
    const Geo geo = Geo::of(d, kWarpBuckets, hf);
    stage_hash<32>(g, vb, d, lane, m, geo, WarpSync{});
    TypeCounts& out = tc;
    PackedCounts pc;
    for (uint32_t j0 = j00; j0 < j1; j0 += kWarpCap) {
      const uint32_t tn = min(kWarpCap, j1 - j0);
      stage_in_arcs<32>(g, h, j0, tn, lane, m, WarpSync{});
      if (kTime) {
        timed_head_pass(g, h, m, tn, d, 0, 1, lane, geo, pc, out, at);
      } else {
        warp_chunk_scan<true>(m, tn, lane);
        // U / 2 chunks of 8 entries: U 16-byte loads in flight per lane, as
        // in the tail side (more raise the registers above 64 and cost
        // this kernel a CTA per SM).
        stream_pass_keyed<(U > 1 ? U / 2 : 1)>(g, m, tn, 0, 1, lane, geo, out, nullptr);
      }
      __syncwarp();
    }
    pc.drain(out);
    __syncwarp();
  }
  flush();
  if (!kVC) flush_counts<256>(tc, ctr);
}

// Head vertices of the block and large classes: one CTA per vertex from a
// dynamic queue, N+(v) (up to `cap` entries, `nb` buckets) and up to `cap`
// in-arcs at a time staged in dynamic shared memory.
template <int THREADS, class Sink, bool kTime, int U>
__global__ void __launch_bounds__(THREADS) k_head_block(Csr g, HeadArcs h,
                                                        const uint32_t* __restrict__ hl,
                                                        uint32_t hclass, uint32_t cap, uint32_t nb,
                                                        uint32_t hf,
                                                        unsigned long long* __restrict__ ctr,
                                                        Sink sink, ArcTimes at) {
  constexpr bool kVC = Sink::kPerVertex;
  constexpr uint32_t kWarps = THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t scan_tmp[THREADS / 32 + 2];
  __shared__ uint32_t s_item;
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const StageMem m = StageMem::carve(smem, cap, nb);
  const uint32_t* list = hl + kHeadPlanWords + hl[hclass];
  const uint32_t cnt = hl[kHeadPlanCount + hclass];
  unsigned long long* queue = ctr + C_HEAD_QUEUE + hclass;
  uint32_t* next = scan_tmp + kWarps + 1;  // the stream's claim counter
  TypeCounts tc;
  // Per-key counts as in k_head_warp, reduced over the CTA at a key change.
  uint32_t cur = 0xFFFFFFFFu;
  auto flush = [&]() {
    if (kVC && cur != 0xFFFFFFFFu) {
      block_key_flush<THREADS>(tc, cur, sink);
      tc = TypeCounts{};
    }
  };
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (uint32_t)atomicAdd(queue, 1ull);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= cnt) break;
    uint32_t v, j1;
    const uint32_t j00 = list[item];
    h.item(j00, hclass, v, j1);
    const uint64_t vb = g.off[v];
    const uint32_t d = (uint32_t)(g.off[v + 1] - vb);
    if (d > cap) {  // uniform over the CTA
      if (threadIdx.x == 0) atomicExch(ctr + C_ERROR, kErrStageCapacity);
      continue;
    }
    if (kVC) {
      const uint32_t key = sink.key(v);  // uniform over the CTA
      if (key != cur) {
        flush();
        cur = key;
      }
    }
    const Geo geo = Geo::of(d, nb, hf);
    stage_hash<THREADS>(g, vb, d, threadIdx.x, m, geo, BlockSync{});
    TypeCounts& out = tc;
    PackedCounts pc;
    for (uint32_t j0 = j00; j0 < j1; j0 += cap) {
      const uint32_t tn = min(cap, j1 - j0);
      // Every warp left the previous tile's stream (barrier at its end), and
      // the staging below passes a barrier before the counter is used.
      if (threadIdx.x == 0) *next = 0;
      stage_in_arcs<THREADS>(g, h, j0, tn, threadIdx.x, m, BlockSync{});
      if (kTime) {
        timed_head_pass(g, h, m, tn, d, w, kWarps, lane, geo, pc, out, at);
      } else {
        block_chunk_scan<THREADS, true>(m, tn, scan_tmp);
        // U chunks of 8 entries: 2 U 16-byte loads in flight per lane.
        stream_pass_keyed<U>(g, m, tn, w, kWarps, lane, geo, out, next);
      }
      __syncthreads();
    }
    pc.drain(out);
  }
  flush();
  if (!kVC) flush_counts<THREADS>(tc, ctr);
}

// Device buffers of the head-side pass (allocated before any capture).
struct HeadBufs {
  uint64_t* keys = nullptr;
  uint64_t* alt = nullptr;
  uint32_t* aend = nullptr;
  uint32_t* runs = nullptr;  // end of each head's run (n)
  uint32_t* hl = nullptr;    // plan words, class lists of work items
  uint8_t* need = nullptr;   // per tail: it keeps arcs for the tail side
  uint32_t* sort_counts = nullptr;
};

HeadBufs head_buffers(stc_ctx* c, const DeviceGraph& g) {
  HeadBufs b;
  b.keys = buffer<uint64_t>(c, B_KEYS_A, g.m_fwd);
  b.alt = buffer<uint64_t>(c, B_KEYS_B, g.m_fwd);
  b.aend = buffer<uint32_t>(c, B_HEAD_END, g.m_fwd);
  b.runs = buffer<uint32_t>(c, B_HEAD_RUNS, g.n);
  // Items: at most one per run (head) plus one per multiple of the
  // smallest item size.
  const size_t items = (size_t)g.n + g.m_fwd / kHeadItemMin + 1;
  b.hl = buffer<uint32_t>(c, B_HEAD_LIST, kHeadPlanWords + items + (g.n + 3) / 4);
  b.need = reinterpret_cast<uint8_t*>(b.hl + kHeadPlanWords + items);
  b.sort_counts = buffer<uint32_t>(c, B_SORT_COUNTS, (size_t)kRadix * kMaxSortGrid);
  return b;
}

// Shared-memory limits of the head-class kernels a head-side pass with this
// tuning launches; called before the pass is enqueued (or captured).
template <class Sink, bool kTime>
void prepare_head(const Tuning& tu) {
  const size_t sb =
      block_stage_bytes(kBlockCap, fit_hash_factor(tu.hash_factor[1], kBlockCap) * kBlockCap);
  const size_t sl =
      block_stage_bytes(kLargeCap, fit_hash_factor(tu.hash_factor[2], kLargeCap) * kLargeCap);
  with_block_threads(kTime ? 256 : tu.block_threads, [&](auto T) {
    with_unroll(kTime ? kStreamUnroll : tu.unroll[1], [&](auto U) {
      constexpr int kT = decltype(T)::value, kU = decltype(U)::value;
      if constexpr (!kTime || (kT == 256 && kU == kStreamUnroll))
        STC_CUDA(cudaFuncSetAttribute(k_head_block<kT, Sink, kTime, kU>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
    });
  });
  with_unroll(kTime ? kStreamUnroll : tu.unroll[2], [&](auto U) {
    constexpr int kU = decltype(U)::value;
    if constexpr (!kTime || kU == kStreamUnroll)
      STC_CUDA(cudaFuncSetAttribute(k_head_block<512, Sink, kTime, kU>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl));
  });
}

// The head-side pass is enqueued on `st` (no host synchronisation) in two
// parts: the keys (before the tail side is classified, which skips the
// tails left without arcs), then the sort, runs, plan and the three
// head-class kernels.  The launch parameters of the block and large classes
// follow the tuning of the tail side's same classes.
inline void enqueue_head_keys(cudaStream_t st, const Csr& csr, const uint32_t* asrc,
                              const uint32_t* fdeg, uint64_t m,
                              const unsigned long long* m_dev, const HeadBufs& b,
                              const uint8_t* d_tables,
                              const unsigned long long* range, unsigned long long* ctr,
                              int& launches) {
  STC_CUDA(cudaMemsetAsync(ctr + C_HEAD_COUNT, 0, 9 * sizeof(unsigned long long), st));
  STC_CUDA(cudaMemsetAsync(ctr + C_HEAD_NKEYS, 0, sizeof(unsigned long long), st));
  STC_CUDA(cudaMemsetAsync(b.need, 0, csr.n, st));
  const uint32_t grid = (uint32_t)std::min<uint64_t>((m + 1023) / 1024, kSMs * 8);
  uint8_t* fbkt = reinterpret_cast<uint8_t*>(b.runs);  // free until the runs are found
  k_fdeg_bucket<<<kSMs * 8, 256, 0, st>>>(fdeg, csr.n, fbkt);
  k_head_keys<<<std::max(1u, grid), 256, 0, st>>>(csr, asrc, fbkt, m, m_dev, d_tables, range,
                                                  b.keys, b.aend, b.need, ctr);
  launches += 2;
}

template <class Sink, bool kTime>
void enqueue_head(cudaStream_t st, const Csr& csr, const uint32_t* asrc, uint64_t m,
                  const HeadBufs& b, unsigned long long* ctr, const Sink& sink,
                  const ArcTimes& at, const Tuning& tu, int& launches,
                  uint32_t class_mask = 0x3F) {
  const uint32_t n = csr.n;
  const uint32_t vbits = std::max<uint32_t>(1, bit_width64(n - 1));
  int sort_launches = 0;
  const uint64_t* sorted = radix_sort(b.keys, b.alt, m, 32, 32 + (int)vbits, b.sort_counts, st,
                                      &sort_launches, ctr + C_HEAD_NKEYS);
  uint32_t* end = b.runs;
  k_head_runs<false><<<kSMs * 4, 256, 0, st>>>(sorted, csr.off, ctr, b.hl, end);
  k_head_plan<<<1, 32, 0, st>>>(ctr, b.hl);
  k_head_runs<true><<<kSMs * 4, 256, 0, st>>>(sorted, csr.off, ctr, b.hl, end);
  const HeadArcs h{sorted, b.aend, end, asrc};
  launches += 3 + sort_launches;
  // Head class c runs with class_mask bit c + 1, as the tail side's class of
  // the same tuning (the autotuner times one class at a time).
  with_unroll(kTime ? kStreamUnroll : tu.unroll[0], [&](auto U) {
    constexpr int kU = decltype(U)::value;
    if constexpr (!kTime || kU == kStreamUnroll)
      if (class_mask & 2u)
        k_head_warp<Sink, kTime, kU><<<kSMs * 4, 256, 0, st>>>(csr, h, b.hl, ctr, sink, at,
                                                               tu.hash_factor[0]);
  });
  if (class_mask & 4u) {
    const uint32_t cap = kBlockCap;
    const uint32_t hf = fit_hash_factor(tu.hash_factor[1], cap);
    const uint32_t nb = hf * cap;
    const size_t smem = block_stage_bytes(cap, nb);
    with_block_threads(kTime ? 256 : tu.block_threads, [&](auto T) {
      with_unroll(kTime ? kStreamUnroll : tu.unroll[1], [&](auto U) {
        constexpr int kT = decltype(T)::value, kU = decltype(U)::value;
        if constexpr (!kTime || (kT == 256 && kU == kStreamUnroll)) {
          const uint32_t per_sm = smem <= 110 * 1024 ? 2 : 1;
          k_head_block<kT, Sink, kTime, kU><<<kSMs * per_sm, kT, smem, st>>>(
              csr, h, b.hl, 1, cap, nb, hf, ctr, sink, at);
        }
      });
    });
  }
  if (class_mask & 8u) {
    const uint32_t cap = kLargeCap;
    const uint32_t hf = fit_hash_factor(tu.hash_factor[2], cap);
    const uint32_t nb = hf * cap;
    const size_t smem = block_stage_bytes(cap, nb);
    with_unroll(kTime ? kStreamUnroll : tu.unroll[2], [&](auto U) {
      constexpr int kU = decltype(U)::value;
      if constexpr (!kTime || kU == kStreamUnroll)
        k_head_block<512, Sink, kTime, kU><<<kSMs, 512, smem, st>>>(csr, h, b.hl, 2, cap, nb, hf,
                                                                     ctr, sink, at);
    });
  }
  launches += 3;
  STC_CUDA(cudaGetLastError());
}

// ------------------------------------------------------- persistent ----
// The persistent engine: the whole count as one sequence without host
// synchronisation, so that it can be captured once in a CUDA graph and
// replayed.  The class lists are planned on the device (k_plan); one
// persistent kernel of 256-thread CTAs then drains two device work queues:
// first the block-class lists, one per CTA at a time; then, with no further
// CTA barriers, each warp takes a warp-class list or 32 tiny lists (one per
// lane) at a time.  Large and giant lists, rare in the small graphs a batch
// holds, keep their own kernels, which read their counts from the plan.
__global__ void k_plan(unsigned long long* __restrict__ ctr, uint32_t* __restrict__ plan) {
  if (threadIdx.x != 0) return;
  uint32_t start = 0;
  for (int c = 0; c < kClasses; c++) {
    const uint32_t cnt = (uint32_t)ctr[C_WORK + c];
    plan[c] = start;
    plan[kPlanCounts + c] = cnt;
    start += cnt;
  }
  plan[kClasses] = start;
  for (int i = 0; i < 8; i++) ctr[C_WORK + i] = 0;  // fill cursors and work queues
  ctr[C_QUEUE_WARP] = 0;
}

constexpr size_t kPersistentSmem =
    StageMem::bytes(kBlockCap, 4 * kBlockCap) > 8 * kWarpStageBytes
        ? StageMem::bytes(kBlockCap, 4 * kBlockCap)
        : 8 * kWarpStageBytes;

template <class Sink>
__global__ void __launch_bounds__(256, 4) k_persistent(Csr g, const uint32_t* __restrict__ lists,
                                                       const uint32_t* __restrict__ plan,
                                                       unsigned long long* __restrict__ ctr, Sink sink,
                                                       const uint8_t* __restrict__ gtables) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint8_t tw[16][16], tb[16][16];
  __shared__ uint32_t scan_tmp[256 / 32 + 2];
  __shared__ uint32_t s_item;
  (&tw[0][0])[threadIdx.x] = gtables[256 * kTableWarp + threadIdx.x];
  (&tb[0][0])[threadIdx.x] = gtables[256 * kTableBlock + threadIdx.x];
  const uint32_t nt = plan[kPlanCounts + 0], nw = plan[kPlanCounts + 1], nb = plan[kPlanCounts + 2];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  TypeCounts tc;
  // Phase 1: block-class lists, the whole CTA on each.
  const StageMem mb = StageMem::carve(smem, kBlockCap, 4 * kBlockCap);
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (uint32_t)atomicAdd(ctr + C_WORK + 5, 1ull);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= nb) break;
    block_vertex<256, Sink, false, kStreamUnroll, false>(g, lists[plan[2] + item], kBlockCap,
                                                  4 * kBlockCap, 4, mb, tb, scan_tmp, ctr, sink,
                                                  ArcTimes{nullptr, nullptr}, kTableBlock, tc);
  }
  // Phase 2: warp-granular items.  Every warp of the CTA has left phase 1
  // (the exit above is uniform), so the slices no longer alias mb in use.
  const StageMem mw = StageMem::carve(smem + w * kWarpStageBytes, kWarpCap, kWarpBuckets);
  const uint32_t total = nw + (nt + 31) / 32;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = (uint32_t)atomicAdd(ctr + C_QUEUE_WARP, 1ull);
    item = __shfl_sync(kFull, item, 0);
    if (item >= total) break;
    if (item < nw) {
      warp_vertex<Sink, false, kStreamUnroll, false>(g, lists[plan[1] + item], lane, mw, tw, 4, ctr,
                                                     sink,
                                              ArcTimes{nullptr, nullptr}, tc);
    } else {
      const uint32_t idx = (item - nw) * 32 + lane;
      if (idx < nt) tiny_vertex<kTinyMax>(g, lists[plan[0] + idx], sink, tw, tc);
    }
  }
  if (!Sink::kPerVertex) flush_counts<256>(tc, ctr);
}

// The head-side pass of a persistent count: its buffers and the arcs.
struct HeadPlan {
  const HeadBufs* bufs = nullptr;  // null: the tables send no arc to the head side
  const uint32_t* asrc = nullptr;
  const uint32_t* fdeg = nullptr;
  uint64_t m = 0;
  const unsigned long long* m_dev = nullptr;  // arc count on the device when m is a capacity
  Tuning tuning;
};

// Enqueues the persistent sequence on `st` (no host synchronisation).
template <class Sink>
void enqueue_persistent(cudaStream_t st, const Csr& csr, const ClassBounds& cb, uint32_t* lists,
                        uint32_t* plan, unsigned long long* ctr, const uint8_t* d_tables,
                        const Sink& sink, const HeadPlan& hp, int& launches) {
  const ArcTimes none{nullptr, nullptr};
  const uint8_t* need = nullptr;
  if (hp.bufs) {
    enqueue_head_keys(st, csr, hp.asrc, hp.fdeg, hp.m, hp.m_dev, *hp.bufs, d_tables, nullptr, ctr,
                      launches);
    need = hp.bufs->need;
  }
  STC_CUDA(cudaMemsetAsync(ctr + C_WORK, 0, 8 * sizeof(uint64_t), st));
  k_classify_count<<<kSMs * 4, 256, 0, st>>>(csr.off, csr.n, cb, ctr, nullptr, need);
  k_plan<<<1, 32, 0, st>>>(ctr, plan);
  k_classify_fill<<<kSMs * 4, 256, 0, st>>>(csr.off, csr.n, cb, lists, plan, ctr + C_WORK, nullptr,
                                            need);
  k_persistent<Sink><<<kSMs * 4, 256, kPersistentSmem, st>>>(csr, lists, plan, ctr, sink,
                                                             d_tables);
  k_block<512, Sink, false, kStreamUnroll, false>
      <<<kSMs, 512, StageMem::bytes(kLargeCap, 2 * kLargeCap), st>>>(
      csr, lists, 0, kLargeCap, 2 * kLargeCap, 2, ctr + C_WORK + 6, ctr, sink,
      d_tables + 256 * kTableLarge, none, kTableLarge, plan, 3);
  k_giant<512, Sink, false><<<kSMs * 2, 512, 0, st>>>(csr, lists, 0, ctr + C_WORK + 7, ctr, sink,
                                                      d_tables + 256 * kTableGiant, none, plan, 4);
  launches += 6;
  if (hp.bufs)
    enqueue_head<Sink, false>(st, csr, hp.asrc, hp.m, *hp.bufs, ctr, sink, none, hp.tuning,
                              launches);
  STC_CUDA(cudaGetLastError());
}

// Identity of a captured persistent sequence: every pointer and size its
// kernels were given.
struct PersistentKey {
  const void* p[17];
  uint64_t v[6];
};

template <class Sink>
void count_persistent(stc_ctx* c, const Csr& csr, const ClassBounds& cb, uint32_t* lists,
                      uint32_t* plan, unsigned long long* ctr, const uint8_t* d_tables,
                      const Sink& sink, const void* s0, const void* s1, uint64_t s2,
                      const HeadPlan& hp) {
  cudaStream_t st = c->stream;
  STC_CUDA(cudaFuncSetAttribute(k_persistent<Sink>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kPersistentSmem));
  STC_CUDA(cudaFuncSetAttribute(k_block<512, Sink, false, kStreamUnroll, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)StageMem::bytes(kLargeCap, 2 * kLargeCap)));
  if (hp.bufs) prepare_head<Sink, false>(hp.tuning);
  // The legacy default stream cannot be captured: launch directly there.
  // So does a count that is itself being captured (a batch group's whole
  // pipeline) or that reads its arc count on the device (the one capped
  // run that sizes such a pipeline's buffers).
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread)
    STC_CUDA(cudaStreamIsCapturing(st, &cs));
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread ||
      cs != cudaStreamCaptureStatusNone || hp.m_dev) {
    enqueue_persistent(st, csr, cb, lists, plan, ctr, d_tables, sink, hp, c->launches);
    return;
  }
  PersistentKey key{};
  const HeadBufs hb = hp.bufs ? *hp.bufs : HeadBufs{};
  const void* ptrs[17] = {csr.off, csr.nbr, csr.sgn, csr.verts, lists, plan, ctr, d_tables, s0,
                          hp.asrc, hb.keys, hb.alt, hb.aend, hb.runs, hb.hl, hp.fdeg, csr.nkey};
  memcpy(key.p, ptrs, sizeof(ptrs));
  key.v[0] = csr.n;
  key.v[1] = cb.tiny_max;
  key.v[2] = s2;
  key.v[3] = reinterpret_cast<uint64_t>(s1);
  key.v[4] = hp.m;
  key.v[5] = reinterpret_cast<uint64_t>(hb.sort_counts) ^
             ((uint64_t)hp.tuning.block_threads << 48) ^ ((uint64_t)hp.tuning.unroll[0] << 56) ^
             ((uint64_t)hp.tuning.unroll[1] << 58) ^ ((uint64_t)hp.tuning.unroll[2] << 60) ^
             ((uint64_t)hp.tuning.hash_factor[0] << 40) ^ ((uint64_t)hp.tuning.hash_factor[1] << 42) ^
             ((uint64_t)hp.tuning.hash_factor[2] << 44);
  static_assert(sizeof(PersistentKey) <= sizeof(c->graph_key), "graph key size");
  if (c->graph_exec && memcmp(c->graph_key, &key, sizeof(key)) == 0) {
    STC_CUDA(cudaGraphLaunch(c->graph_exec, st));
    c->launches += c->graph_launches;
    return;
  }
  if (c->graph_exec) {
    STC_CUDA(cudaGraphExecDestroy(c->graph_exec));
    c->graph_exec = nullptr;
  }
  int launches = 0;
  cudaGraph_t graph = nullptr;
  STC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_persistent(st, csr, cb, lists, plan, ctr, d_tables, sink, hp, launches);
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  STC_CUDA(cudaStreamEndCapture(st, &graph));
  const cudaError_t e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  STC_CUDA(e);
  memcpy(c->graph_key, &key, sizeof(key));
  c->graph_launches = launches;
  STC_CUDA(cudaGraphLaunch(c->graph_exec, st));
  c->launches += launches;
}

// ------------------------------------------------------------- split ----
// The sign-split copy of the arc heads (the layout of
// MC/tc_merge_sign_split.cpp:20-146 and GM/signed_tc.hxx:302-396, kept beside
// the sorted heads instead of replacing them): each list's positive heads,
// then its negative heads, both ascending; psplit[u] = positive heads of u.
// Each lane takes one vertex; a list of up to 32 heads is split by its lane
// alone (count the positives, then place every head), and the warp splits
// the longer lists of its 32 vertices together, 32 heads per step, placing
// them with ballots and the popcounts of the lanes below.
constexpr uint32_t kSplitShort = 32;

__global__ void k_split_csr(const uint64_t* __restrict__ off, const uint32_t* __restrict__ nbr,
                            const int8_t* __restrict__ sgn, uint32_t n,
                            uint32_t* __restrict__ out, uint32_t* __restrict__ psplit) {
  const uint32_t lane = lane_id();
  const uint32_t lt = lanemask_lt();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint32_t u = base + lane;
    const bool valid = u < n;
    const uint64_t b = valid ? off[u] : 0, e = valid ? off[u + 1] : 0;
    if (valid && e - b <= kSplitShort) {
      uint32_t pos = 0;
      for (uint64_t i = b; i < e; i++) pos += sgn[i] >= 0;
      uint32_t wp = 0, wn = 0;
      for (uint64_t i = b; i < e; i++) {
        const uint32_t x = nbr[i];
        if (sgn[i] >= 0) out[b + wp++] = x;
        else out[b + pos + wn++] = x;
      }
      psplit[u] = pos;
    }
    uint32_t longs = __ballot_sync(kFull, valid && e - b > kSplitShort);
    while (longs) {
      const int src = __ffs(longs) - 1;
      longs &= longs - 1;
      const uint64_t lb = __shfl_sync(kFull, b, src), le = __shfl_sync(kFull, e, src);
      uint32_t pos = 0;
      for (uint64_t at = lb; at < le; at += 32) {
        const uint64_t i = at + lane;
        pos += __popc(__ballot_sync(kFull, i < le && sgn[i] >= 0));
      }
      uint32_t wp = 0, wn = 0;
      for (uint64_t at = lb; at < le; at += 32) {
        const uint64_t i = at + lane;
        const bool in = i < le;
        const bool p = in && sgn[i] >= 0;
        const uint32_t bp = __ballot_sync(kFull, p), bn = __ballot_sync(kFull, in && !p);
        if (p) out[lb + wp + __popc(bp & lt)] = nbr[i];
        else if (in) out[lb + pos + wn + __popc(bn & lt)] = nbr[i];
        wp += __popc(bp);
        wn += __popc(bn);
      }
      if (lane == 0) psplit[base + src] = pos;
    }
  }
}

// ------------------------------------------------------------ shards ----
// A shard of a count is a contiguous range of source vertices in rank space
// chosen so that the shards carry about the same merge-model cost: vertex u
// costs 1 + sum over v in N+(u) of (d+(u) + d+(v)), saturated at 2^32 - 1.
// With P(r) the cost of the ranks below r, shard s of S starts at the first
// rank r with P(r) >= ceil(P(n) s / S).  Every triangle is counted by the
// shard of its lowest-ranked vertex, so the shards' counts add up to the
// whole graph's.
struct VertexCost {
  const uint64_t* off;
  const uint32_t* nbr;
  __device__ uint32_t operator()(uint64_t u) const {
    const uint64_t b = off[u], e = off[u + 1], du = e - b;
    uint64_t cost = 1;
    for (uint64_t i = b; i < e; i++) {
      const uint32_t v = nbr[i];
      cost += du + (off[v + 1] - off[v]);
    }
    return (uint32_t)(cost < 0xFFFFFFFFull ? cost : 0xFFFFFFFFull);
  }
};
struct EmitPrefix {
  uint64_t* pre;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t) const { pre[i] = pos; }
};

// Thread 0 writes the shard's first rank, thread 1 its end.
__global__ void k_shard_bounds(const uint64_t* __restrict__ pre, uint32_t n, uint32_t shard,
                               uint32_t shards, unsigned long long* __restrict__ ctr) {
  if (threadIdx.x > 1) return;
  const uint32_t s = shard + threadIdx.x;
  uint32_t r = 0;
  if (s >= shards) {
    r = n;
  } else if (s > 0) {
    const uint64_t target = (pre[n] * s + shards - 1) / shards;
    uint32_t lo = 0, hi = n;  // first r with pre[r] >= target (pre[n] = total)
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo) >> 1);
      if (pre[mid] < target) lo = mid + 1; else hi = mid;
    }
    r = lo;
  }
  ctr[C_SHARD_LO + threadIdx.x] = r;
}

// Writes the rank range of cfg.shard into the counters (device side only).
void shard_range(stc_ctx* c, const DeviceGraph& g, uint32_t shard, uint32_t shards) {
  uint64_t* pre = buffer<uint64_t>(c, B_SHARD_COST, (size_t)g.n + 1);
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  range_scan(VertexCost{g.off, g.nbr}, EmitPrefix{pre}, g.n, sums, c->stream, &c->launches);
  STC_CUDA(cudaMemcpyAsync(pre + g.n, sums + range_partition(g.n, kScanTile, kMaxSortGrid).grid,
                           sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
  k_shard_bounds<<<1, 32, 0, c->stream>>>(pre, g.n, shard, shards, (unsigned long long*)counters(c));
  c->launches++;
}

}  // namespace

// Fixed degree-threshold dispatch: HEAD when A' is not the longer list
// (bucket |A'| <= bucket |B|) and |B| <= 4095 (for lists of the warp class,
// which also decides tiny lists, only when |B| >= 8: short arcs of short
// lists cost less on the tail side than an entry in the head side's sort,
// while a longer list would be staged there for a handful of them), SEARCH
// when B is at least 16x longer than A', MERGE when both are short, HASH
// otherwise (the giant class, which stages no hash, merges instead of
// hashing).  Without `head`, the tail-side table of the first version (no
// HEAD cells), which per-vertex counts and the no-allocation path use.
void fixed_dispatch_tables(uint8_t* out, bool head) {
  for (int t = 0; t < kTableClasses; t++)
    for (int a = 0; a < 16; a++)
      for (int b = 0; b < 16; b++) {
        uint8_t s = STC_STRATEGY_HASH;
        const int bmin = t == kTableWarp ? 4 : 1;
        if (head && b >= bmin && b <= 12 && a <= b) s = STC_STRATEGY_HEAD;
        else if (b >= a + 4) s = STC_STRATEGY_SEARCH;
        else if (a <= 3 && b <= 5) s = STC_STRATEGY_MERGE;
        out[256 * t + 16 * a + b] = s;
      }
}

namespace {
// Cached tables in B_DISPATCH_FIXED: the fixed tables with and without HEAD,
// and the forced-HEAD tables (HEAD wherever it applies, HASH elsewhere).
enum { kFixedHead = 0, kFixedNoHead = 1, kForcedHead = 2, kCachedTables = 3 };
}  // namespace

// Device copy of the dispatch tables a call uses: a forced strategy fills
// every cell (HEAD only the cells where it applies); otherwise the learned
// tables when the context holds a model and the call asks for them, else
// the fixed ones.  Per-vertex counts take tables without HEAD (the head
// side reports per graph, not per source vertex).  `uses_head` (optional)
// receives whether the tables send any cell to the head side.
const uint8_t* dispatch_tables(stc_ctx* c, const CountConfig& cfg, bool* uses_head) {
  const bool head_ok = cfg.vertex_counts == nullptr;
  if (uses_head) *uses_head = false;
  if (!c->fixed_ready) {
    uint8_t h[kCachedTables * kTableBytes];
    fixed_dispatch_tables(h + kFixedHead * kTableBytes, true);
    fixed_dispatch_tables(h + kFixedNoHead * kTableBytes, false);
    for (size_t i = 0; i < kTableBytes; i++)
      h[kForcedHead * kTableBytes + i] =
          (i & 15) <= 12 ? (uint8_t)STC_STRATEGY_HEAD : (uint8_t)STC_STRATEGY_HASH;
    uint8_t* t = buffer<uint8_t>(c, B_DISPATCH_FIXED, sizeof(h));
    STC_CUDA(cudaMemcpyAsync(t, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    STC_CUDA(cudaStreamSynchronize(c->stream));  // `h` is pageable and leaves scope
    c->fixed_ready = true;
  }
  const uint8_t* cached = buffer<uint8_t>(c, B_DISPATCH_FIXED, kCachedTables * kTableBytes);
  if (cfg.strategy == STC_STRATEGY_HEAD) {
    if (uses_head) *uses_head = head_ok;
    if (head_ok) return cached + kForcedHead * kTableBytes;
    uint8_t* t = buffer<uint8_t>(c, B_WORK2, kTableBytes);
    STC_CUDA(cudaMemsetAsync(t, (int)STC_STRATEGY_HASH, kTableBytes, c->stream));
    return t;
  }
  if (cfg.strategy != STC_STRATEGY_AUTO) {
    uint8_t* t = buffer<uint8_t>(c, B_WORK2, kTableBytes);
    STC_CUDA(cudaMemsetAsync(t, (int)cfg.strategy, kTableBytes, c->stream));
    return t;
  }
  if (!head_ok) return cached + kFixedNoHead * kTableBytes;
  if (cfg.dispatch == STC_DISPATCH_LEARNED && c->model_loaded) {
    if (uses_head) *uses_head = c->learned_uses_head;
    return buffer<uint8_t>(c, B_DISPATCH, kTableBytes);
  }
  if (uses_head) *uses_head = true;
  return cached + kFixedHead * kTableBytes;
}

// Builds the sign-split copy of g's heads on the context's stream.
void build_split(stc_ctx* c, DeviceGraph& g) {
  g.nbr_split = buffer<uint32_t>(c, B_SPLIT_NBR, g.m_fwd + 4);
  g.psplit = buffer<uint32_t>(c, B_SPLIT_POS, g.n);
  STC_CUDA(cudaMemsetAsync(g.nbr_split + g.m_fwd, 0, 4 * sizeof(uint32_t), c->stream));
  k_split_csr<<<kSMs * 8, 256, 0, c->stream>>>(g.off, g.nbr, g.sgn, g.n, g.nbr_split, g.psplit);
  c->launches++;
  STC_CUDA(cudaGetLastError());
}

void count_triangles(stc_ctx* c, const DeviceGraph& gin, const CountConfig& cfg) {
  if (gin.n == 0 || gin.m_fwd == 0) return;
  cudaStream_t st = c->stream;
  DeviceGraph g = gin;
  const bool split = cfg.strategy == STC_STRATEGY_SPLIT ||
                     (cfg.strategy == STC_STRATEGY_AUTO && cfg.dispatch == STC_DISPATCH_LEARNED &&
                      c->model_loaded && c->learned_uses_split);
  if (split) build_split(c, g);
  Csr csr{g.off, g.nbr, g.sgn, g.verts, g.n, g.nbr_split, g.psplit, g.nkey};
  unsigned long long* ctr = (unsigned long long*)counters(c);
  bool uses_head = false;
  const uint8_t* d_table = dispatch_tables(c, cfg, &uses_head);
  // The head-side pass runs when the tables send arcs there (never for
  // per-vertex counts, whose tables have no HEAD cells).
  const bool head = uses_head && (cfg.class_mask & 0x20u) && g.asrc != nullptr &&
                    g.nkey != nullptr && g.n >= 2;
  HeadBufs hb;
  if (head) hb = head_buffers(c, g);
  const bool timed = cfg.arc_cycles != nullptr;
  const ArcTimes at{(unsigned long long*)cfg.arc_cycles, (unsigned long long*)cfg.arc_counts};
  const unsigned long long* range = nullptr;
  if (cfg.shards > 1) {
    shard_range(c, g, cfg.shard, cfg.shards);
    range = ctr + C_SHARD_LO;
  }

  // Vertex classes (a forced strategy disables the tiny class, which only
  // implements the search form; so does timing, so that every strategy's
  // timings cover the same arcs).
  const bool tiny =
      !timed && (cfg.strategy == STC_STRATEGY_AUTO || cfg.strategy == STC_STRATEGY_SEARCH);
  const ClassBounds cb{tiny ? kTinyMax : 1u, kWarpCap, kBlockCap, kLargeCap};

  // The persistent engine has no SPLIT path: counts that use SPLIT take the
  // per-class kernels.
  if (cfg.persistent && !timed && cfg.shards <= 1 && !split) {
    uint32_t* lists = buffer<uint32_t>(c, B_WORK, (size_t)g.n + kPlanWords + 8);
    uint32_t* plan = lists + g.n + 4;
    HeadPlan hp;
    if (head) {
      hp.bufs = &hb;
      hp.asrc = g.asrc;
      hp.fdeg = g.fdeg;
      hp.m = g.m_fwd;
      hp.m_dev = g.m_dev;
      hp.tuning = c->tuning;
    }
    if (cfg.vertex_counts) {
      const VertexSink sink{(unsigned long long*)cfg.vertex_counts, g.verts};
      count_persistent(c, csr, cb, lists, plan, ctr, d_table, sink, sink.vcounts, nullptr, 1, hp);
    } else if (cfg.graph_counts) {
      const GraphSink sink{(unsigned long long*)cfg.graph_counts, g.gbase, g.G};
      count_persistent(c, csr, cb, lists, plan, ctr, d_table, sink, sink.gcounts, sink.gbase,
                       2 + ((uint64_t)g.G << 8), hp);
    } else {
      count_persistent(c, csr, cb, lists, plan, ctr, d_table, TotalSink{}, nullptr, nullptr, 0,
                       hp);
    }
    return;
  }
  const uint8_t* need = nullptr;
  if (head) {
    enqueue_head_keys(st, csr, g.asrc, g.fdeg, g.m_fwd, g.m_dev, hb, d_table, range, ctr,
                      c->launches);
    need = hb.need;
  }
  k_classify_count<<<kSMs * 4, 256, 0, st>>>(g.off, g.n, cb, ctr, range, need);
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, counters(c) + C_WORK,
                           (C_MAX_FDEG + 1 - C_WORK) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  const uint32_t max_fdeg = (uint32_t)c->h_pinned[C_MAX_FDEG];
  uint32_t counts[kClasses], starts[kClasses + 1];
  starts[0] = 0;
  for (int i = 0; i < kClasses; i++) {
    counts[i] = (uint32_t)c->h_pinned[C_WORK + i];
    starts[i + 1] = starts[i] + counts[i];
  }
  uint32_t* lists = buffer<uint32_t>(c, B_WORK, (size_t)starts[kClasses] + 8);
  uint32_t* d_starts = lists + starts[kClasses];
  STC_CUDA(cudaMemcpyAsync(d_starts, starts, kClasses * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  // Cursors of the fill, then the dynamic queues, live in C_WORK ...
  STC_CUDA(cudaMemsetAsync(counters(c) + C_WORK, 0, 8 * sizeof(uint64_t), st));
  k_classify_fill<<<kSMs * 4, 256, 0, st>>>(g.off, g.n, cb, lists, d_starts, ctr + C_WORK, range,
                                            need);
  STC_CUDA(cudaMemsetAsync(counters(c) + C_WORK, 0, 8 * sizeof(uint64_t), st));
  c->launches += 2;

  auto run = [&](const auto& sink, auto time_tag) {
    using Sink = std::decay_t<decltype(sink)>;
    constexpr bool kT = decltype(time_tag)::value;
    launch_classes<Sink, kT>(st, csr, lists, counts, starts, max_fdeg, ctr, d_table, sink, at,
                             c->tuning, cfg.class_mask, c->launches);
    if (head) {
      prepare_head<Sink, kT>(c->tuning);
      enqueue_head<Sink, kT>(st, csr, g.asrc, g.m_fwd, hb, ctr, sink, at, c->tuning,
                             c->launches, cfg.class_mask);
    }
  };
  if (timed) {
    run(TotalSink{}, std::true_type{});
  } else if (cfg.vertex_counts) {
    run(VertexSink{(unsigned long long*)cfg.vertex_counts, g.verts}, std::false_type{});
  } else if (cfg.graph_counts) {
    run(GraphSink{(unsigned long long*)cfg.graph_counts, g.gbase, g.G}, std::false_type{});
  } else {
    run(TotalSink{}, std::false_type{});
  }
  STC_CUDA(cudaGetLastError());
}

}  // namespace stc

// ===================================================== no-allocation path ===
// stc_count_oriented_csr_noalloc counts an oriented forward CSR that already
// sits in device memory without allocating anything: for callers that cannot
// call cudaMalloc (code running under a custom device allocator or inside a
// memory budget it does not control).  Its scratch (vertex worklists, the
// dispatch table, counters) lives in one file-scope device array of fixed
// size; every GPU that loads the library holds that array until exit, every
// call shares it, and calls that overlap on the GPU race on it.
namespace stc {
namespace {

constexpr uint32_t kNoAllocMaxVertices = 1u << 22;  // 16 MiB of worklists
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
  unsigned long long ctr[C_SLOTS];
  uint8_t table[kTableBytes];
  uint32_t lists[kNoAllocMaxVertices + 8];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Input checks on the device, in two grid-stride passes with coalesced
// reads and no per-list loop, so that a long list (a hub keeps its whole
// degree under an id-ordered orientation) costs no more than other entries.
// Any violation sets ctr[C_ERROR] = kDeviceErrCsr.
// Per vertex: offsets start at 0, never decrease and end at m, and the first
// head of a non-empty list is above its tail.
__global__ void k_check_offsets(const uint64_t* __restrict__ off, const uint32_t* __restrict__ heads,
                                uint32_t n, uint64_t m, unsigned long long* __restrict__ ctr) {
  const uint32_t stride = gridDim.x * blockDim.x;
  if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || off[n] != m))
    atomicExch(ctr + C_ERROR, (unsigned long long)kDeviceErrCsr);
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    const uint64_t b = off[u], e = off[u + 1];
    const bool bad = e < b || e > m || (e > b && heads[b] <= u);
    if (bad) atomicExch(ctr + C_ERROR, (unsigned long long)kDeviceErrCsr);
  }
}

// Per arc: every head is below n and above the head before it, unless it
// starts its list (then the pass above compared it with its tail).  Only a
// head not above its predecessor looks up its list, by a binary search of
// the offsets: in a valid CSR that happens at most once per list.
__global__ void k_check_heads(const uint64_t* __restrict__ off, const uint32_t* __restrict__ heads,
                              uint32_t n, uint64_t m, unsigned long long* __restrict__ ctr) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t h = heads[i];
    bool bad = h >= n;
    if (!bad && i > 0 && h <= heads[i - 1]) {
      uint32_t lo = 0, hi = n;  // largest u in [0, n) with off[u] <= i
      while (hi - lo > 1) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (off[mid] <= i) lo = mid; else hi = mid;
      }
      bad = off[lo] != i;  // i must start the list of u
    }
    if (bad) atomicExch(ctr + C_ERROR, (unsigned long long)kDeviceErrCsr);
  }
}

// The scratch array's device address in the current context.  It is looked
// up (cudaGetSymbolAddress) once per CUDA context: the first call in a
// context, with that context current, and again whenever the current
// context differs from the last one seen on that device, as after
// cudaDeviceReset or under a caller's own context.  Contexts are told apart
// by the driver's context id, reached through the runtime's driver entry
// points (so libstc needs no link to the driver library); without them the
// address is looked up on every call.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_noalloc_mu;
struct NoAllocSlot {
  unsigned long long ctx_id = 0;
  bool valid = false;
  void* addr = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

bool current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) ==
            cudaSuccess &&
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) ==
            cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    (void)cudaGetLastError();
  }
  if (!get_current || !get_id) return false;
  CUcontext cx = nullptr;
  if (get_current(&cx) != CUDA_SUCCESS || cx == nullptr) return false;
  return get_id(cx, id) == CUDA_SUCCESS;
}

cudaError_t noalloc_scratch(int device, NoAllocScratch** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  NoAllocSlot& slot = g_noalloc_slot[device];
  if (!have_id || !slot.valid || slot.ctx_id != id) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    slot.addr = p;
    slot.ctx_id = id;
    slot.valid = have_id;
  }
  *out = static_cast<NoAllocScratch*>(slot.addr);
  return cudaSuccess;
}

stc_status noalloc_cuda(cudaError_t e) {
  (void)cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? STC_ERR_OUT_OF_MEMORY : STC_ERR_CUDA;
}

}  // namespace

}  // namespace stc

#define STC_NA(call)                                   \
  do {                                                 \
    const cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return stc::noalloc_cuda(e_); \
  } while (0)

extern "C" stc_status stc_count_oriented_csr_noalloc(const uint64_t* d_offsets,
                                                      const uint32_t* d_heads,
                                                      const int8_t* d_signs, uint32_t n,
                                                      uint64_t m, void* stream, stc_counts* out) {
  using namespace stc;
  if (!out || !d_offsets || (m && (!d_heads || !d_signs))) return STC_ERR_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(d_heads) & 15) || (reinterpret_cast<uintptr_t>(d_signs) & 3))
    return STC_ERR_INVALID_ARGUMENT;
  if (n > kNoAllocMaxVertices || m >= (1ull << 32)) return STC_ERR_LIMIT;
  *out = stc_counts{0, 0, 0, 0};
  if (n == 0) return STC_OK;
  int device = 0;
  STC_NA(cudaGetDevice(&device));
  if (device < 0 || device >= kNoAllocMaxDevices) return STC_ERR_NO_DEVICE;
  NoAllocScratch* scr = nullptr;
  STC_NA(noalloc_scratch(device, &scr));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long* ctr = scr->ctr;
  STC_NA(cudaMemsetAsync(ctr, 0, sizeof(scr->ctr), st));
  k_check_offsets<<<kSMs * 4, 256, 0, st>>>(d_offsets, d_heads, n, m, ctr);
  if (m) k_check_heads<<<kSMs * 8, 256, 0, st>>>(d_offsets, d_heads, n, m, ctr);
  STC_NA(cudaGetLastError());
  uint64_t slots[C_SLOTS];
  STC_NA(cudaMemcpyAsync(slots, ctr, sizeof(slots), cudaMemcpyDeviceToHost, st));
  STC_NA(cudaStreamSynchronize(st));
  if (slots[C_ERROR]) return STC_ERR_INVALID_ARGUMENT;
  if (m == 0) return STC_OK;

  uint8_t table[kTableBytes];
  fixed_dispatch_tables(table, false);
  STC_NA(cudaMemcpyAsync(scr->table, table, sizeof(table), cudaMemcpyHostToDevice, st));
  const ClassBounds cb{kTinyMax, kWarpCap, kBlockCap, kLargeCap};
  k_classify_count<<<kSMs * 4, 256, 0, st>>>(d_offsets, n, cb, ctr, nullptr);
  STC_NA(cudaMemcpyAsync(slots, ctr, sizeof(slots), cudaMemcpyDeviceToHost, st));
  STC_NA(cudaStreamSynchronize(st));
  const uint32_t max_fdeg = (uint32_t)slots[C_MAX_FDEG];
  uint32_t counts[kClasses], starts[kClasses + 1];
  starts[0] = 0;
  for (int i = 0; i < kClasses; i++) {
    counts[i] = (uint32_t)slots[C_WORK + i];
    starts[i + 1] = starts[i] + counts[i];
  }
  uint32_t* lists = scr->lists;
  uint32_t* d_starts = lists + starts[kClasses];
  STC_NA(cudaMemcpyAsync(d_starts, starts, kClasses * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  STC_NA(cudaMemsetAsync(ctr + C_WORK, 0, 8 * sizeof(uint64_t), st));
  k_classify_fill<<<kSMs * 4, 256, 0, st>>>(d_offsets, n, cb, lists, d_starts, ctr + C_WORK,
                                            nullptr);
  STC_NA(cudaMemsetAsync(ctr + C_WORK, 0, 8 * sizeof(uint64_t), st));

  const Csr csr{d_offsets, d_heads, d_signs, nullptr, n, nullptr, nullptr};
  int launches = 0;
  try {
    launch_classes<TotalSink, false>(st, csr, lists, counts, starts, max_fdeg, ctr, scr->table,
                                     TotalSink{}, ArcTimes{nullptr, nullptr}, Tuning{}, 0x1Fu,
                                     launches);
  } catch (const Error& e) {
    (void)cudaGetLastError();
    return e.status;
  }
  STC_NA(cudaGetLastError());
  STC_NA(cudaMemcpyAsync(slots, ctr, sizeof(slots), cudaMemcpyDeviceToHost, st));
  STC_NA(cudaStreamSynchronize(st));
  if (slots[C_ERROR]) return STC_ERR_INTERNAL;
  out->t0 = slots[C_T0];
  out->t1 = slots[C_T1];
  out->t2 = slots[C_T2];
  out->t3 = slots[C_T3];
  return STC_OK;
}
