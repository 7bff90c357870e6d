// Stable LSD radix sort of 64-bit keys over a bit window [lo, hi), plus the
// range-partitioned scans the graph build and the sharded count use.  The
// kernels have internal linkage: every translation unit that includes this
// header gets its own copy.
//
// Design (B200): every pass is a reduce-then-scan over a fixed grid of
// CTA-contiguous key ranges (4 CTAs per SM), so no kernel ever waits on
// another CTA:
//   upsweep   per-CTA digit histogram of its range      (reads 8 B/key;
//             per-warp shared-memory atomics)
//   scan      one CTA turns [digit][cta] counts into offsets
//   downsweep per 4096-key tile: warp-striped match.any ranking (stable),
//             tile-local reorder through shared memory, coalesced scatter
//             (reads 8 B/key, writes 8 B/key).
// Bits of the key outside [lo, hi) ride along untouched, which is how the
// edge sign travels in bit 63 without a separate payload array.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "stc_device.cuh"

namespace stc {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys
constexpr int kRadix = 256;
constexpr int kMaxSortGrid = kSMs * 4;
constexpr int kUpItems = 8;  // keys per thread per upsweep iteration

struct RangePartition {
  uint32_t grid;     // CTAs
  uint64_t per_cta;  // keys per CTA, a multiple of the tile
};

inline RangePartition range_partition(uint64_t m, uint64_t tile, uint32_t max_grid) {
  uint64_t tiles = (m + tile - 1) / tile;
  if (tiles == 0) tiles = 1;
  uint64_t grid = tiles < max_grid ? tiles : max_grid;
  uint64_t per = (tiles + grid - 1) / grid;
  grid = (tiles + per - 1) / per;
  return RangePartition{(uint32_t)grid, per * tile};
}

static __global__ void __launch_bounds__(kSortThreads) k_radix_upsweep(
    const uint64_t* __restrict__ keys, uint64_t m, uint64_t per_cta, int shift,
    uint32_t dmask, uint32_t* __restrict__ counts, uint32_t grid,
    const unsigned long long* __restrict__ m_dev) {
  __shared__ uint32_t hist[kSortWarps][kRadix + 1];
  const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  if (m_dev && *m_dev < m) m = *m_dev;
  for (unsigned i = tid; i < kSortWarps * (kRadix + 1); i += kSortThreads) (&hist[0][0])[i] = 0;
  __syncthreads();
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < m ? begin + per_cta : m;
  // kUpItems independent loads in flight per thread, then one shared-memory
  // atomic per key into the warp's own histogram.
  for (uint64_t base = begin + warp * 32 * kUpItems; base < end; base += kSortThreads * kUpItems) {
    uint32_t d[kUpItems];
#pragma unroll
    for (int j = 0; j < kUpItems; j++) {
      const uint64_t i = base + j * 32 + lane;
      d[j] = i < end ? (uint32_t)(__ldcs(keys + i) >> shift) & dmask : kRadix;
    }
#pragma unroll
    for (int j = 0; j < kUpItems; j++)
      if (d[j] != kRadix) atomicAdd(&hist[warp][d[j]], 1u);
  }
  __syncthreads();
  for (unsigned d = tid; d < kRadix; d += kSortThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) s += hist[w][d];
    counts[(uint64_t)d * grid + blockIdx.x] = s;
  }
}

// Exclusive scan of `n` 32-bit counts in place by one CTA of 1024 threads.
// Each warp takes a contiguous run of 32-entry rows, read and written a
// row at a time (coalesced): a first pass sums its run, the 32 sums are
// scanned in shared memory, and a second pass scans row by row with the
// warp's carry.
static __global__ void __launch_bounds__(1024) k_scan_counts(uint32_t* __restrict__ a, uint32_t n) {
  __shared__ uint32_t wbase[32];
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t rows = (n + 31) / 32;
  const uint32_t per = (rows + 31) / 32;
  const uint32_t r0 = min(rows, warp * per), r1 = min(rows, r0 + per);
  uint32_t s = 0;
#pragma unroll 4
  for (uint32_t r = r0; r < r1; r++) {
    const uint32_t i = r * 32 + lane;
    s += i < n ? a[i] : 0u;
  }
  s = __reduce_add_sync(kFull, s);
  if (lane == 0) wbase[warp] = s;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = wbase[lane];
    const uint32_t inc = warp_inclusive_scan(t);
    wbase[lane] = inc - t;
  }
  __syncthreads();
  uint32_t carry = wbase[warp];
#pragma unroll 4
  for (uint32_t r = r0; r < r1; r++) {
    const uint32_t i = r * 32 + lane;
    const uint32_t x = i < n ? a[i] : 0u;
    const uint32_t inc = warp_inclusive_scan(x);
    if (i < n) a[i] = carry + inc - x;
    carry += __shfl_sync(kFull, inc, 31);
  }
}

// Ranks one tile's keys (stable): r[j] = the key's rank among the keys of
// its digit in its warp's slice, whist[warp][digit] = the slice's count.
// kFull: every key of the tile is valid, so digits fit 8 bits and the warp
// match takes 8 ballots; a partial tile marks invalid keys with the digit
// kRadix (9 bits).
template <bool kFull>
__device__ __forceinline__ void rank_tile(const uint64_t (&k)[kSortItems], uint64_t wbase,
                                          uint64_t end, int shift, uint32_t dmask,
                                          uint16_t (*whist)[kRadix + 1], unsigned warp,
                                          unsigned lt, uint32_t (&r)[kSortItems]) {
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const bool valid = kFull || wbase + (uint64_t)j * 32 < end;
    const uint32_t dg = valid ? (uint32_t)(k[j] >> shift) & dmask : kRadix;
    const unsigned peers = kFull ? match_label<8>(dg) : match_label<9>(dg);
    const uint32_t base = whist[warp][dg];
    const uint32_t below = __popc(peers & lt);
    __syncwarp();
    if (below == 0 && valid) whist[warp][dg] = (uint16_t)(base + __popc(peers));
    __syncwarp();
    r[j] = base + below;
  }
}

static __global__ void __launch_bounds__(kSortThreads, 3) k_radix_downsweep(
    const uint64_t* __restrict__ in, uint64_t* __restrict__ out, uint64_t m, uint64_t per_cta,
    int shift, uint32_t dmask, const uint32_t* __restrict__ offsets, uint32_t grid,
    const unsigned long long* __restrict__ m_dev) {
  __shared__ uint64_t sbuf[kSortTile];
  __shared__ uint16_t whist[kSortWarps][kRadix + 1];
  __shared__ uint32_t tile_start[kRadix];
  __shared__ uint32_t gofs[kRadix];
  __shared__ uint32_t scan_tmp[kSortWarps + 1];
  const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  if (m_dev && *m_dev < m) m = *m_dev;
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < m ? begin + per_cta : m;
  // gofs[d]: where digit d's next key goes in the output
  for (unsigned d = tid; d < kRadix; d += kSortThreads) gofs[d] = offsets[(uint64_t)d * grid + blockIdx.x];
  const unsigned lt = lanemask_lt();
  for (uint64_t tile = begin; tile < end; tile += kSortTile) {
    for (unsigned i = tid; i < kSortWarps * (kRadix + 1); i += kSortThreads) (&whist[0][0])[i] = 0;
    __syncthreads();
    uint64_t k[kSortItems];
    uint32_t r[kSortItems];
    const uint64_t wbase = tile + (uint64_t)warp * (32 * kSortItems) + lane;
    const bool full = end - tile >= (uint64_t)kSortTile;
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      const uint64_t idx = wbase + (uint64_t)j * 32;
      k[j] = (full || idx < end) ? __ldcs(in + idx) : 0;
    }
    if (full)
      rank_tile<true>(k, wbase, end, shift, dmask, whist, warp, lt, r);
    else
      rank_tile<false>(k, wbase, end, shift, dmask, whist, warp, lt, r);
    __syncthreads();
    // Thread d: the tile's count of digit d, then every warp's slot for it
    // as a tile position (digit start + the warps before).
    const unsigned d = tid;  // kSortThreads == kRadix
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) cnt += whist[w][d];
    uint32_t total;
    const uint32_t st = block_exclusive_scan<kSortThreads>(cnt, scan_tmp, total);
    {
      uint32_t run = st;
#pragma unroll
      for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = whist[w][d];
        whist[w][d] = (uint16_t)run;
        run += c;
      }
    }
    tile_start[d] = gofs[d] - st;  // output index of tile position p is tile_start[digit] + p
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      if (full || wbase + (uint64_t)j * 32 < end) {
        const uint32_t dg = (uint32_t)(k[j] >> shift) & dmask;
        sbuf[whist[warp][dg] + r[j]] = k[j];
      }
    }
    __syncthreads();
    const uint32_t valid = (uint32_t)(end - tile < (uint64_t)kSortTile ? end - tile : kSortTile);
    for (uint32_t i = tid; i < valid; i += kSortThreads) {
      const uint64_t key = sbuf[i];
      const uint32_t dk = (uint32_t)(key >> shift) & dmask;
      out[(uint32_t)(tile_start[dk] + i)] = key;  // indices are below m < 2^32
    }
    __syncthreads();
    gofs[d] += cnt;
    __syncthreads();
  }
}

// Scratch for radix_sort: `counts` holds kRadix * kMaxSortGrid words.
// Sorts keys[0, m) by bits [lo, hi) stably; returns the buffer that holds the
// result (`keys` or `alt`).  m must be below 2^32.  With `m_dev`, the sort
// covers only the first min(m, *m_dev) keys, a count known on the device
// alone (the launches are sized for m, so the sequence can be captured).
inline uint64_t* radix_sort(uint64_t* keys, uint64_t* alt, uint64_t m, int lo, int hi,
                            uint32_t* counts, cudaStream_t st, int* launches = nullptr,
                            const unsigned long long* m_dev = nullptr) {
  if (m <= 1 || hi <= lo) return keys;
  RangePartition p = range_partition(m, kSortTile, kMaxSortGrid);
  uint64_t* src = keys;
  uint64_t* dst = alt;
  for (int shift = lo; shift < hi; shift += 8) {
    const int w = hi - shift < 8 ? hi - shift : 8;
    const uint32_t dmask = (1u << w) - 1;
    k_radix_upsweep<<<p.grid, kSortThreads, 0, st>>>(src, m, p.per_cta, shift, dmask, counts, p.grid,
                                                     m_dev);
    k_scan_counts<<<1, 1024, 0, st>>>(counts, kRadix * p.grid);
    k_radix_downsweep<<<p.grid, kSortThreads, 0, st>>>(src, dst, m, p.per_cta, shift, dmask, counts,
                                                       p.grid, m_dev);
    if (launches) *launches += 3;
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// ------------------------------------------------------- range scans ----
// Exclusive scan of 32-bit values produced by functor F (F(i) for i < n)
// into 64-bit outputs; `emit(i, prefix, value)` receives each element's
// exclusive prefix.  Three launches, no inter-CTA waiting:
//   k_range_reduce -> k_scan_small -> k_range_apply.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class F>
__global__ void __launch_bounds__(kScanThreads) k_range_reduce(F f, uint64_t n, uint64_t per_cta,
                                                               uint64_t* __restrict__ sums) {
  __shared__ uint64_t tmp[kScanThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < n ? begin + per_cta : n;
  uint64_t s = 0;
  for (uint64_t i = begin + threadIdx.x; i < end; i += kScanThreads) s += f(i);
  s = warp_sum(s);
  if (lane_id() == 0) tmp[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < kScanThreads / 32; w++) t += tmp[w];
    sums[blockIdx.x] = t;
  }
}

// Exclusive scan of a[0, n) in place; a[n] receives the total.
static __global__ void __launch_bounds__(1024) k_scan_small(uint64_t* __restrict__ a, uint32_t n) {
  __shared__ uint64_t tmp[33];
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
  uint64_t s = 0;
  for (uint32_t i = b; i < e; i++) s += a[i];
  uint64_t total;
  uint64_t run = block_exclusive_scan<1024>(s, tmp, total);
  for (uint32_t i = b; i < e; i++) {
    uint64_t x = a[i];
    a[i] = run;
    run += x;
  }
  if (threadIdx.x == 0) a[n] = total;
}

// Index into a tile buffer with one padding word per 32: the blocked reads
// (thread t, item j at t * kScanItems + j) then hit 32 distinct banks.
__device__ __forceinline__ uint32_t tile_pad(uint32_t x) { return x + (x >> 5); }

// Every element's exclusive prefix to `emit`, tile by tile: f is evaluated
// and emit called in a striped order (consecutive threads on consecutive
// elements, so that the loads inside f and the stores inside emit
// coalesce), while the scan itself runs over a blocked copy of the tile's
// values in shared memory.
template <class F, class E>
__global__ void __launch_bounds__(kScanThreads) k_range_apply(F f, E emit, uint64_t n,
                                                              uint64_t per_cta,
                                                              const uint64_t* __restrict__ offs) {
  constexpr uint32_t kPadded = kScanTile + kScanTile / 32;
  __shared__ uint64_t tmp[kScanThreads / 32 + 1];
  __shared__ uint32_t sv[kPadded];  // values
  __shared__ uint64_t sp[kPadded];  // tile-relative exclusive prefixes
  const uint64_t begin = (uint64_t)blockIdx.x * per_cta;
  const uint64_t end = begin + per_cta < n ? begin + per_cta : n;
  uint64_t carry = offs[blockIdx.x];
  for (uint64_t tile = begin; tile < end; tile += kScanTile) {
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      const uint32_t x = j * kScanThreads + threadIdx.x;
      sv[tile_pad(x)] = tile + x < end ? f(tile + x) : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      v[j] = sv[tile_pad(threadIdx.x * kScanItems + j)];
      s += v[j];
    }
    uint64_t total;
    uint64_t run = block_exclusive_scan<kScanThreads>(s, tmp, total);
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      sp[tile_pad(threadIdx.x * kScanItems + j)] = run;
      run += v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      const uint32_t x = j * kScanThreads + threadIdx.x;
      if (tile + x < end) emit(tile + x, carry + sp[tile_pad(x)], sv[tile_pad(x)]);
    }
    carry += total;
    __syncthreads();  // the next tile reuses sv and sp
  }
}

// The first two launches of a range scan: per-CTA totals, then their
// exclusive scan in place; the grand total lands in sums[grid], and the
// returned grid is what range_apply needs.  `sums` needs kMaxSortGrid + 1
// words.
template <class F>
inline uint32_t range_reduce_scan(F f, uint64_t n, uint64_t* sums, cudaStream_t st,
                                  int* launches = nullptr) {
  RangePartition p = range_partition(n, kScanTile, kMaxSortGrid);
  k_range_reduce<<<p.grid, kScanThreads, 0, st>>>(f, n, p.per_cta, sums);
  k_scan_small<<<1, 1024, 0, st>>>(sums, p.grid);
  if (launches) *launches += 2;
  return p.grid;
}

// The third launch: every element's exclusive prefix to `emit`, from the
// offsets range_reduce_scan left in `sums` (which the caller may read, e.g.
// the total, in between).
template <class F, class E>
inline void range_apply(F f, E emit, uint64_t n, const uint64_t* sums, cudaStream_t st,
                        int* launches = nullptr) {
  RangePartition p = range_partition(n, kScanTile, kMaxSortGrid);
  k_range_apply<<<p.grid, kScanThreads, 0, st>>>(f, emit, n, p.per_cta, sums);
  if (launches) *launches += 1;
}

// The whole three-launch scan.
template <class F, class E>
inline void range_scan(F f, E emit, uint64_t n, uint64_t* sums, cudaStream_t st,
                       int* launches = nullptr) {
  range_reduce_scan(f, n, sums, st, launches);
  range_apply(f, emit, n, sums, st, launches);
}

}  // namespace stc
