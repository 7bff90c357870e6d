// Device-side helpers shared by the graph-build and counting kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace stc {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Inclusive warp scan.
template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T x = __shfl_up_sync(kFull, v, o);
    if (lane >= (unsigned)o) v += x;
  }
  return v;
}

// Exclusive scan over a block of BLOCK threads; returns the block total in
// `total`.  `smem` must hold BLOCK/32 entries.
template <int BLOCK, class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T& total) {
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < BLOCK / 32 ? smem[lane] : T(0);
    T wi = warp_inclusive_scan(w);
    if (lane < BLOCK / 32) smem[lane] = wi - w;
    if (lane == BLOCK / 32 - 1) smem[BLOCK / 32] = wi;
  }
  __syncthreads();
  T r = smem[warp] + inc - v;
  total = smem[BLOCK / 32];
  __syncthreads();
  return r;
}

// Lanes of the warp holding the same BITS-bit label as this lane, computed
// with one ballot per label bit (a cheaper warp multi-split than
// __match_any_sync).  All 32 lanes must call it; labels must fit BITS bits.
template <int BITS>
__device__ __forceinline__ unsigned match_label(uint32_t label) {
  unsigned peers = kFull;
#pragma unroll
  for (int b = 0; b < BITS; b++) {
    const unsigned set = __ballot_sync(kFull, (label >> b) & 1u);
    peers &= ((label >> b) & 1u) ? set : ~set;
  }
  return peers;
}

__host__ __device__ __forceinline__ uint32_t bit_width64(uint64_t x) {
  uint32_t b = 0;
  while (b < 64 && (x >> b) != 0) b++;
  return b;
}

}  // namespace stc
