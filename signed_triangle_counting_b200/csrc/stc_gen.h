// Seeded, counter-based generators for the synthetic signed graphs.
//
// Every value is a pure function of (seed, stream, index): the same edge list
// comes out of the host code (used by the oracle and the tests) and of the
// device kernels (used by the benchmark), with no floating point on any path
// that decides an edge or a sign.  The reference ships no datasets
// (Signed_TC/Multicore Implementations/Tests/*.csv name *.mtx files that are not
// in the repository), so these generators stand in for them.
//
// Conventions shared by every family:
//  * edges are emitted as (u, v) with u != v (no self-loops: the reference's
//    loader mis-sizes its arrays when it meets one, graph_io.h:147,191-192);
//  * the sign of an undirected edge is a function of the unordered pair
//    {min, max} of its FINAL ids, so duplicate samples always agree in sign
//    (conflicting duplicates leave the reference's survivor unspecified,
//    graph_io.h:244,251-256);
//  * vertex ids are passed through a seeded bijection of [0, n) (random
//    relabelling).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define STC_HD __host__ __device__ __forceinline__
#else
#define STC_HD static inline
#endif

namespace stcgen {

// Stream identifiers: independent random streams per purpose.
enum : uint64_t {
  kStreamPerm = 1,
  kStreamSign = 2,
  kStreamER = 3,
  kStreamRmat = 4,
  kStreamHub = 5,
  kStreamBackbone = 6,
  kStreamDelaunay = 7,
  kStreamDelete = 8,
  kStreamBatch = 9,
};

// SplitMix64 finaliser (Stafford "mix13").
STC_HD uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// i-th output of a SplitMix64 sequence whose state is keyed by (seed, stream).
STC_HD uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
  uint64_t key = mix64(seed ^ mix64(stream * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull));
  return mix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}

STC_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

// Uniform integer in [0, n) from a 64-bit draw (Lemire's multiply-high map).
STC_HD uint64_t uniform(uint64_t r, uint64_t n) { return mulhi64(r, n); }

// Sign of the undirected edge {a, b}: +1 when the draw falls below
// `pos_threshold` (= floor(p * 2^64), computed once on the host), else -1.
STC_HD int8_t edge_sign(uint64_t seed, uint32_t a, uint32_t b, uint64_t pos_threshold) {
  uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
  uint64_t r = draw(seed, kStreamSign, (lo << 32) | hi);
  return r < pos_threshold ? (int8_t)1 : (int8_t)-1;
}

// Seeded bijection of [0, n): a 4-round balanced Feistel network on the
// smallest even-bit power of two >= n, with cycle walking back into [0, n).
struct Perm {
  uint64_t n;
  uint32_t half_bits;
  uint64_t keys[4];
};

STC_HD Perm make_perm(uint64_t seed, uint64_t n) {
  Perm p;
  p.n = n;
  uint32_t bits = 0;
  while (bits < 64 && (1ull << bits) < n) bits++;
  p.half_bits = (bits + 1) / 2;
  if (p.half_bits == 0) p.half_bits = 1;
  for (int r = 0; r < 4; r++) p.keys[r] = draw(seed, kStreamPerm, (uint64_t)r);
  return p;
}

STC_HD uint64_t perm_apply(const Perm& p, uint64_t x) {
  if (p.n <= 1) return x;
  const uint64_t mask = (1ull << p.half_bits) - 1;
  do {
    uint64_t L = x >> p.half_bits, R = x & mask;
    for (int r = 0; r < 4; r++) {
      uint64_t F = mix64(R ^ p.keys[r]) & mask;
      uint64_t nl = R;
      R = L ^ F;
      L = nl;
    }
    x = (L << p.half_bits) | R;
  } while (x >= p.n);
  return x;
}

// ---------------------------------------------------------------- RMAT ----
// Quadrant thresholds as 32-bit fixed point: a, a+b, a+b+c.
struct RmatParams {
  uint32_t scale;        // ids are drawn in [0, 2^scale)
  uint64_t n;            // ids >= n are redrawn (n <= 2^scale)
  uint32_t t_a, t_ab, t_abc;
};

// One RMAT endpoint pair from a stream of draws starting at `ctr`.
STC_HD void rmat_pair(uint64_t seed, uint64_t ctr, const RmatParams& rp,
                      uint64_t* src, uint64_t* dst) {
  uint64_t s = 0, d = 0;
  uint64_t r = 0;
  for (uint32_t l = 0; l < rp.scale; l++) {
    if ((l & 1) == 0) r = draw(seed, kStreamRmat, ctr * 32 + (l >> 1));
    uint32_t x = (l & 1) ? (uint32_t)(r >> 32) : (uint32_t)r;
    uint64_t sb = (x >= rp.t_ab) ? 1 : 0;
    uint64_t db = (x < rp.t_a) ? 0 : (x < rp.t_ab) ? 1 : (x < rp.t_abc) ? 0 : 1;
    s = (s << 1) | sb;
    d = (d << 1) | db;
  }
  *src = s;
  *dst = d;
}

// Sample i of an RMAT graph (before relabelling): redraws (deterministically,
// with an attempt counter) self-loops and ids >= n.
STC_HD void rmat_sample(uint64_t seed, uint64_t i, const RmatParams& rp,
                        uint32_t* u, uint32_t* v) {
  for (uint64_t attempt = 0;; attempt++) {
    uint64_t s, d;
    rmat_pair(seed, i * 64 + attempt, rp, &s, &d);
    if (s != d && s < rp.n && d < rp.n) {
      *u = (uint32_t)s;
      *v = (uint32_t)d;
      return;
    }
  }
}

// ------------------------------------------------------ uniform pairs ----
// Sample i of a uniform random pair in [0, n)^2 without self-loop.
STC_HD void uniform_pair(uint64_t seed, uint64_t stream, uint64_t i, uint64_t n,
                         uint32_t* u, uint32_t* v) {
  for (uint64_t attempt = 0;; attempt++) {
    uint64_t a = uniform(draw(seed, stream, (i * 16 + attempt) * 2), n);
    uint64_t b = uniform(draw(seed, stream, (i * 16 + attempt) * 2 + 1), n);
    if (a != b) {
      *u = (uint32_t)a;
      *v = (uint32_t)b;
      return;
    }
  }
}

// Edge j of hub h in the skew family: (h, uniform target != h).
STC_HD void hub_edge(uint64_t seed, uint32_t h, uint64_t j, uint64_t n,
                     uint32_t* u, uint32_t* v) {
  for (uint64_t attempt = 0;; attempt++) {
    uint64_t t = uniform(draw(seed, kStreamHub + ((uint64_t)h << 8), j * 16 + attempt), n);
    if (t != h) {
      *u = h;
      *v = (uint32_t)t;
      return;
    }
  }
}

}  // namespace stcgen
