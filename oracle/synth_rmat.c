/* ORACLE — test infrastructure, not product code.
 *
 * An independent C restatement of the package's seeded RMAT generator (the
 * counter-based recipe of include/stc_synth.h: SplitMix64 draws keyed by
 * (seed, stream, index), two quadrant bits per 64-bit draw, redraw of
 * self-loops and of ids >= n, relabelling by a 4-round Feistel bijection
 * with cycle walking, and a sign drawn from the final unordered pair).  The
 * reference ships no datasets, so the benchmark's CPU baseline feeds the
 * reference's own code with this generator's output: it produces the same
 * edge list as the package's generator bit for bit (tests/test_oracle.py
 * checks that), without loading the package's library.
 *
 * Also here: a plain-text writer of `u v sign` lines, the input format of
 * the reference programs (MC/graph_io.h:100-212, "Signed_TC/Multicore
 * Implementations/").
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "stc_oracle.h"

enum { kStreamPerm = 1, kStreamSign = 2, kStreamRmat = 4 };

static inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* The i-th value of a SplitMix64 sequence keyed by (seed, stream). */
static inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
  const uint64_t key = mix64(seed ^ mix64(stream * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull));
  return mix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}

typedef struct {
  uint64_t n;
  uint32_t half_bits;
  uint64_t keys[4];
} perm_t;

static perm_t make_perm(uint64_t seed, uint64_t n) {
  perm_t p;
  uint32_t bits = 0;
  p.n = n;
  while (bits < 64 && (1ull << bits) < n) bits++;
  p.half_bits = (bits + 1) / 2;
  if (p.half_bits == 0) p.half_bits = 1;
  for (int r = 0; r < 4; r++) p.keys[r] = draw(seed, kStreamPerm, (uint64_t)r);
  return p;
}

/* Balanced Feistel network on 2 * half_bits bits, walked back into [0, n). */
static inline uint64_t perm_apply(const perm_t* p, uint64_t x) {
  if (p->n <= 1) return x;
  const uint64_t mask = (1ull << p->half_bits) - 1;
  do {
    uint64_t L = x >> p->half_bits, R = x & mask;
    for (int r = 0; r < 4; r++) {
      const uint64_t F = mix64(R ^ p->keys[r]) & mask;
      const uint64_t nl = R;
      R = L ^ F;
      L = nl;
    }
    x = (L << p->half_bits) | R;
  } while (x >= p->n);
  return x;
}

static uint32_t threshold32(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return UINT32_MAX;
  return (uint32_t)ldexp(p, 32);
}

static uint64_t threshold64(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return UINT64_MAX;
  return (uint64_t)ldexp(p, 64);
}

int orc_synth_rmat(uint64_t seed, uint32_t scale, uint64_t n, uint64_t samples, double a,
                   double b, double c, double p_pos, uint32_t* src, uint32_t* dst, int8_t* sign) {
  if (scale == 0 || scale > 31 || n < 2 || n > (1ull << scale) || !src || !dst || !sign) return 1;
  const uint32_t t_a = threshold32(a), t_ab = threshold32(a + b), t_abc = threshold32(a + b + c);
  const uint64_t thr = threshold64(p_pos);
  const perm_t perm = make_perm(seed, n);
#pragma omp parallel for schedule(static, 65536)
  for (uint64_t i = 0; i < samples; i++) {
    uint64_t s = 0, d = 0;
    for (uint64_t attempt = 0;; attempt++) {
      /* One endpoint pair: level l takes 32 bits of draw ctr * 32 + l / 2. */
      const uint64_t ctr = i * 64 + attempt;
      uint64_t r = 0;
      s = d = 0;
      for (uint32_t l = 0; l < scale; l++) {
        if ((l & 1) == 0) r = draw(seed, kStreamRmat, ctr * 32 + (l >> 1));
        const uint32_t x = (l & 1) ? (uint32_t)(r >> 32) : (uint32_t)r;
        const uint64_t sb = x >= t_ab;
        const uint64_t db = x < t_a ? 0 : x < t_ab ? 1 : x < t_abc ? 0 : 1;
        s = (s << 1) | sb;
        d = (d << 1) | db;
      }
      if (s != d && s < n && d < n) break;
    }
    const uint32_t u = (uint32_t)perm_apply(&perm, s), v = (uint32_t)perm_apply(&perm, d);
    const uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
    src[i] = u;
    dst[i] = v;
    sign[i] = draw(seed, kStreamSign, (lo << 32) | hi) < thr ? (int8_t)1 : (int8_t)-1;
  }
  return 0;
}

/* `u v sign` lines with sign 1 / -1, as the reference's loader reads them. */
int orc_write_edge_text(const char* path, const uint32_t* u, const uint32_t* v, const int8_t* s,
                        uint64_t m) {
  FILE* f = fopen(path, "wb");
  if (!f) return 2;
  enum { kBuf = 1 << 20 };
  char* buf = (char*)malloc(kBuf + 64);
  if (!buf) {
    fclose(f);
    return 4;
  }
  size_t at = 0;
  for (uint64_t i = 0; i < m; i++) {
    char tmp[12];
    for (int k = 0; k < 2; k++) {
      uint32_t x = k ? v[i] : u[i];
      int len = 0;
      do {
        tmp[len++] = (char)('0' + x % 10);
        x /= 10;
      } while (x);
      while (len) buf[at++] = tmp[--len];
      buf[at++] = ' ';
    }
    if (s[i] < 0) buf[at++] = '-';
    buf[at++] = '1';
    buf[at++] = '\n';
    if (at >= kBuf) {
      if (fwrite(buf, 1, at, f) != at) {
        free(buf);
        fclose(f);
        return 2;
      }
      at = 0;
    }
  }
  int rc = 0;
  if (at && fwrite(buf, 1, at, f) != at) rc = 2;
  free(buf);
  if (fclose(f) != 0) rc = 2;
  return rc;
}
