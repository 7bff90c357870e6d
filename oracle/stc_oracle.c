/* ORACLE — test infrastructure, not product code (see stc_oracle.h).
 *
 * Single-threaded C restatement of the reference CPU path.  Each function
 * names the reference lines it follows ("Signed_TC/Multicore Implementations/"
 * is abbreviated MC/).  The one deliberate deviation: a self-loop line is
 * dropped without leaving an uninitialised slot behind (MC/graph_io.h sizes
 * its arrays by line count at :147,:157-161 but skips self-loops at :191-192,
 * so the reference reads garbage there); inputs with self-loops are therefore
 * outside the parity contract.
 */
#define _GNU_SOURCE
#include "stc_oracle.h"

#include <fcntl.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

/* ---------------------------------------------------------------- ingest */

/* MC/graph_io.h:77-83: decimal digits, uint32 wrap-around, no leading blanks. */
static const char* parse_uint(const char* p, const char* end, uint32_t* out) {
  uint32_t x = 0;
  while (p < end && *p >= '0' && *p <= '9') x = x * 10u + (uint32_t)(*p++ - '0');
  *out = x;
  return p;
}

/* MC/graph_io.h:72-76 */
static const char* skip_blanks(const char* p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\t')) p++;
  return p;
}

/* MC/graph_io.h:84-97: '-' gives -1, anything else +1; digits are skipped. */
static const char* parse_sign(const char* p, const char* end, int8_t* out) {
  int8_t s = 1;
  if (p < end && *p == '-') {
    s = -1;
    p++;
  } else if (p < end && *p == '+') {
    p++;
  }
  while (p < end && *p >= '0' && *p <= '9') p++;
  *out = s;
  return p;
}

static int alloc_edges(orc_edge_list* el, uint64_t cap) {
  uint64_t c = cap ? cap : 1;
  el->src = (uint32_t*)malloc(c * sizeof(uint32_t));
  el->dst = (uint32_t*)malloc(c * sizeof(uint32_t));
  el->sign = (int8_t*)malloc(c);
  if (!el->src || !el->dst || !el->sign) {
    orc_free_edge_list(el);
    return 4;
  }
  return 0;
}

/* MC/graph_io.h:117-211, as one sequential pass (the reference's per-thread
 * chunks always end on a line boundary, :124-131, so the result is the same). */
int orc_parse_text(const char* data, uint64_t size, orc_edge_list* out) {
  memset(out, 0, sizeof(*out));
  if (size == 0) return alloc_edges(out, 0); /* :104-105: n = 0, m = 0 */
  const char* end = data + size;
  uint64_t lines = 0;
  for (const char* p = data; p < end;) { /* first pass, :137-150 */
    if (*p == '\n' || *p == '\r') {
      p++;
      continue;
    }
    if (*p == '#' || *p == '%') {
      while (p < end && *p != '\n') p++;
      continue;
    }
    lines++;
    while (p < end && *p != '\n') p++;
  }
  if (alloc_edges(out, lines)) return 4;
  uint64_t w = 0;
  uint32_t max_id = 0;
  for (const char* p = data; p < end;) { /* second pass, :171-202 */
    if (*p == '\n' || *p == '\r') {
      p++;
      continue;
    }
    if (*p == '#' || *p == '%') {
      while (p < end && *p != '\n') p++;
      continue;
    }
    uint32_t u, v;
    int8_t s;
    p = parse_uint(p, end, &u);
    p = skip_blanks(p, end);
    p = parse_uint(p, end, &v);
    p = skip_blanks(p, end);
    p = parse_sign(p, end, &s);
    while (p < end && *p != '\n') p++;
    if (u == v) continue;
    out->src[w] = u < v ? u : v;
    out->dst[w] = u < v ? v : u;
    out->sign[w] = s;
    w++;
    if (u > max_id) max_id = u;
    if (v > max_id) max_id = v;
  }
  out->n = max_id + 1u; /* :210 */
  out->lines = lines;
  out->m = w;
  return 0;
}

int orc_load_graph(const char* path, orc_edge_list* out) {
  memset(out, 0, sizeof(*out));
  int fd = open(path, O_RDONLY);
  if (fd < 0) return 2;
  struct stat st;
  if (fstat(fd, &st) < 0) {
    close(fd);
    return 2;
  }
  uint64_t size = (uint64_t)st.st_size;
  if (size == 0) {
    close(fd);
    return orc_parse_text(NULL, 0, out);
  }
  const char* data = (const char*)mmap(NULL, size, PROT_READ, MAP_PRIVATE, fd, 0);
  if (data == MAP_FAILED) {
    close(fd);
    return 2;
  }
  int rc = orc_parse_text(data, size, out);
  munmap((void*)data, size);
  close(fd);
  return rc;
}

int orc_edge_list_from_arrays(const uint32_t* u, const uint32_t* v, const int8_t* s,
                              uint64_t m, orc_edge_list* out) {
  memset(out, 0, sizeof(*out));
  if (alloc_edges(out, m)) return 4;
  uint64_t w = 0;
  uint32_t max_id = 0;
  for (uint64_t i = 0; i < m; i++) {
    if (u[i] == v[i]) continue;
    out->src[w] = u[i] < v[i] ? u[i] : v[i];
    out->dst[w] = u[i] < v[i] ? v[i] : u[i];
    out->sign[w] = s[i] < 0 ? (int8_t)-1 : (int8_t)1;
    if (out->dst[w] > max_id) max_id = out->dst[w];
    w++;
  }
  out->n = m ? max_id + 1u : 0u;
  out->lines = m;
  out->m = w;
  return 0;
}

void orc_free_edge_list(orc_edge_list* el) {
  free(el->src);
  free(el->dst);
  free(el->sign);
  el->src = el->dst = NULL;
  el->sign = NULL;
  el->n = 0;
  el->m = el->lines = 0;
}

/* ------------------------------------------------------------ CSR build */

/* Stable LSD radix sort of (key, payload) pairs, 16-bit digits. */
static int radix_sort_pairs(uint64_t* key, int8_t* val, uint64_t m, int key_bits) {
  uint64_t* k2 = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  int8_t* v2 = (int8_t*)malloc(m ? m : 1);
  uint64_t* cnt = (uint64_t*)malloc(65536 * sizeof(uint64_t));
  if (!k2 || !v2 || !cnt) {
    free(k2);
    free(v2);
    free(cnt);
    return 4;
  }
  for (int shift = 0; shift < key_bits; shift += 16) {
    memset(cnt, 0, 65536 * sizeof(uint64_t));
    for (uint64_t i = 0; i < m; i++) cnt[(key[i] >> shift) & 0xFFFF]++;
    uint64_t sum = 0;
    for (int d = 0; d < 65536; d++) {
      uint64_t c = cnt[d];
      cnt[d] = sum;
      sum += c;
    }
    for (uint64_t i = 0; i < m; i++) {
      uint64_t pos = cnt[(key[i] >> shift) & 0xFFFF]++;
      k2[pos] = key[i];
      v2[pos] = val[i];
    }
    memcpy(key, k2, m * sizeof(uint64_t));
    memcpy(val, v2, m);
  }
  free(k2);
  free(v2);
  free(cnt);
  return 0;
}

static int cmp_u32_sign(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return (x >> 8) < (y >> 8) ? -1 : (x >> 8) > (y >> 8);
}

int orc_build_forward_csr(const orc_edge_list* el, orc_forward_csr* out) {
  memset(out, 0, sizeof(*out));
  const uint32_t n = el->n;
  const uint64_t m = el->m;

  /* Dedup: sort by (u, v) and keep the first of equal keys
   * (MC/graph_io.h:221-259; stable here, so "first" is input order). */
  uint64_t* key = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  int8_t* sg = (int8_t*)malloc(m ? m : 1);
  if (!key || !sg) {
    free(key);
    free(sg);
    return 4;
  }
  for (uint64_t i = 0; i < m; i++) {
    key[i] = ((uint64_t)el->src[i] << 32) | el->dst[i];
    sg[i] = el->sign[i];
  }
  if (radix_sort_pairs(key, sg, m, 64)) {
    free(key);
    free(sg);
    return 4;
  }
  uint64_t um = 0;
  for (uint64_t i = 0; i < m; i++) {
    if (um > 0 && key[um - 1] == key[i]) continue;
    key[um] = key[i];
    sg[um] = sg[i];
    um++;
  }

  /* Degree (MC/graph_io.h:261-268). */
  uint32_t* degree = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
  /* Rank: counting sort by degree, ties by ascending id (:270-317). */
  uint32_t* rank = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  uint32_t* fdeg = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
  uint64_t* offsets = (uint64_t*)malloc(((uint64_t)n + 1) * sizeof(uint64_t));
  if (!degree || !rank || !fdeg || !offsets) goto oom;
  for (uint64_t i = 0; i < um; i++) {
    degree[key[i] >> 32]++;
    degree[(uint32_t)key[i]]++;
  }
  {
    uint32_t max_deg = 0;
    for (uint32_t i = 0; i < n; i++)
      if (degree[i] > max_deg) max_deg = degree[i];
    uint64_t bsz = (uint64_t)max_deg + 2;
    uint64_t* bucket = (uint64_t*)calloc(bsz, sizeof(uint64_t));
    if (!bucket) goto oom;
    for (uint32_t i = 0; i < n; i++) bucket[degree[i] + 1]++;
    for (uint64_t d = 1; d < bsz; d++) bucket[d] += bucket[d - 1];
    for (uint32_t i = 0; i < n; i++) rank[i] = (uint32_t)bucket[degree[i]]++;
    free(bucket);
  }
  /* Orientation u -> v iff rank[u] < rank[v] (:319-330); offsets (:332-367). */
  for (uint64_t i = 0; i < um; i++) {
    uint32_t u = (uint32_t)(key[i] >> 32), v = (uint32_t)key[i];
    fdeg[rank[u] < rank[v] ? u : v]++;
  }
  offsets[0] = 0;
  for (uint32_t v = 0; v < n; v++) offsets[v + 1] = offsets[v] + fdeg[v];
  {
    uint64_t total = n ? offsets[n] : 0;
    uint32_t* edges = (uint32_t*)malloc((total ? total : 1) * sizeof(uint32_t));
    int8_t* signs = (int8_t*)malloc(total ? total : 1);
    uint64_t* cur = (uint64_t*)malloc(((uint64_t)n + 1) * sizeof(uint64_t));
    if (!edges || !signs || !cur) {
      free(edges);
      free(signs);
      free(cur);
      goto oom;
    }
    memcpy(cur, offsets, (uint64_t)n * sizeof(uint64_t));
    for (uint64_t i = 0; i < um; i++) { /* scatter (:373-394) */
      uint32_t u = (uint32_t)(key[i] >> 32), v = (uint32_t)key[i];
      uint32_t from = rank[u] < rank[v] ? u : v, to = rank[u] < rank[v] ? v : u;
      uint64_t pos = cur[from]++;
      edges[pos] = to;
      signs[pos] = sg[i];
    }
    free(cur);
    /* sort_adj_lists (MC/tc_serial.cpp:33-93): ascending neighbour id. */
    uint64_t* tmp = NULL;
    uint32_t max_f = 0;
    for (uint32_t v = 0; v < n; v++)
      if (fdeg[v] > max_f) max_f = fdeg[v];
    tmp = (uint64_t*)malloc(((uint64_t)max_f + 1) * sizeof(uint64_t));
    if (!tmp) {
      free(edges);
      free(signs);
      goto oom;
    }
    for (uint32_t v = 0; v < n; v++) {
      uint32_t d = fdeg[v];
      if (d < 2) continue;
      uint64_t b = offsets[v];
      for (uint32_t i = 0; i < d; i++)
        tmp[i] = ((uint64_t)edges[b + i] << 8) | (uint8_t)signs[b + i];
      qsort(tmp, d, sizeof(uint64_t), cmp_u32_sign);
      for (uint32_t i = 0; i < d; i++) {
        edges[b + i] = (uint32_t)(tmp[i] >> 8);
        signs[b + i] = (int8_t)(uint8_t)(tmp[i] & 0xFF);
      }
    }
    free(tmp);
    out->n = n;
    out->m = total;
    out->offsets = offsets;
    out->edges = edges;
    out->signs = signs;
    out->fdeg = fdeg;
    out->rank = rank;
  }
  free(degree);
  free(key);
  free(sg);
  return 0;
oom:
  free(degree);
  free(rank);
  free(fdeg);
  free(offsets);
  free(key);
  free(sg);
  return 4;
}

void orc_free_forward_csr(orc_forward_csr* c) {
  free(c->offsets);
  free(c->edges);
  free(c->signs);
  free(c->fdeg);
  free(c->rank);
  memset(c, 0, sizeof(*c));
}

/* ------------------------------------------------------------- counting */

/* classify (MC/tc_serial.cpp:95-112): neg count 0..3 -> T3, T2, T1, T0. */
static inline void classify(int8_t a, int8_t b, int8_t c, uint64_t t[4]) {
  int neg = ((1 - a) >> 1) + ((1 - b) >> 1) + ((1 - c) >> 1);
  t[3 - neg]++;
}

/* merge_intersect (MC/tc_serial.cpp:114-136). */
static void merge_intersect(const orc_forward_csr* c, uint32_t u, uint32_t v, int8_t s_uv,
                            uint64_t t[4]) {
  uint64_t i = c->offsets[u], ie = c->offsets[u + 1];
  uint64_t j = c->offsets[v], je = c->offsets[v + 1];
  uint32_t ru = c->rank[u], rv = c->rank[v];
  while (i < ie && j < je) {
    uint32_t a = c->edges[i], b = c->edges[j];
    if (a == b) {
      if (c->rank[a] > ru && c->rank[a] > rv) classify(s_uv, c->signs[i], c->signs[j], t);
      i++;
      j++;
    } else if (a < b) {
      i++;
    } else {
      j++;
    }
  }
}

void orc_vertex_counts(const orc_forward_csr* c, uint64_t* cnt) {
  for (uint32_t u = 0; u < c->n; u++) { /* MC/tc_serial.cpp:143-158 */
    uint64_t t[4] = {0, 0, 0, 0};
    for (uint64_t e = c->offsets[u]; e < c->offsets[u + 1]; e++)
      merge_intersect(c, u, c->edges[e], c->signs[e], t);
    for (int k = 0; k < 4; k++) cnt[4 * (uint64_t)u + k] = t[k];
  }
}

void orc_count_triangles(const orc_forward_csr* c, uint64_t t[4]) {
  t[0] = t[1] = t[2] = t[3] = 0;
  for (uint32_t u = 0; u < c->n; u++)
    for (uint64_t e = c->offsets[u]; e < c->offsets[u + 1]; e++)
      merge_intersect(c, u, c->edges[e], c->signs[e], t);
}

/* intersect_signed_ranked + its driver loop (MC/tc_merge_sign_enu.cpp:12-44,
 * :132-144): balanced iff the sign product is positive. */
void orc_count_merge(const orc_forward_csr* c, uint64_t* balanced, uint64_t* unbalanced) {
  uint64_t bal = 0, unb = 0;
  for (uint32_t v = 0; v < c->n; v++) {
    uint64_t a0 = c->offsets[v], a1 = c->offsets[v + 1];
    for (uint64_t e = a0; e < a1; e++) {
      uint32_t w = c->edges[e];
      uint64_t i = a0, j = c->offsets[w], je = c->offsets[w + 1];
      uint32_t rv = c->rank[v], rw = c->rank[w];
      while (i < a1 && j < je) {
        uint32_t x = c->edges[i], y = c->edges[j];
        if (x == y) {
          if (c->rank[x] > rv && c->rank[x] > rw) {
            int prod = c->signs[e] * c->signs[i] * c->signs[j];
            if (prod > 0)
              bal++;
            else
              unb++;
          }
          i++;
          j++;
        } else if (x < y) {
          i++;
        } else {
          j++;
        }
      }
    }
  }
  *balanced = bal;
  *unbalanced = unb;
}

/* AdjHashTable::hash32 / next_pow2 (MC/tc_hash_sign_enu.cpp:58-73). */
static inline uint32_t hash32(uint32_t x) {
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  return (x >> 16) ^ x;
}
static inline uint32_t next_pow2(uint32_t x) {
  if (x == 0) return 1;
  x--;
  x |= x >> 1;
  x |= x >> 2;
  x |= x >> 4;
  x |= x >> 8;
  x |= x >> 16;
  return x + 1;
}

/* Per-vertex linear-probe tables in one arena (MC/tc_hash_sign_enu.cpp:100-117)
 * probed from the smaller list (:125-165). */
int orc_count_hash(const orc_forward_csr* c, uint64_t* balanced, uint64_t* unbalanced) {
  const uint32_t n = c->n;
  uint64_t* ho = (uint64_t*)malloc(((uint64_t)n + 1) * sizeof(uint64_t));
  if (!ho) return 4;
  ho[0] = 0;
  for (uint32_t v = 0; v < n; v++) ho[v + 1] = ho[v] + next_pow2(c->fdeg[v] * 2 + 1);
  uint32_t* hk = (uint32_t*)malloc((ho[n] ? ho[n] : 1) * sizeof(uint32_t));
  int8_t* hs = (int8_t*)malloc(ho[n] ? ho[n] : 1);
  if (!hk || !hs) {
    free(ho);
    free(hk);
    free(hs);
    return 4;
  }
  for (uint32_t v = 0; v < n; v++) {
    uint32_t mask = (uint32_t)(ho[v + 1] - ho[v]) - 1;
    uint32_t* K = hk + ho[v];
    int8_t* S = hs + ho[v];
    for (uint32_t i = 0; i <= mask; i++) K[i] = UINT32_MAX;
    for (uint64_t e = c->offsets[v]; e < c->offsets[v + 1]; e++) {
      uint32_t pos = hash32(c->edges[e]) & mask;
      while (K[pos] != UINT32_MAX) pos = (pos + 1) & mask;
      K[pos] = c->edges[e];
      S[pos] = c->signs[e];
    }
  }
  uint64_t bal = 0, unb = 0;
  for (uint32_t v = 0; v < n; v++) {
    for (uint64_t wi = c->offsets[v]; wi < c->offsets[v + 1]; wi++) {
      uint32_t w = c->edges[wi];
      if (c->rank[v] >= c->rank[w]) continue;
      int8_t s_vw = c->signs[wi];
      int v_small = c->fdeg[v] <= c->fdeg[w];
      uint32_t it = v_small ? v : w, pr = v_small ? w : v;
      uint32_t mask = (uint32_t)(ho[pr + 1] - ho[pr]) - 1;
      const uint32_t* K = hk + ho[pr];
      const int8_t* S = hs + ho[pr];
      for (uint64_t i = c->offsets[it]; i < c->offsets[it + 1]; i++) {
        uint32_t u = c->edges[i];
        if (c->rank[u] <= c->rank[v] || c->rank[u] <= c->rank[w]) continue;
        uint32_t pos = hash32(u) & mask;
        while (K[pos] != UINT32_MAX && K[pos] != u) pos = (pos + 1) & mask;
        if (K[pos] != u) continue;
        int prod = s_vw * c->signs[i] * S[pos];
        if (prod > 0)
          bal++;
        else
          unb++;
      }
    }
  }
  free(ho);
  free(hk);
  free(hs);
  *balanced = bal;
  *unbalanced = unb;
  return 0;
}

int orc_count_arrays(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m,
                     uint64_t t[4]) {
  orc_edge_list el;
  orc_forward_csr csr;
  int rc = orc_edge_list_from_arrays(u, v, s, m, &el);
  if (rc) return rc;
  rc = orc_build_forward_csr(&el, &csr);
  orc_free_edge_list(&el);
  if (rc) return rc;
  orc_count_triangles(&csr, t);
  orc_free_forward_csr(&csr);
  return 0;
}
