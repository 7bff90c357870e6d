/* ORACLE — test infrastructure, not product code.
 *
 * A plain-C, single-threaded restatement of the reference's CPU path for
 * signed triangle counting (NikhilBisht2/Signed_Triangle_Counting,
 * "Signed_TC/Multicore Implementations/"), used only by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and only as the
 * checker.  Nothing in the product links or calls it.
 *
 * Parity is pinned against the reference itself: oracle/Makefile compiles the
 * reference's own programs from their sources into oracle/_ref/, and
 * tests/golden/make_golden.py records their outputs as fixtures that the
 * oracle must reproduce (tests/test_oracle.py).
 */
#ifndef STC_ORACLE_H
#define STC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EdgeList (graph_io.h:14-20) plus the raw line count the reference
 * reports as `raw_edges`. */
typedef struct orc_edge_list {
  uint32_t n;      /* max kept id + 1 (graph_io.h:210) */
  uint64_t lines;  /* non-comment, non-blank lines (graph_io.h:135-151) */
  uint64_t m;      /* kept edges (self-loops dropped, graph_io.h:191-192) */
  uint32_t* src;   /* min endpoint (graph_io.h:193) */
  uint32_t* dst;   /* max endpoint (graph_io.h:194) */
  int8_t* sign;
} orc_edge_list;

/* ForwardCSR (graph_io.h:22-30) with lists sorted by neighbour id as
 * sort_adj_lists leaves them (tc_serial.cpp:33-93). */
typedef struct orc_forward_csr {
  uint32_t n;
  uint64_t m;
  uint64_t* offsets; /* n + 1 */
  uint32_t* edges;
  int8_t* signs;
  uint32_t* fdeg;
  uint32_t* rank;
} orc_forward_csr;

/* load_graph (graph_io.h:100-212) over an in-memory buffer / a file. */
int orc_parse_text(const char* data, uint64_t size, orc_edge_list* out);
int orc_load_graph(const char* path, orc_edge_list* out);
/* The normalisation load_graph applies per parsed line, over arrays. */
int orc_edge_list_from_arrays(const uint32_t* u, const uint32_t* v, const int8_t* s,
                              uint64_t m, orc_edge_list* out);
void orc_free_edge_list(orc_edge_list* el);

/* build_forward_csr (graph_io.h:231-402) + sort_adj_lists (tc_serial.cpp:33-93).
 * Duplicates keep their first occurrence in input order. */
int orc_build_forward_csr(const orc_edge_list* el, orc_forward_csr* out);
void orc_free_forward_csr(orc_forward_csr* csr);

/* count_triangles (tc_serial.cpp:138-170): t[0..3] = T0 (---), T1 (+--),
 * T2 (++-), T3 (+++). */
void orc_count_triangles(const orc_forward_csr* csr, uint64_t t[4]);
/* Per-source counts cnt[4u + k] as tc_serial.cpp:141-158 keeps them. */
void orc_vertex_counts(const orc_forward_csr* csr, uint64_t* cnt);
/* tc_merge_sign_enu.cpp:12-44,128-144: balanced / unbalanced. */
void orc_count_merge(const orc_forward_csr* csr, uint64_t* balanced, uint64_t* unbalanced);
/* tc_hash_sign_enu.cpp:11-74,100-165: balanced / unbalanced. */
int orc_count_hash(const orc_forward_csr* csr, uint64_t* balanced, uint64_t* unbalanced);

/* Whole path on arrays: normalise, build, count. */
int orc_count_arrays(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m,
                     uint64_t t[4]);

/* synth_rmat.c: the package's seeded RMAT workload generator restated
 * (same arguments and output as stc_synth_rmat in include/stc_synth.h), so
 * that the reference's code can be fed the benchmark input without the
 * package's library; OpenMP over the samples. */
int orc_synth_rmat(uint64_t seed, uint32_t scale, uint64_t n, uint64_t samples, double a,
                   double b, double c, double p_pos, uint32_t* src, uint32_t* dst, int8_t* sign);
/* Writes `u v sign` lines (sign 1 or -1): the reference programs' input. */
int orc_write_edge_text(const char* path, const uint32_t* u, const uint32_t* v, const int8_t* s,
                        uint64_t m);

#ifdef __cplusplus
}
#endif

#endif
