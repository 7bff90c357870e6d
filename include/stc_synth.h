/* Seeded synthetic signed graphs for the five benchmark workloads.
 *
 * These have no counterpart in the reference, which ships no datasets
 * (Signed_TC/Multicore Implementations/Tests/*.csv name *.mtx inputs that are
 * not in the repository).  Every generator is a pure function of its seed:
 * the host functions below and the device generator in stc.h produce the
 * same edge lists bit for bit.  Edges never contain self-loops, duplicate
 * samples of one undirected edge always carry the same sign, and vertex ids
 * are randomly relabelled by a seeded bijection of [0, n).
 */
#ifndef STC_SYNTH_H
#define STC_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Host edge list owned by the library; release with stc_synth_free. */
typedef struct stc_synth_graph {
  uint64_t n;      /* vertex-id space [0, n) */
  uint64_t m;      /* number of emitted edges (may include same-sign duplicates) */
  uint32_t* src;
  uint32_t* dst;
  int8_t* sign;
} stc_synth_graph;

enum stc_synth_kind {
  STC_SYNTH_ER = 0,       /* G(n, m): m distinct uniform pairs */
  STC_SYNTH_RMAT = 1,     /* RMAT samples, symmetrised by the consumer's dedup */
  STC_SYNTH_DELAUNAY = 2, /* Delaunay triangulation of n uniform points, edges deleted */
  STC_SYNTH_SKEW = 3      /* uniform backbone + hubs of log-uniform degree */
};

/* Per-graph recipe of the batched workload (one entry per graph). */
typedef struct stc_batch_spec {
  uint64_t seed;           /* per-graph seed */
  uint64_t n;              /* log-uniform in [1e3, 1e6] */
  uint32_t kind;           /* STC_SYNTH_ER, STC_SYNTH_RMAT or STC_SYNTH_DELAUNAY */
  uint32_t rmat_scale;     /* ceil(log2 n) for RMAT, else 0 */
  uint64_t m_target;       /* ER: 4n edges; RMAT: 8n samples; Delaunay: 0 */
  double p_pos;            /* uniform in [0.3, 0.9] */
} stc_batch_spec;

/* Status codes are those of stc.h: 0 = success, 1 = invalid argument,
 * 4 = out of host memory. */
int stc_synth_er(uint64_t seed, uint64_t n, uint64_t m, double p_pos,
                 stc_synth_graph* out);
int stc_synth_rmat(uint64_t seed, uint32_t scale, uint64_t n, uint64_t samples,
                   double a, double b, double c, double p_pos,
                   stc_synth_graph* out);
int stc_synth_delaunay(uint64_t seed, uint64_t n, double delete_frac,
                       double p_pos, stc_synth_graph* out);
int stc_synth_skew(uint64_t seed, uint64_t n, uint64_t m_total, uint32_t hubs,
                   uint64_t hub_deg_min, uint64_t hub_deg_max, double p_pos,
                   stc_synth_graph* out);

/* Recipes of the G graphs of the batched workload. */
int stc_synth_batch_specs(uint64_t seed, uint32_t G, stc_batch_spec* specs);
/* Builds graph `spec` of a batch. */
int stc_synth_batch_graph(const stc_batch_spec* spec, stc_synth_graph* out);

/* Graphs [g_begin, g_end) of a batch, generated in parallel and packed back
 * to back into `out` (ids local to each graph); offsets[i] (g_end - g_begin
 * + 1 entries, caller-owned) receives the start of graph g_begin + i. */
int stc_synth_batch_packed(const stc_batch_spec* specs, uint32_t g_begin, uint32_t g_end,
                           stc_synth_graph* out, uint64_t* offsets);

/* The five named workloads: 1 = ER(1e4, 1e5, p=.7); 2 = Delaunay(1e6 points,
 * 20% deleted, p=.6); 3 = RMAT(scale 24, ef 16, .57/.19/.19/.05, p=.5);
 * 5 = skew(64Mi vertices, 128Mi samples, 32 hubs in [1e5, 1e7], p=.8).
 * `shrink` (0 = full size) divides the sizes by 2^shrink for quick tests.
 * Workload 4 is a batch: use stc_synth_batch_specs. */
int stc_synth_workload(int workload, uint32_t shrink, stc_synth_graph* out);
uint64_t stc_synth_workload_seed(int workload);

/* Host threads used by the generators (0 = all hardware threads). */
void stc_synth_set_threads(uint32_t threads);

void stc_synth_free(stc_synth_graph* g);

#ifdef __cplusplus
}
#endif

#endif /* STC_SYNTH_H */
