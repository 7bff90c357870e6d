// ORACLE — test infrastructure, not product code.
//
// In-memory harness around the reference's own CPU code.  It is compiled
// from the reference sources where they lie (oracle/Makefile passes their
// directory with -I); nothing of the reference is copied here.  It exists
// because the batched workload's text form would be tens of GB: the harness
// hands arrays straight to the reference's build_forward_csr,
// sort_adj_lists and count_triangles ("Signed_TC/Multicore
// Implementations/tc_serial.cpp" and "graph_io.h").
#include <cstdint>
#include <cstring>

#define main stc_reference_tc_serial_main
#include "tc_serial.cpp"
#undef main

namespace {

// The EdgeList that load_graph (graph_io.h:164-210) produces for these
// lines: src = min, dst = max, self-loops skipped, n = max id + 1.  Unlike
// load_graph, no uninitialised slots are left for skipped self-loops.
EdgeList make_edge_list(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m) {
  EdgeList el{};
  el.src = new uint32_t[m ? m : 1];
  el.dst = new uint32_t[m ? m : 1];
  el.sign = new int8_t[m ? m : 1];
  uint64_t w = 0;
  uint32_t max_id = 0;
  for (uint64_t i = 0; i < m; i++) {
    if (u[i] == v[i]) continue;
    el.src[w] = std::min(u[i], v[i]);
    el.dst[w] = std::max(u[i], v[i]);
    el.sign[w] = s[i] < 0 ? (int8_t)-1 : (int8_t)1;
    max_id = std::max(max_id, el.dst[w]);
    w++;
  }
  el.n = m ? max_id + 1 : 0;
  el.m = (uint32_t)w;
  return el;
}

}  // namespace

extern "C" {

// Per-type counts t[0..3] = T0, T1, T2, T3 from the reference code, the
// seconds spent in build_forward_csr, sort_adj_lists and count_triangles, and
// the number of forward edges (= undirected edges after dedup).
int stc_ref_count_arrays(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m,
                         uint64_t t[4], double seconds[3], uint64_t* forward_edges) {
  if (m >= (1ull << 32)) return 1;  // EdgeList::m is uint32 (graph_io.h:16)
  EdgeList el = make_edge_list(u, v, s, m);
  Timer tb;
  ForwardCSR csr = build_forward_csr(el);
  double t_build = tb.elapsed_sec();
  free_edge_list(el);
  Timer ts;
  sort_adj_lists(csr);
  double t_sort = ts.elapsed_sec();
  Timer tc;
  GlobalTriCounts g = count_triangles(csr);
  double t_count = tc.elapsed_sec();
  if (forward_edges) *forward_edges = csr.m;
  free_forward_csr(csr);
  t[0] = g.t0;
  t[1] = g.t1;
  t[2] = g.t2;
  t[3] = g.t3;
  if (seconds) {
    seconds[0] = t_build;
    seconds[1] = t_sort;
    seconds[2] = t_count;
  }
  return 0;
}

// The reference's sorted forward CSR for these edges, copied into caller
// buffers sized n + 1 (offsets), n (fdeg, rank) and m (edges, signs).  Call
// once with null buffers to learn n and m.
int stc_ref_forward_csr(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m,
                        uint32_t* n_out, uint64_t* m_out, uint64_t* offsets, uint32_t* edges,
                        int8_t* signs, uint32_t* fdeg, uint32_t* rank) {
  if (m >= (1ull << 32)) return 1;
  EdgeList el = make_edge_list(u, v, s, m);
  ForwardCSR csr = build_forward_csr(el);
  free_edge_list(el);
  sort_adj_lists(csr);
  *n_out = csr.n;
  *m_out = csr.m;
  if (offsets) {
    std::memcpy(offsets, csr.offsets, ((uint64_t)csr.n + 1) * sizeof(uint64_t));
    std::memcpy(edges, csr.edges, csr.m * sizeof(uint32_t));
    std::memcpy(signs, csr.signs, csr.m);
    std::memcpy(fdeg, csr.fdeg, (uint64_t)csr.n * sizeof(uint32_t));
    std::memcpy(rank, csr.rank_, (uint64_t)csr.n * sizeof(uint32_t));
  }
  free_forward_csr(csr);
  return 0;
}

// ---------------------------------------------------------------------
// A reference CSR kept between calls, so that the benchmark's CPU baseline
// can time count_triangles on a bounded sample of a large graph: the
// sample is the sources whose id is below a bound.  The generators relabel
// ids by a seeded bijection, so such a prefix is a uniform random sample of
// the vertices.

namespace {
ForwardCSR g_kept{};
bool g_have_kept = false;
}  // namespace

// OpenMP threads the reference's parallel loops use.
int stc_ref_threads(void) { return omp_get_max_threads(); }

void stc_ref_release(void) {
  if (g_have_kept) free_forward_csr(g_kept);
  g_kept = ForwardCSR{};
  g_have_kept = false;
}

// build_forward_csr + sort_adj_lists of these edges, kept for
// stc_ref_count_prefix; seconds[0] and seconds[1] receive their times.
int stc_ref_prepare(const uint32_t* u, const uint32_t* v, const int8_t* s, uint64_t m,
                    double seconds[2], uint32_t* n_out, uint64_t* forward_edges) {
  if (m >= (1ull << 32)) return 1;
  stc_ref_release();
  EdgeList el = make_edge_list(u, v, s, m);
  Timer tb;
  g_kept = build_forward_csr(el);
  const double t_build = tb.elapsed_sec();
  free_edge_list(el);
  Timer ts;
  sort_adj_lists(g_kept);
  const double t_sort = ts.elapsed_sec();
  g_have_kept = true;
  if (seconds) {
    seconds[0] = t_build;
    seconds[1] = t_sort;
  }
  if (n_out) *n_out = g_kept.n;
  if (forward_edges) *forward_edges = g_kept.m;
  return 0;
}

// Sources [0, n_sources) of the kept CSR: their forward edges and their
// merge work, the sum over those edges u -> v of fdeg[u] + fdeg[v] (the
// entries a merge of both lists scans).
int stc_ref_prefix_size(uint32_t n_sources, uint64_t* arcs, uint64_t* merge_work) {
  if (!g_have_kept || n_sources > g_kept.n) return 1;
  uint64_t w = 0;
  for (uint32_t x = 0; x < n_sources; x++)
    for (uint64_t e = g_kept.offsets[x]; e < g_kept.offsets[x + 1]; e++)
      w += (uint64_t)g_kept.fdeg[x] + g_kept.fdeg[g_kept.edges[e]];
  if (arcs) *arcs = g_kept.offsets[n_sources];
  if (merge_work) *merge_work = w;
  return 0;
}

// count_triangles (tc_serial.cpp:138-170), unchanged, over the sources with
// id below n_sources of the kept CSR: it runs on a copy of the CSR header
// whose n is n_sources, while every array stays whole, so each source's
// merges read its neighbours' lists as in a full count.  t[0..3] receives
// the counts of the triangles whose first vertex in the CSR's orientation
// is one of those sources, `seconds` the time of the call.
int stc_ref_count_prefix(uint32_t n_sources, uint64_t t[4], double* seconds) {
  if (!g_have_kept || n_sources > g_kept.n) return 1;
  ForwardCSR view = g_kept;
  view.n = n_sources;
  Timer tc;
  GlobalTriCounts g = count_triangles(view);
  if (seconds) *seconds = tc.elapsed_sec();
  t[0] = g.t0;
  t[1] = g.t1;
  t[2] = g.t2;
  t[3] = g.t3;
  return 0;
}

}  // extern "C"
