/* stc — signed triangle counting on NVIDIA B200 (sm_100a), C ABI.
 *
 * Drop-in boundary for the counting path of NikhilBisht2/Signed_Triangle_Counting
 * ("Signed_TC/Multicore Implementations/", abbreviated MC/ below, and the
 * Gunrock plug-ins under "Signed_TC/GPU Implementations/", abbreviated GM/).
 *
 * Rules of the ABI: plain C types only, no exceptions cross it, every call
 * returns an stc_status, and buffers passed in are owned by the caller.
 * Buffers the library returns (edge lists, forward CSRs) are released with
 * the matching stc_free_* call.  Device memory is owned by an stc_ctx; use
 * one context per host thread (a context is not thread-safe).
 *
 * Semantics follow the reference CPU code:
 *  - an edge line/element (u, v, s) with u == v is dropped (MC/graph_io.h:191);
 *  - s < 0 means a negative edge, anything else positive (MC/graph_io.h:84-97);
 *  - (u, v) and (v, u) are the same undirected edge; duplicates keep their
 *    first occurrence (MC/graph_io.h:221-259);
 *  - vertices are ordered by (degree, id) and every edge is oriented from the
 *    lower to the higher vertex of that order (MC/graph_io.h:261-330);
 *  - a triangle's type is its number of negative edges: 0 -> T3 (+++),
 *    1 -> T2 (++-), 2 -> T1 (+--), 3 -> T0 (---) (MC/tc_serial.cpp:95-112).
 * Counts of totals (stc_count, stc_count_text, batches of graphs whose ids
 * stay below 2^31 - 1 in all) take any 32-bit vertex id: a list whose
 * largest id reaches 2^31 - 1 is relabelled on the device to dense ids in
 * the same order first, which changes no count.  Calls that report per
 * vertex or per id (vertex counts, CSR export, shards, the timing recorder
 * and the autotuner) need ids below 2^31 - 1.  An edge list stays below
 * 2^32 elements, and a list's distinct ids below 2^31 - 1.
 */
#ifndef STC_H
#define STC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STC_ABI_VERSION 2

typedef enum stc_status {
  STC_OK = 0,
  STC_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad option, malformed CSR */
  STC_ERR_IO = 2,               /* file cannot be opened / read (MC/graph_io.h:40-59) */
  STC_ERR_CUDA = 3,             /* a CUDA call failed; see stc_ctx_last_error */
  STC_ERR_OUT_OF_MEMORY = 4,    /* host or device allocation failed */
  STC_ERR_LIMIT = 5,            /* id >= 2^31 - 1 where ids are reported, list >= 2^32 elements */
  STC_ERR_DEVICE_TIMEOUT = 6,   /* a bounded device-side wait expired */
  STC_ERR_NO_DEVICE = 7,        /* no CUDA device, or not an sm_100 part */
  STC_ERR_INTERNAL = 8          /* a self-check failed (e.g. strategies disagree) */
} stc_status;

/* GlobalTriCounts (MC/tc_serial.cpp:11-31). */
typedef struct stc_counts {
  uint64_t t0; /* --- unbalanced */
  uint64_t t1; /* +-- balanced   */
  uint64_t t2; /* ++- unbalanced */
  uint64_t t3; /* +++ balanced   */
} stc_counts;

static inline uint64_t stc_balanced(const stc_counts* c) { return c->t1 + c->t3; }
static inline uint64_t stc_unbalanced(const stc_counts* c) { return c->t0 + c->t2; }
static inline uint64_t stc_total(const stc_counts* c) { return c->t0 + c->t1 + c->t2 + c->t3; }

/* EdgeList (MC/graph_io.h:14-20) plus the reference's `raw_edges` line count. */
typedef struct stc_edge_list {
  uint32_t n;      /* max kept id + 1 */
  uint64_t lines;  /* non-blank, non-comment lines (printed as raw_edges) */
  uint64_t m;      /* kept edges */
  uint32_t* src;   /* min endpoint */
  uint32_t* dst;   /* max endpoint */
  int8_t* sign;    /* +1 / -1 */
} stc_edge_list;

/* ForwardCSR (MC/graph_io.h:22-30) with every list sorted by neighbour id,
 * i.e. as MC/tc_serial.cpp:33-93 (sort_adj_lists) leaves it. */
typedef struct stc_forward_csr {
  uint32_t n;
  uint64_t m;        /* forward edges */
  uint64_t* offsets; /* n + 1 */
  uint32_t* edges;   /* m */
  int8_t* signs;     /* m */
  uint32_t* fdeg;    /* n */
  uint32_t* rank;    /* n: position of each vertex in (degree, id) order */
} stc_forward_csr;

/* One graph of a batch (host or device arrays, see STC_F_DEVICE_INPUT). */
typedef struct stc_graph {
  const uint32_t* src;
  const uint32_t* dst;
  const int8_t* sign;
  uint64_t m;
} stc_graph;

/* Intersection strategy selection. */
typedef enum stc_strategy {
  STC_STRATEGY_AUTO = 0,   /* dispatcher picks per edge bucket (default) */
  STC_STRATEGY_MERGE = 1,  /* force the warp-cooperative sorted merge */
  STC_STRATEGY_HASH = 2,   /* force the shared-memory hash probe */
  STC_STRATEGY_SEARCH = 3, /* force binary search / galloping */
  STC_STRATEGY_SPLIT = 4,  /* force the sign-split stream: B is read from a copy of the
                              forward CSR whose lists hold their positive heads, then
                              their negative heads, so a head's sign follows from its
                              position and no sign byte is loaded; each element is
                              probed in the staged hash of N+(u)
                              (MC/tc_merge_sign_split.cpp:20-146, GM/signed_tc.hxx:302-396) */
  STC_STRATEGY_HEAD = 5    /* force the head-side probe where it applies: the arc u -> v
                              is counted while the head's list N+(v) is staged as a
                              shared-memory hash, by streaming A' (the part of N+(u) after
                              v) through it; the other probe direction of the reference's
                              hash program, which iterates the shorter list and probes the
                              other's table (MC/tc_hash_sign_enu.cpp:146-160).  It applies
                              to arcs with 1 <= |N+(v)| <= 4095; other arcs run HASH */
} stc_strategy;

typedef enum stc_dispatch {
  STC_DISPATCH_FIXED = 0,   /* fixed degree thresholds (fallback) */
  STC_DISPATCH_LEARNED = 1  /* learned per-bucket choice, when a model is loaded */
} stc_dispatch;

/* Option flags. */
#define STC_F_DEVICE_INPUT 0x1u /* input pointers are device pointers */
#define STC_F_TIMING 0x2u       /* record per-stage device times (stc_ctx_last_stats) */
#define STC_F_PERSISTENT 0x8u   /* count with the persistent engine: the device plans the
                                   class worklists and one persistent kernel pulls lists
                                   from a device work queue; the sequence is captured in a
                                   CUDA graph once per set of buffers and replayed (on the
                                   legacy default stream it is launched directly) */

typedef struct stc_opts {
  uint32_t strategy; /* stc_strategy */
  uint32_t dispatch; /* stc_dispatch */
  uint32_t flags;    /* STC_F_* */
  uint32_t reserved;
  void* stream;      /* cudaStream_t to run on; NULL = the context's own stream */
} stc_opts;

/* Per-call statistics of the last call on a context. */
typedef struct stc_stats {
  uint64_t n;             /* vertices */
  uint64_t m_input;       /* input edges */
  uint64_t m_unique;      /* undirected edges after dedup */
  uint64_t m_forward;     /* forward edges (arcs) */
  uint64_t alg_bytes;     /* merge-model bytes: sum over arcs of 5 (d+(u) + d+(v)) + 25 */
  uint64_t triangles;     /* total */
  double ms_h2d;          /* host -> device copy of the input */
  double ms_dedup;        /* ingest, sort, unique */
  double ms_orient;       /* degree, (degree, id) rank, orientation */
  double ms_csr;          /* forward CSR build (arc sort, offsets) */
  double ms_count;        /* intersection engine */
  double ms_total;        /* whole call on the device */
  uint32_t kernel_launches;
  uint32_t groups_replayed; /* batch groups run as one replayed CUDA graph (persistent engine) */
  uint64_t probe_bytes;   /* probe-model bytes: sum over arcs of 5 min(|A'|, |B|) + 30, the
                             shorter list of each arc streamed once (A' = the part of N+(u)
                             after v, B = N+(v)), the arc's 25 bytes and its entry staged */
} stc_stats;

typedef struct stc_ctx stc_ctx;

/* ------------------------------------------------------------ context ---- */
/* Opens a context on CUDA device `device`.  Fails with STC_ERR_NO_DEVICE when
 * the device is missing or not compute capability 10.x. */
stc_status stc_ctx_create(int device, stc_ctx** out);
void stc_ctx_destroy(stc_ctx* ctx);
/* Message of the last failure on this context ("" when none). */
const char* stc_ctx_last_error(const stc_ctx* ctx);
stc_status stc_ctx_last_stats(const stc_ctx* ctx, stc_stats* out);
/* Releases the context's cached device buffers. */
stc_status stc_ctx_trim(stc_ctx* ctx);
const char* stc_status_string(stc_status s);
int stc_abi_version(void);

/* --------------------------------------------------------------- ingest ---- */
/* load_graph / free_edge_list (MC/graph_io.h:100-219): parses a `u v sign`
 * text file on the host ('#'/'%' lines are comments) with all host threads. */
stc_status stc_load_edge_list(const char* path, stc_edge_list* out);
/* Same parse over an in-memory buffer. */
stc_status stc_parse_edge_text(const char* data, uint64_t size, stc_edge_list* out);
void stc_free_edge_list(stc_edge_list* el);

/* MatrixMarket input, for the graphs the reference's GPU drivers read
 * (GM/tc_split/signed_tc.cu:21-33): a `%%MatrixMarket matrix coordinate`
 * file, field real, double, integer or pattern, symmetry general or
 * symmetric, 1-based entries `i j [w]`.  Vertex i - 1 and j - 1 get an
 * undirected edge, diagonal entries are dropped, and `n` is the matrix
 * dimension.  Signs: w < 0 is negative by default (the rule of the CPU
 * programs' text input); with STC_MTX_ZERO_NEGATIVE, w <= 0 is negative,
 * the GPU drivers' rule (GM/signed_tc.hxx:317); weights are read as float
 * as there, and pattern entries are positive.  A malformed header, an
 * index out of range or an entry count that differs from the size line's
 * returns STC_ERR_INVALID_ARGUMENT.  Free with stc_free_edge_list. */
#define STC_MTX_ZERO_NEGATIVE 0x1u
stc_status stc_load_mtx(const char* path, uint32_t flags, stc_edge_list* out);
stc_status stc_parse_mtx(const char* data, uint64_t size, uint32_t flags, stc_edge_list* out);

/* ---------------------------------------------------------- whole path ---- */
/* The reference programs' path (MC/tc_serial.cpp:172-210; the Gunrock
 * plug-in GM/signed_tc.hxx:527-542): dedup, (degree, id) orientation, forward
 * CSR with int8 signs and the intersection engine, all on the GPU.
 * src/dst/sign are host arrays, or device arrays with STC_F_DEVICE_INPUT. */
stc_status stc_count(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                     const int8_t* sign, uint64_t m, const stc_opts* opts,
                     stc_counts* out);

/* One shard of stc_count, for counting one graph on several GPUs (one
 * process per GPU, each building the same forward CSR; no counterpart in the
 * reference, whose programs use one machine).  Shard `shard` of `shards`
 * (shards <= 65535) counts only the triangles whose lowest vertex in
 * (degree, id) order has its rank in the shard's range; the ranges split
 * rank space into contiguous pieces of about equal merge-model cost (vertex
 * u costs 1 + the sum over its forward arcs u -> v of d+(u) + d+(v),
 * saturated at 2^32 - 1; shard s starts at the first rank whose cost prefix
 * reaches ceil(total * s / shards)).  The shards' counts add up to
 * stc_count's, so the caller sums them across processes (one all-reduce of
 * four words).  `range_out` (optional, 2 words) receives the shard's rank
 * range [lo, hi). */
stc_status stc_count_shard(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                           const int8_t* sign, uint64_t m, const stc_opts* opts, uint32_t shard,
                           uint32_t shards, stc_counts* out, uint64_t* range_out);

/* The whole path from `u v sign` text, parsed on the GPU: load_graph's
 * grammar (MC/graph_io.h:72-212, as stc_parse_edge_text) followed by
 * stc_count.  `data` is host memory, or device memory with
 * STC_F_DEVICE_INPUT; it is copied into a device buffer and split into lines,
 * parsed and compacted by kernels.  `info` (optional) receives the data line
 * count and n as stc_parse_edge_text reports them.  stats.ms_h2d covers the
 * copy and the parse. */
typedef struct stc_text_info {
  uint64_t lines; /* data lines (the reference's raw_edges) */
  uint32_t n;     /* max kept id + 1 (1 when no edge is kept, 0 for empty text) */
  uint32_t reserved;
} stc_text_info;
stc_status stc_count_text(stc_ctx* ctx, const char* data, uint64_t size, const stc_opts* opts,
                          stc_counts* out, stc_text_info* info);

/* The GPU parser's edge list, copied to host arrays (free with
 * stc_free_edge_list): identical to stc_parse_edge_text's for the same
 * bytes. */
stc_status stc_parse_edge_text_gpu(stc_ctx* ctx, const char* data, uint64_t size,
                                   const stc_opts* opts, stc_edge_list* out);

/* build_forward_csr + sort_adj_lists (MC/graph_io.h:231-402,
 * MC/tc_serial.cpp:33-93) on the GPU; the result is returned in host memory
 * in the reference's layout.  Free with stc_free_forward_csr. */
stc_status stc_build_forward_csr(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                 const int8_t* sign, uint64_t m, const stc_opts* opts,
                                 stc_forward_csr* out);
void stc_free_forward_csr(stc_forward_csr* csr);

/* count_triangles (MC/tc_serial.cpp:138-170) over a host forward CSR in the
 * reference layout (lists sorted by id, every edge from lower to higher rank). */
stc_status stc_count_forward_csr(stc_ctx* ctx, const stc_forward_csr* csr,
                                 const stc_opts* opts, stc_counts* out);

/* Per-source counts, the cnt[4n] array of MC/tc_serial.cpp:141-158: entry
 * 4u + k is the number of type-k triangles (k = 0..3 as in stc_counts) whose
 * lowest-ranked vertex is u.  `counts` is a host array of 4 * n words where n
 * is max id + 1 of the kept edges. */
stc_status stc_vertex_counts(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                             const int8_t* sign, uint64_t m, const stc_opts* opts,
                             uint64_t* counts, uint64_t counts_len, uint32_t* n_out);

/* ---------------------------------------------------------------- batch ---- */
/* Counts G independent graphs (gathered on the device, then counted as by
 * stc_count_batch_packed); outs[g] receives graph g's counts. */
stc_status stc_count_batch(stc_ctx* ctx, const stc_graph* graphs, uint32_t G,
                           const stc_opts* opts, stc_counts* outs);

/* ------------------------------------------------------- no allocation ---- */
/* No counterpart in the reference.  Counts the triangles of an oriented
 * forward CSR that already sits in device memory, and allocates nothing:
 * for callers that cannot call cudaMalloc, such as code that must draw all
 * device memory from its own pool or allocator, or that runs inside a memory
 * budget where an allocation by a library would fail or fragment the heap.
 * Input: d_offsets (n + 1 entries), d_heads and d_signs (m entries each plus
 * 4 readable padding entries; d_heads 16-byte aligned, d_signs 4-byte
 * aligned); each list sorted ascending and each head above its tail (any
 * acyclic orientation gives the same counts); a negative sign byte marks a
 * negative edge.  The input is checked on the device first: a malformed CSR
 * returns STC_ERR_INVALID_ARGUMENT.  Limits: n <= 4,194,304 and m < 2^32,
 * else STC_ERR_LIMIT.
 * Scratch: one file-scope device array of about 16 MiB, which every GPU that
 * loads the library keeps until the process exits.  All calls share it, so
 * calls that overlap on the GPU race.  The first call in a CUDA context
 * looks up the array's device address there (cudaGetSymbolAddress) with
 * that context current, and a call looks it up again when the current
 * context is not the one it last saw on that device (after cudaDeviceReset,
 * or under a caller's own context); make the first call in a context before
 * any stream capture.  `stream` may be NULL (the legacy default stream). */
stc_status stc_count_oriented_csr_noalloc(const uint64_t* d_offsets, const uint32_t* d_heads,
                                          const int8_t* d_signs, uint32_t n, uint64_t m,
                                          void* stream, stc_counts* out);

/* Counts G graphs stored back to back: graph g owns elements
 * [offsets[g], offsets[g + 1]) of src/dst/sign (host arrays, or device arrays
 * with STC_F_DEVICE_INPUT) with ids local to the graph; `offsets` is a host
 * array of G + 1 entries and outs[g] receives graph g's counts.  The graphs
 * are counted together as one disjoint union whose vertex order is
 * graph-major and (degree, id) within each graph, so every graph is oriented
 * exactly as it would be alone.  With STC_F_PERSISTENT on a stream other
 * than the legacy default stream, each group of graphs (at most 1.5 Gi
 * input edges) is captured whole, build and count, as one CUDA graph on its
 * third call with the same input pointers, sizes and options, and replayed
 * on every call after that while the context's buffers stay in place
 * (stc_stats.groups_replayed); a group whose graphs outgrow the sizes it
 * was captured at is counted again without the graph, with the same
 * results.  No counterpart in the reference, which counts one graph per
 * process. */
stc_status stc_count_batch_packed(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                  const int8_t* sign, const uint64_t* offsets, uint32_t G,
                                  const stc_opts* opts, stc_counts* outs);

/* ----------------------------------------------------------- dispatcher ---- */
/* No counterpart in the reference, whose programs each run one strategy
 * (merge in MC/tc_merge_sign_enu.cpp, hash in MC/tc_hash_sign_enu.cpp).
 * Every arc u -> v falls in a dispatch cell: the class of u's list (0 = warp,
 * |N+(u)| <= 128; 1 = block, <= 1024; 2 = large, <= 4096; 3 = giant) and the
 * buckets a = min(15, bit width of |A'|), b = min(15, bit width of |B|),
 * where A' is the part of N+(u) after v and B = N+(v).  Cell index =
 * 256 class + 16 a + b.  A dispatch table holds one stc_strategy per cell;
 * all strategies give the same counts, so a table changes only speed. */
#define STC_DISPATCH_CELLS 1024
#define STC_DISPATCH_FEATURES 6
#define STC_DISPATCH_STRATEGIES 5
#define STC_DISPATCH_MODEL_PARAMS 197

/* Timing recorder: the whole path as stc_count (opts->strategy is usually
 * forced to one strategy), with every arc of the staged and giant classes
 * processed alone by one warp and timed.  cycles[cell] receives the SM
 * cycles spent on the cell's arcs and arcs[cell] their number
 * (STC_DISPATCH_CELLS words each).  Lists of 8 or fewer arcs, which are
 * otherwise counted one thread per list, join the warp class here, so that
 * runs with different forced strategies time the same arcs.  `out` receives
 * the counts, which equal stc_count's. */
stc_status stc_record_bucket_times(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                   const int8_t* sign, uint64_t m, const stc_opts* opts,
                                   uint64_t* cycles, uint64_t* arcs, stc_counts* out);

/* Input features of every cell (STC_DISPATCH_CELLS x STC_DISPATCH_FEATURES
 * floats, row-major), computed on the host: the log-bucketed lengths a and
 * b, their difference (the log of the |B| / |A'| ratio), a log-degree
 * representative of u's class and its difference to b (the log of the
 * deg(u) / deg(v) ratio), and whether the class stages a hash, each scaled
 * to about [-1, 1]. */
stc_status stc_dispatch_features(float* out);

/* Trains the dispatcher's perceptron on the device.  The perceptron has
 * STC_DISPATCH_FEATURES inputs, 16 hidden ReLU units and one output per
 * strategy (STC_DISPATCH_STRATEGIES: MERGE, HASH, SEARCH, SPLIT, HEAD): the
 * predicted log2 of the SM cycles one arc of the cell costs under that
 * strategy.  Training is full-batch Adam over `samples` rows of `features`,
 * `targets` (samples x STC_DISPATCH_STRATEGIES measured log2 cycles per arc,
 * NaN where a strategy is unavailable) and non-negative `weights`,
 * minimising the weighted squared error plus weight_decay / 2 times the
 * squared weights.  Deterministic for a given seed.  `params` receives the
 * STC_DISPATCH_MODEL_PARAMS trained parameters (W1[16][6], b1[16], W2[5][16],
 * b2[5]) and `loss` (optional) the final weighted squared error.
 * samples <= 4096. */
stc_status stc_dispatcher_train(stc_ctx* ctx, const float* features, const float* targets,
                                const float* weights, uint32_t samples, uint32_t epochs,
                                float learning_rate, float weight_decay, uint64_t seed,
                                float* params, float* loss);

/* Loads a trained model into the context: an inference kernel evaluates it
 * on every cell and writes the learned tables on the device.  A cell takes
 * the strategy of least predicted cost where that is predicted at least 5%
 * cheaper than the fixed table's choice, and keeps the fixed choice
 * elsewhere (the giant class, which stages no hash, never gets HASH or
 * SPLIT; HEAD only to cells where the fixed table holds it, since the
 * recorder does not time the head side's sort and staging).  `support` (optional, STC_DISPATCH_CELLS bytes) limits the
 * overrides to the cells marked non-zero, normally the cells the model's
 * training data covered, so that the model is not trusted where it would
 * extrapolate; NULL allows them everywhere.  Calls with dispatch
 * STC_DISPATCH_LEARNED then use these tables.  params = NULL unloads the
 * model; without a model, LEARNED falls back to the fixed tables. */
stc_status stc_ctx_set_dispatch_model(stc_ctx* ctx, const float* params, const uint8_t* support);

/* Copies to `out` (STC_DISPATCH_CELLS bytes) the tables a call with
 * strategy AUTO and this dispatch would use on this context. */
stc_status stc_dispatch_tables(stc_ctx* ctx, uint32_t dispatch, uint8_t* out);

/* ------------------------------------------------------------ autotuner ---- */
/* No counterpart in the reference.  Launch parameters of the three staged
 * list classes (index 0 = warp class, |N+(u)| <= 128; 1 = block, <= 1024;
 * 2 = large, <= 4096), used by the per-class kernels (not by the persistent
 * engine, which keeps the defaults). */
typedef struct stc_tuning {
  uint32_t block_threads;  /* CTA threads of the block class: 128, 256 (default) or 512 */
  uint32_t hash_factor[3]; /* hash buckets (of two keys) per staged element: 2, 4 or 8;
                              defaults 4, 4, 2; lowered where the table would not fit
                              a CTA's shared memory */
  uint32_t unroll[3];      /* int4 chunks of B in flight per lane in the stream pass
                              (the merge tile width): 1, 2 (default) or 4 */
} stc_tuning;

/* Sets the context's tuning (NULL restores the defaults); values outside the
 * lists above return STC_ERR_INVALID_ARGUMENT. */
stc_status stc_ctx_set_tuning(stc_ctx* ctx, const stc_tuning* tuning);
stc_status stc_ctx_get_tuning(const stc_ctx* ctx, stc_tuning* out);

/* Autotuner: builds the graph of (src, dst, sign) once, in the order counts
 * of totals use, then, class by class (warp, block, large), counts that
 * class alone, on both sides of the engine (the tail side's lists and the
 * head side's heads of that class), under every candidate setting (hash
 * factor x unroll, and for the block class x block threads),
 * `reps` times each, timed with CUDA events, and keeps the fastest.  Every
 * candidate must give the same counts (else STC_ERR_INTERNAL).  The result
 * is set on the context and copied to `out`. */
stc_status stc_autotune(stc_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                        const int8_t* sign, uint64_t m, const stc_opts* opts, uint32_t reps,
                        stc_tuning* out);

/* --------------------------------------------------- device generator ---- */
/* Writes the RMAT samples of stc_synth_rmat (include/stc_synth.h) for the
 * same arguments directly into device arrays of `samples` elements. */
stc_status stc_synth_rmat_device(stc_ctx* ctx, uint64_t seed, uint32_t scale, uint64_t n,
                                 uint64_t samples, double a, double b, double c, double p_pos,
                                 uint32_t* d_src, uint32_t* d_dst, int8_t* d_sign);

#ifdef __cplusplus
}
#endif

#endif /* STC_H */
