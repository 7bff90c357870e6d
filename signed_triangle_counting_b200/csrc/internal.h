// Host-side internals of libstc: the context, device buffers and the stages
// of the counting path.  Nothing here crosses the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "stc.h"

namespace stc {

// Internal error carrying an ABI status; caught at every extern "C" entry.
struct Error {
  stc_status status;
  std::string msg;
};

[[noreturn]] void fail(stc_status s, const std::string& msg);
void cuda_check(cudaError_t e, const char* what);
#define STC_CUDA(call) ::stc::cuda_check((call), #call)

// Named device allocations cached on a context and grown on demand.
enum BufId {
  B_IN_SRC, B_IN_DST, B_IN_SIGN,  // staged host input
  B_KEYS_A, B_KEYS_B,             // sort double buffer
  B_UKEYS,                        // unique undirected keys
  B_DEG, B_RANK, B_VERTS, B_FDEG,
  B_VKEYS_A, B_VKEYS_B,
  B_OFF, B_NBR, B_SGN, B_ASRC,
  B_SORT_COUNTS, B_SCAN_SUMS,
  B_COUNTERS,                     // per-type counters, totals, flags
  B_WORK,                         // work queues / strategy worklists
  B_WORK2,
  B_EXPORT_OFF, B_EXPORT_FDEG,
  B_VCOUNTS,
  B_BATCH_META, B_BATCH_SPACE, B_BATCH_COUNTS,
  B_DISPATCH,                     // learned dispatch tables (kTableBytes)
  B_DISPATCH_FIXED,               // fixed dispatch tables (kTableBytes)
  B_DISPATCH_TRAIN,               // dispatcher training samples and parameters
  B_TIMES,                        // timing recorder: cycles and arcs per cell
  B_SHARD_COST,                   // cost prefix of a sharded count (n + 1 words)
  B_TEXT,                         // text input of the GPU parser (padded to 16 bytes)
  B_SPLIT_NBR,                    // sign-split copy of the arc heads (m + 4)
  B_SPLIT_POS,                    // positive arcs per vertex (n)
  B_HEAD_END,                     // head-side pass: end of each arc's tail list (m)
  B_HEAD_RUNS,                    // head-side pass: in-arc range per head vertex (2 n)
  B_HEAD_LIST,                    // head-side pass: head vertices by class, plan, flags
  B_NKEY,                         // arcs: head << 1 | negative (m + 8)
  B_RELABEL,                      // ids >= 2^31 - 1: the edges relabelled to dense ids (2 m)
  B_DISTINCT,                     // ids >= 2^31 - 1: the sorted distinct ids
  B_COUNT_
};

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// Device counters block (B_COUNTERS), 64-bit words.
enum CounterSlot {
  C_T0 = 0, C_T1, C_T2, C_T3,  // per-type triangle counts
  C_MAX_ID = 4,                // max kept id (u32 in the low word)
  C_SELF = 5,                  // self-loop count
  C_MAX_DEG = 6,
  C_ALG_BYTES = 7,
  C_WORK = 8,                  // dynamic work counters (8 slots)
  C_ERROR = 16,                // device error word (0 = ok)
  C_MAX_FDEG = 17,             // largest out-degree of the forward CSR
  C_SHARD_LO = 18,             // rank range [lo, hi) of a sharded count
  C_SHARD_HI = 19,
  C_QUEUE_WARP = 20,           // warp-granular work queue of the persistent engine
  C_HEAD_COUNT = 21,           // head-side pass: head vertices per class (3 slots),
  C_HEAD_CURSOR = 24,          // their list fill cursors (3 slots)
  C_HEAD_QUEUE = 27,           // and the classes' work queues (3 slots)
  C_PROBE_BYTES = 30,          // probe-model bytes of the CSR
  C_HEAD_NKEYS = 31,           // head-side pass: keys (HEAD arcs) appended
  C_BATCH_N = 32,              // capped batch build: vertices of the union
  C_BATCH_MU = 33,             // capped batch build: unique edges (= arcs)
  C_OVERFLOW = 34,             // capped batch build: a capacity was exceeded (results void)
  C_SLOTS = 40
};

// Values of the device error word: 1 = malformed forward CSR,
// 2 = a bounded device-side wait expired, 3 = a list exceeded its staged
// shared-memory capacity (the kernel skipped it instead of overrunning).
constexpr uint64_t kDeviceErrCsr = 1;
constexpr uint64_t kDeviceErrTimeout = 2;

// Dispatch tables: per list class that consults one, a 16 x 16 table
// indexed by (bucket |A'|, bucket |B|), bucket(x) = min(15, bit width of x),
// holding an stc_strategy.  Cell index = 256 * class + 16 * a + b.
enum TableClass { kTableWarp = 0, kTableBlock = 1, kTableLarge = 2, kTableGiant = 3, kTableClasses = 4 };
constexpr size_t kTableBytes = 256 * kTableClasses;
static_assert(kTableBytes == STC_DISPATCH_CELLS, "one table byte per dispatch cell");

// The dispatcher's multilayer perceptron: STC_DISPATCH_FEATURES inputs, one
// hidden ReLU layer, one predicted log2 cost per strategy (MERGE, HASH,
// SEARCH, SPLIT, HEAD).
// Parameter layout: W1[hidden][in], b1[hidden], W2[out][hidden], b2[out].
constexpr int kMlpIn = STC_DISPATCH_FEATURES;
constexpr int kMlpHidden = 16;
constexpr int kMlpOut = STC_DISPATCH_STRATEGIES;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;
static_assert(kMlpParams == STC_DISPATCH_MODEL_PARAMS, "parameter count of the ABI");

// Tuned launch parameters of the staged classes (warp, block, large):
// block-class CTA threads, hash buckets per staged element, and int4 chunks
// in flight per lane in the stream pass.  The defaults are the untuned
// engine.
struct Tuning {
  uint32_t block_threads = 256;
  uint32_t hash_factor[3] = {4, 4, 2};
  uint32_t unroll[3] = {2, 2, 2};
};

// Sizes a batch group's build is launched with when nothing is read back to
// the host between its stages: vertex capacity of the union, id bits of the
// arc keys, degree bits of the vertex sort key and the degree sample shift.
// They come from an earlier build of a group of the same shape; the device
// checks the new group against them (C_OVERFLOW).
struct BatchCaps {
  uint32_t n = 0;
  uint32_t bits = 1;
  uint32_t dbits = 0;
  uint32_t shift = 0;
};

// A batch group's whole pipeline (counters, build, count) as one captured
// CUDA graph: the key it was built for, its capacities, and how far it got
// (1 = capacities known from an uncapped build, 2 = buffers sized by one
// capped run, 3 = captured; -1 = capture failed, always run uncapped).
struct GroupPipeline {
  uint64_t key[16] = {};
  BatchCaps caps;
  int state = 0;
  cudaGraphExec_t exec = nullptr;
  uint64_t gen = 0;   // buffer generation the graph was captured with
  int launches = 0;   // kernels per replay
  uint64_t last_use = 0;
};

}  // namespace stc

struct stc_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  stc::DevBuf bufs[stc::B_COUNT_];
  uint64_t* h_pinned = nullptr;  // C_SLOTS words of pinned host memory
  std::string last_error;
  stc_stats stats{};
  cudaEvent_t ev[8] = {};
  // A sign array copied from host memory on aux_stream while the ids are
  // scanned and ranked (stc_count): ev_sign marks its end, and sign_pending
  // says the call's stream has not waited for it yet (wait_sign).
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_ids = nullptr, ev_sign = nullptr;
  bool sign_pending = false;
  bool timing = false;
  int launches = 0;
  bool fixed_ready = false;   // B_DISPATCH_FIXED holds the fixed tables
  bool model_loaded = false;  // B_DISPATCH holds the tables of a loaded model
  bool learned_uses_split = false;  // the learned tables pick STC_STRATEGY_SPLIT somewhere
  bool learned_uses_head = false;   // ... STC_STRATEGY_HEAD somewhere
  // The persistent count captured in a CUDA graph, and the pointers and
  // sizes it was captured with (replayed while they stay the same).
  cudaGraphExec_t graph_exec = nullptr;
  uint64_t graph_key[24] = {};
  int graph_launches = 0;  // kernels per replay of graph_exec
  stc::Tuning tuning;
  // Batch groups captured whole (at most four, the least recently used
  // replaced), the pinned staging of a group's edge offsets they copy from,
  // and the buffer generation: bumped whenever a device buffer or the
  // staging moves, which retires every captured graph.
  std::vector<stc::GroupPipeline> pipes;
  uint64_t* h_eoff = nullptr;
  size_t h_eoff_cap = 0;
  uint64_t buf_gen = 1;
  uint64_t pipe_clock = 0;
};

namespace stc {

template <class T>
T* buffer(stc_ctx* c, BufId id, size_t count) {
  DevBuf& b = c->bufs[id];
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = 16;
  if (b.cap < bytes) {
    c->buf_gen++;
    if (b.p) STC_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes + bytes / 8;  // headroom for slightly larger reuse
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      e = cudaMalloc(&b.p, bytes);
      want = bytes;
    }
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      b.p = nullptr;
      fail(STC_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    b.cap = want;
  }
  return static_cast<T*>(b.p);
}

// The graph built on the device, in rank space: vertex r is the r-th vertex
// of (degree, id) order, and every arc goes from lower to higher rank.
struct DeviceGraph {
  uint32_t n = 0;        // max kept id + 1
  uint32_t bits = 1;     // bits per id inside a 64-bit key
  uint64_t m_input = 0;
  uint64_t m_valid = 0;  // without self-loops
  uint64_t m_unique = 0;
  uint64_t m_fwd = 0;
  uint32_t max_deg = 0;
  uint64_t* ukeys = nullptr;  // sorted unique keys: min << bits | max, sign in bit 63
  uint32_t* deg = nullptr;    // undirected degree, by id
  uint32_t* rank = nullptr;   // id -> rank
  uint32_t* verts = nullptr;  // rank -> id
  uint64_t* off = nullptr;    // n + 1, rank space
  uint32_t* nbr = nullptr;    // arcs: head vertex (rank), sorted within each list
  int8_t* sgn = nullptr;      // arcs: +1 / -1
  uint32_t* fdeg = nullptr;   // out-degree by rank
  uint32_t* asrc = nullptr;   // arcs: tail vertex (rank)
  uint32_t* nkey = nullptr;   // arcs: head << 1 | negative, padded by 8 (the head side's stream)
  // A capped batch build (BatchCaps) leaves n and m_fwd as capacities: the
  // arc count is then on the device (m_dev), vertices past the union's last
  // rank have no arcs.
  const unsigned long long* m_dev = nullptr;
  uint32_t dbits = 0;  // degree bits of the vertex sort key (totals path)
  uint32_t shift = 0;  // degree sample shift (totals path)
  // Batches: G graphs whose vertices (ids and ranks) are contiguous; graph
  // g owns [gbase[g], gbase[g + 1]).  G == 0 for a single graph.
  uint32_t G = 0;
  uint64_t* gbase = nullptr;
  // Sign-split copy of the arc heads (each list's positive heads, then its
  // negative heads, both ascending) and the positive count per vertex; built
  // when a count uses STC_STRATEGY_SPLIT.
  uint32_t* nbr_split = nullptr;
  uint32_t* psplit = nullptr;
};

// Stage timing helper: records an event when the context is timing.
void mark(stc_ctx* c, int slot);
// Makes the call's stream wait for a sign array still being copied on the
// auxiliary stream (no-op when none is).
void wait_sign(stc_ctx* c);

// Graph build: input device arrays -> DeviceGraph (all fields).  With
// `totals`, for counts of totals only: the vertex order is (degree over the
// input's edge copies, id), so no dedup runs before the orientation (the
// arc sort drops the copies, keeping the first), and g.ukeys stays null.
// Without it, the reference's (unique degree, id) order, which per-vertex
// counts, shards, CSR export, the timing recorder and the autotuner use.
void build_graph(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst, const int8_t* d_sign,
                 uint64_t m, DeviceGraph& g, bool totals = false);
// Rank-space CSR from a reference-layout forward CSR already on the device.
void graph_from_forward_csr(stc_ctx* c, uint32_t n, uint64_t m, const uint64_t* d_off,
                            const uint32_t* d_edges, const int8_t* d_signs, const uint32_t* d_rank,
                            DeviceGraph& g);
// Batch of G graphs stored back to back (host edge offsets h_eoff, G + 1
// entries): the disjoint union with graph-major ranks; sets g.G / g.gbase.
void build_graph_batch(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst,
                       const int8_t* d_sign, uint64_t m, const uint64_t* h_eoff, uint32_t G,
                       DeviceGraph& g, bool totals = false);
// The totals build of a batch at fixed capacities, with no host
// synchronisation (capturable): edge offsets are copied from the pinned
// staging c->h_eoff; g.n and g.m_fwd are capacities and g.m_dev the device
// arc count; C_BATCH_N / C_BATCH_MU receive the real sizes and C_OVERFLOW is
// set when the group does not fit `caps` (its counts are then void).
void build_graph_batch_capped(stc_ctx* c, const uint32_t* d_src, const uint32_t* d_dst,
                              const int8_t* d_sign, uint64_t m, uint32_t G, const BatchCaps& caps,
                              DeviceGraph& g);
// GPU text ingest: parses `size` bytes at d_text (device, padded to a
// multiple of 16 bytes) into the device input arrays; returns the kept edge
// count, the data line count and n.
uint64_t parse_text_device(stc_ctx* c, const char* d_text, uint64_t size, uint32_t** src,
                           uint32_t** dst, int8_t** sign, uint64_t* lines_out, uint32_t* n_out);
// Forward CSR in the reference's id-space layout, copied to host arrays.
void export_forward_csr(stc_ctx* c, const DeviceGraph& g, stc_forward_csr* out);

// Intersection engine: adds per-type counts into the C_T0..C_T3 slots.
struct CountConfig {
  uint32_t strategy = STC_STRATEGY_AUTO;
  uint32_t dispatch = STC_DISPATCH_FIXED;
  uint64_t* vertex_counts = nullptr;  // optional per-source counts, 4 per vertex id
  uint64_t* graph_counts = nullptr;   // optional per-graph counts of a batch, 4 per graph
  // Timing recorder (device arrays of kTableBytes words, or null): adds each
  // arc's SM cycles and one arc to its dispatch cell.
  uint64_t* arc_cycles = nullptr;
  uint64_t* arc_counts = nullptr;
  // Sharded count: only source vertices of shard `shard` of `shards` (equal
  // merge-model cost ranges of rank space); the range lands in
  // C_SHARD_LO / C_SHARD_HI.
  uint32_t shard = 0;
  uint32_t shards = 1;
  // Persistent engine captured in a CUDA graph (STC_F_PERSISTENT).
  bool persistent = false;
  // Vertex classes to count (bit c: class c = tiny, warp, block, large,
  // giant; bit 5: the head-side pass); the autotuner times one class at a
  // time.
  uint32_t class_mask = 0x3F;
};
void count_triangles(stc_ctx* c, const DeviceGraph& g, const CountConfig& cfg);

// Dispatch: the fixed tables (kTableBytes, host), the per-cell features
// (kTableBytes x kMlpIn, host), the learned tables of a model computed on
// the device into B_DISPATCH, and the on-device training of a model.
void fixed_dispatch_tables(uint8_t* out, bool head = true);
void dispatch_features(float* out);
const uint8_t* dispatch_tables(stc_ctx* c, const CountConfig& cfg, bool* uses_head = nullptr);
void load_dispatch_model(stc_ctx* c, const float* params, const uint8_t* support);
void train_dispatcher(stc_ctx* c, const float* features, const float* targets,
                      const float* weights, uint32_t samples, uint32_t epochs, float lr, float wd,
                      uint64_t seed, float* params, float* loss);

uint64_t* counters(stc_ctx* c);

}  // namespace stc
