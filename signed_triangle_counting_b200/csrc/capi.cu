// C ABI of libstc (include/stc.h): contexts, the whole counting path, CSR
// export/import, per-source counts and the device RMAT generator.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <new>
#include <string>
#include <vector>

#include "internal.h"
#include "stc.h"
#include "stc_device.cuh"
#include "stc_gen.h"
#include "stc_synth.h"

namespace stc {

void fail(stc_status s, const std::string& msg) { throw Error{s, msg}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  (void)cudaGetLastError();
  fail(e == cudaErrorMemoryAllocation ? STC_ERR_OUT_OF_MEMORY : STC_ERR_CUDA,
       std::string(what) + ": " + cudaGetErrorString(e));
}

uint64_t* counters(stc_ctx* c) { return buffer<uint64_t>(c, B_COUNTERS, C_SLOTS); }

void mark(stc_ctx* c, int slot) {
  if (!c->timing) return;
  // Inside a capture the event becomes a node of the graph that records it
  // on every replay (an external record), so stage times stay readable.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (c->stream != nullptr && c->stream != cudaStreamLegacy && c->stream != cudaStreamPerThread)
    STC_CUDA(cudaStreamIsCapturing(c->stream, &cs));
  if (cs == cudaStreamCaptureStatusActive)
    STC_CUDA(cudaEventRecordWithFlags(c->ev[slot], c->stream, cudaEventRecordExternal));
  else
    STC_CUDA(cudaEventRecord(c->ev[slot], c->stream));
}

void wait_sign(stc_ctx* c) {
  if (!c->sign_pending) return;
  c->sign_pending = false;
  STC_CUDA(cudaStreamWaitEvent(c->stream, c->ev_sign, 0));
}

void release_pipelines(stc_ctx* c) {
  for (auto& p : c->pipes)
    if (p.exec) cudaGraphExecDestroy(p.exec);
  c->pipes.clear();
}

namespace {

// Runs `body` with the context's error handling; every ABI entry uses it.
template <class F>
stc_status guarded(stc_ctx* c, F body) {
  try {
    if (c) {
      c->last_error.clear();
      STC_CUDA(cudaSetDevice(c->device));
    }
    body();
    return STC_OK;
  } catch (const Error& e) {
    if (c) c->last_error = e.msg;
    if (c && c->sign_pending) {  // the caller's sign array stays in use until the copy ends
      c->sign_pending = false;
      cudaStreamSynchronize(c->aux_stream);
      (void)cudaGetLastError();
    }
    return e.status;
  } catch (const std::bad_alloc&) {
    if (c) c->last_error = "host allocation failed";
    return STC_ERR_OUT_OF_MEMORY;
  } catch (...) {
    if (c) c->last_error = "unexpected internal error";
    return STC_ERR_INTERNAL;
  }
}

void begin_call(stc_ctx* c, const stc_opts* o) {
  c->stream = (o && o->stream) ? (cudaStream_t)o->stream : c->own_stream;
  c->timing = o && (o->flags & STC_F_TIMING);
  c->launches = 0;
  c->stats = stc_stats{};
  STC_CUDA(cudaMemsetAsync(counters(c), 0, C_SLOTS * sizeof(uint64_t), c->stream));
  mark(c, 0);
}

float elapsed(stc_ctx* c, int a, int b) {
  float ms = 0.f;
  STC_CUDA(cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]));
  return ms;
}

// Reads the per-type counters and fills the statistics.
void end_call(stc_ctx* c, const DeviceGraph& g, stc_counts* out) {
  STC_CUDA(cudaMemcpyAsync(c->h_pinned, counters(c), C_SLOTS * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, c->stream));
  STC_CUDA(cudaStreamSynchronize(c->stream));
  STC_CUDA(cudaGetLastError());
  if (c->h_pinned[C_ERROR]) {
    const uint64_t e = c->h_pinned[C_ERROR];
    fail(e == kDeviceErrTimeout ? STC_ERR_DEVICE_TIMEOUT : STC_ERR_INTERNAL,
         "device reported error word " + std::to_string(e));
  }
  if (out) {
    out->t0 = c->h_pinned[C_T0];
    out->t1 = c->h_pinned[C_T1];
    out->t2 = c->h_pinned[C_T2];
    out->t3 = c->h_pinned[C_T3];
  }
  stc_stats& s = c->stats;
  s.n = g.n;
  s.m_input = g.m_input;
  s.m_unique = g.m_unique;
  s.m_forward = g.m_fwd;
  s.alg_bytes = c->h_pinned[C_ALG_BYTES];
  s.probe_bytes = c->h_pinned[C_PROBE_BYTES];
  s.triangles = c->h_pinned[C_T0] + c->h_pinned[C_T1] + c->h_pinned[C_T2] + c->h_pinned[C_T3];
  s.kernel_launches = (uint32_t)c->launches;
  if (c->timing) {
    s.ms_h2d = elapsed(c, 0, 1);
    s.ms_dedup = elapsed(c, 1, 2);
    s.ms_orient = elapsed(c, 2, 3);
    s.ms_csr = elapsed(c, 3, 4);
    s.ms_count = elapsed(c, 4, 5);
    s.ms_total = elapsed(c, 0, 5);
  }
}

struct DeviceInput {
  const uint32_t* src;
  const uint32_t* dst;
  const int8_t* sign;
};

// Device copies of host input (device input as it is).  With defer_sign
// the sign array is copied on the auxiliary stream after the ids, so that
// it overlaps the id scan, degrees and ranking; the build waits for it
// (wait_sign) before its first read of the signs.
DeviceInput stage_input(stc_ctx* c, const uint32_t* src, const uint32_t* dst, const int8_t* sign,
                        uint64_t m, const stc_opts* o, bool defer_sign = false) {
  if (m && (!src || !dst || !sign)) fail(STC_ERR_INVALID_ARGUMENT, "null edge array");
  if (o && (o->flags & STC_F_DEVICE_INPUT)) return DeviceInput{src, dst, sign};
  uint32_t* ds = buffer<uint32_t>(c, B_IN_SRC, m);
  uint32_t* dd = buffer<uint32_t>(c, B_IN_DST, m);
  int8_t* dg = buffer<int8_t>(c, B_IN_SIGN, m);
  if (m) {
    STC_CUDA(cudaMemcpyAsync(ds, src, m * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    STC_CUDA(cudaMemcpyAsync(dd, dst, m * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    if (defer_sign) {
      STC_CUDA(cudaEventRecord(c->ev_ids, c->stream));
      STC_CUDA(cudaStreamWaitEvent(c->aux_stream, c->ev_ids, 0));
      STC_CUDA(cudaMemcpyAsync(dg, sign, m, cudaMemcpyHostToDevice, c->aux_stream));
      STC_CUDA(cudaEventRecord(c->ev_sign, c->aux_stream));
      c->sign_pending = true;
    } else {
      STC_CUDA(cudaMemcpyAsync(dg, sign, m, cudaMemcpyHostToDevice, c->stream));
    }
  }
  return DeviceInput{ds, dd, dg};
}

// Graphs of a batch are counted in groups of at most this many edges (one
// pass of the union pipeline each), which bounds the device memory a batch
// needs to about 45 bytes per edge of a group.
constexpr uint64_t kBatchGroupEdges = 1536ull << 20;

// ------------------------------------------------- batch group pipeline ----
// A group of a batch on the persistent engine runs as one captured CUDA
// graph once it has been seen: counters, offsets upload, the whole totals
// build and the count, with no host synchronisation between the stages.
// The build then cannot read sizes back, so it runs at capacities (BatchCaps)
// taken from an earlier, uncapped build of a group with the same key (input
// pointers, sizes and count configuration), and the device checks that the
// new data fits them.  A group that does not fit (C_OVERFLOW) is counted
// again uncapped and its sizes become the new capacities.  Sequence for one
// key: uncapped (learns capacities) -> capped, uncaptured (sizes every
// buffer, so that the capture allocates nothing) -> captured and replayed
// on every later call while no device buffer has moved (c->buf_gen).
constexpr size_t kMaxPipelines = 4;

// Capacities from an uncapped build: vertices with 1/16 headroom, as far as
// the id bits allow.
bool caps_from(const DeviceGraph& g, BatchCaps& caps) {
  if (g.n == 0 || g.m_fwd == 0) return false;
  caps.bits = std::max<uint32_t>(1, bit_width64(g.n - 1));
  const uint64_t room = std::min<uint64_t>(1ull << caps.bits, (1ull << 31) - 2);
  caps.n = (uint32_t)std::max<uint64_t>(g.n, std::min<uint64_t>(g.n + g.n / 16 + 64, room));
  caps.dbits = g.dbits;
  caps.shift = g.shift;
  return true;
}

void stage_offsets(stc_ctx* c, const std::vector<uint64_t>& eoff) {
  if (c->h_eoff_cap < eoff.size()) {
    STC_CUDA(cudaStreamSynchronize(c->stream));  // no earlier copy still reads it
    if (c->h_eoff) STC_CUDA(cudaFreeHost(c->h_eoff));
    c->h_eoff = nullptr;
    c->h_eoff_cap = 0;
    const size_t want = eoff.size() + eoff.size() / 8;
    STC_CUDA(cudaMallocHost(&c->h_eoff, want * sizeof(uint64_t)));
    c->h_eoff_cap = want;
    c->buf_gen++;
  }
  memcpy(c->h_eoff, eoff.data(), eoff.size() * sizeof(uint64_t));
}

// Per-graph counts (4 per graph) into h and the counters into c->h_pinned.
void finish_group(stc_ctx* c, uint32_t gn, std::vector<uint64_t>& h) {
  const uint64_t* gc = buffer<uint64_t>(c, B_BATCH_COUNTS, 4ull * gn);
  STC_CUDA(cudaMemcpyAsync(h.data(), gc, 4ull * gn * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                           c->stream));
  STC_CUDA(cudaMemcpyAsync(c->h_pinned, counters(c), C_SLOTS * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, c->stream));
  STC_CUDA(cudaStreamSynchronize(c->stream));
}

struct GroupOut {
  uint64_t n = 0, m_unique = 0;
  bool replayed = false;
};

GroupOut eager_group(stc_ctx* c, const DeviceInput& in, uint64_t me,
                     const std::vector<uint64_t>& eoff, uint32_t gn, CountConfig cfg,
                     std::vector<uint64_t>& h, DeviceGraph& g) {
  STC_CUDA(cudaMemsetAsync(counters(c), 0, C_SLOTS * sizeof(uint64_t), c->stream));
  build_graph_batch(c, in.src, in.dst, in.sign, me, eoff.data(), gn, g, /*totals=*/true);
  uint64_t* gc = buffer<uint64_t>(c, B_BATCH_COUNTS, 4ull * gn);
  STC_CUDA(cudaMemsetAsync(gc, 0, 4ull * gn * sizeof(uint64_t), c->stream));
  cfg.graph_counts = gc;
  count_triangles(c, g, cfg);
  mark(c, 5);
  finish_group(c, gn, h);
  return GroupOut{g.n, g.m_unique, false};
}

// The capturable sequence of a group at capacities `caps`.
void enqueue_capped_group(stc_ctx* c, const DeviceInput& in, uint64_t me, uint32_t gn,
                          const BatchCaps& caps, CountConfig cfg) {
  STC_CUDA(cudaMemsetAsync(counters(c), 0, C_SLOTS * sizeof(uint64_t), c->stream));
  uint64_t* gc = buffer<uint64_t>(c, B_BATCH_COUNTS, 4ull * gn);
  STC_CUDA(cudaMemsetAsync(gc, 0, 4ull * gn * sizeof(uint64_t), c->stream));
  DeviceGraph g;
  build_graph_batch_capped(c, in.src, in.dst, in.sign, me, gn, caps, g);
  cfg.graph_counts = gc;
  count_triangles(c, g, cfg);
  mark(c, 5);
}

enum class Capture { kOk, kRetry, kFailed };

Capture capture_group(stc_ctx* c, GroupPipeline& p, const DeviceInput& in, uint64_t me,
                      uint32_t gn, const CountConfig& cfg) {
  if (p.exec) {
    STC_CUDA(cudaGraphExecDestroy(p.exec));
    p.exec = nullptr;
  }
  const uint64_t gen0 = c->buf_gen;
  const int l0 = c->launches;
  cudaGraph_t graph = nullptr;
  STC_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  try {
    enqueue_capped_group(c, in, me, gn, p.caps, cfg);
  } catch (...) {
    cudaStreamEndCapture(c->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    (void)cudaGetLastError();
    c->launches = l0;
    return Capture::kFailed;
  }
  STC_CUDA(cudaStreamEndCapture(c->stream, &graph));
  const int launches = c->launches - l0;
  c->launches = l0;
  if (c->buf_gen != gen0) {  // a buffer grew inside the capture: size it uncaptured first
    cudaGraphDestroy(graph);
    return Capture::kRetry;
  }
  const cudaError_t e = cudaGraphInstantiate(&p.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    p.exec = nullptr;
    return Capture::kFailed;
  }
  p.gen = c->buf_gen;
  p.launches = launches;
  p.state = 3;
  return Capture::kOk;
}

// Counts one group of a batch (see the pipeline notes above); h receives
// its per-graph counts and c->h_pinned the counters.
GroupOut count_group(stc_ctx* c, const DeviceInput& in, uint64_t me,
                     const std::vector<uint64_t>& eoff, uint32_t gn, const CountConfig& cfg,
                     std::vector<uint64_t>& h) {
  DeviceGraph g;
  const bool stream_ok = c->stream != nullptr && c->stream != cudaStreamLegacy &&
                         c->stream != cudaStreamPerThread;
  const bool learned_split = cfg.strategy == STC_STRATEGY_AUTO &&
                             cfg.dispatch == STC_DISPATCH_LEARNED && c->model_loaded &&
                             c->learned_uses_split;
  if (!cfg.persistent || me == 0 || !stream_ok || cfg.strategy == STC_STRATEGY_SPLIT ||
      learned_split)
    return eager_group(c, in, me, eoff, gn, cfg, h, g);

  uint64_t key[16] = {};
  key[0] = reinterpret_cast<uint64_t>(in.src);
  key[1] = reinterpret_cast<uint64_t>(in.dst);
  key[2] = reinterpret_cast<uint64_t>(in.sign);
  key[3] = me;
  key[4] = gn;
  key[5] = (uint64_t)cfg.strategy | ((uint64_t)cfg.dispatch << 8) |
           ((uint64_t)c->model_loaded << 16) | ((uint64_t)c->learned_uses_head << 17) |
           ((uint64_t)c->timing << 18) | ((uint64_t)cfg.class_mask << 24);
  key[6] = reinterpret_cast<uint64_t>(c->stream);
  const Tuning& tu = c->tuning;
  key[7] = (uint64_t)tu.block_threads | ((uint64_t)tu.hash_factor[0] << 16) |
           ((uint64_t)tu.hash_factor[1] << 24) | ((uint64_t)tu.hash_factor[2] << 32) |
           ((uint64_t)tu.unroll[0] << 40) | ((uint64_t)tu.unroll[1] << 48) |
           ((uint64_t)tu.unroll[2] << 56);
  GroupPipeline* p = nullptr;
  for (auto& q : c->pipes)
    if (memcmp(q.key, key, sizeof(key)) == 0) p = &q;
  if (!p) {
    const GroupOut o = eager_group(c, in, me, eoff, gn, cfg, h, g);
    if (c->pipes.size() >= kMaxPipelines) {  // replace the least recently used
      auto lru = c->pipes.begin();
      for (auto it = c->pipes.begin(); it != c->pipes.end(); ++it)
        if (it->last_use < lru->last_use) lru = it;
      if (lru->exec) STC_CUDA(cudaGraphExecDestroy(lru->exec));
      c->pipes.erase(lru);
    }
    GroupPipeline q;
    memcpy(q.key, key, sizeof(key));
    q.state = caps_from(g, q.caps) ? 1 : -1;
    q.last_use = ++c->pipe_clock;
    c->pipes.push_back(q);
    return o;
  }
  p->last_use = ++c->pipe_clock;
  if (p->state < 0) return eager_group(c, in, me, eoff, gn, cfg, h, g);
  stage_offsets(c, eoff);
  bool replayed = false;
  if (p->state >= 2 && (p->state == 2 || !p->exec || p->gen != c->buf_gen)) {
    const Capture r = capture_group(c, *p, in, me, gn, cfg);
    if (r == Capture::kFailed) {
      p->state = -1;
      return eager_group(c, in, me, eoff, gn, cfg, h, g);
    }
    if (r == Capture::kRetry) p->state = 1;
  }
  if (p->state == 3) {
    STC_CUDA(cudaGraphLaunch(p->exec, c->stream));
    c->launches += p->launches;
    replayed = true;
  } else {
    enqueue_capped_group(c, in, me, gn, p->caps, cfg);
  }
  finish_group(c, gn, h);
  if (c->h_pinned[C_OVERFLOW]) {
    if (p->exec) STC_CUDA(cudaGraphExecDestroy(p->exec));
    p->exec = nullptr;
    const GroupOut o = eager_group(c, in, me, eoff, gn, cfg, h, g);
    p->state = caps_from(g, p->caps) ? 1 : -1;
    return o;
  }
  if (p->state == 1) p->state = 2;
  return GroupOut{c->h_pinned[C_BATCH_N], c->h_pinned[C_BATCH_MU], replayed};
}

CountConfig count_config(const stc_opts* o) {
  CountConfig cfg;
  if (o) {
    if (o->strategy > STC_STRATEGY_HEAD) fail(STC_ERR_INVALID_ARGUMENT, "unknown strategy");
    if (o->dispatch > STC_DISPATCH_LEARNED) fail(STC_ERR_INVALID_ARGUMENT, "unknown dispatch");
    cfg.strategy = o->strategy;
    cfg.dispatch = o->dispatch;
    cfg.persistent = (o->flags & STC_F_PERSISTENT) != 0;
  }
  return cfg;
}

__global__ void k_synth_rmat(uint64_t seed, stcgen::RmatParams rp, stcgen::Perm perm,
                             uint64_t pos_thr, uint64_t samples, uint32_t* __restrict__ src,
                             uint32_t* __restrict__ dst, int8_t* __restrict__ sign) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < samples; i += stride) {
    uint32_t u, v;
    stcgen::rmat_sample(seed, i, rp, &u, &v);
    u = (uint32_t)stcgen::perm_apply(perm, u);
    v = (uint32_t)stcgen::perm_apply(perm, v);
    src[i] = u;
    dst[i] = v;
    sign[i] = stcgen::edge_sign(seed, u, v, pos_thr);
  }
}

}  // namespace
}  // namespace stc

using namespace stc;

extern "C" {

const char* stc_status_string(stc_status s) {
  switch (s) {
    case STC_OK: return "ok";
    case STC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case STC_ERR_IO: return "i/o error";
    case STC_ERR_CUDA: return "CUDA error";
    case STC_ERR_OUT_OF_MEMORY: return "out of memory";
    case STC_ERR_LIMIT: return "input beyond supported limits";
    case STC_ERR_DEVICE_TIMEOUT: return "device-side wait expired";
    case STC_ERR_NO_DEVICE: return "no usable CUDA device";
    case STC_ERR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

int stc_abi_version(void) { return STC_ABI_VERSION; }

stc_status stc_ctx_create(int device, stc_ctx** out) {
  if (!out) return STC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    (void)cudaGetLastError();
    return STC_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    (void)cudaGetLastError();
    return STC_ERR_NO_DEVICE;
  }
  stc_ctx* c = new (std::nothrow) stc_ctx();
  if (!c) return STC_ERR_OUT_OF_MEMORY;
  c->device = device;
  stc_status s = guarded(c, [&] {
    STC_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    STC_CUDA(cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking));
    STC_CUDA(cudaEventCreateWithFlags(&c->ev_ids, cudaEventDisableTiming));
    STC_CUDA(cudaEventCreateWithFlags(&c->ev_sign, cudaEventDisableTiming));
    c->stream = c->own_stream;
    STC_CUDA(cudaMallocHost(&c->h_pinned, C_SLOTS * sizeof(uint64_t)));
    for (auto& e : c->ev) STC_CUDA(cudaEventCreate(&e));
    (void)counters(c);
  });
  if (s != STC_OK) {
    stc_ctx_destroy(c);
    return s;
  }
  *out = c;
  return STC_OK;
}

void stc_ctx_destroy(stc_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->own_stream) cudaStreamSynchronize(c->own_stream);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  release_pipelines(c);
  for (auto& b : c->bufs)
    if (b.p) cudaFree(b.p);
  if (c->h_eoff) cudaFreeHost(c->h_eoff);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->aux_stream) {
    cudaStreamSynchronize(c->aux_stream);
    cudaStreamDestroy(c->aux_stream);
  }
  if (c->ev_ids) cudaEventDestroy(c->ev_ids);
  if (c->ev_sign) cudaEventDestroy(c->ev_sign);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  (void)cudaGetLastError();
  delete c;
}

const char* stc_ctx_last_error(const stc_ctx* c) { return c ? c->last_error.c_str() : ""; }

stc_status stc_ctx_last_stats(const stc_ctx* c, stc_stats* out) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  *out = c->stats;
  return STC_OK;
}

stc_status stc_ctx_trim(stc_ctx* c) {
  if (!c) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    STC_CUDA(cudaStreamSynchronize(c->own_stream));
    if (c->graph_exec) {  // it refers to the buffers released below
      STC_CUDA(cudaGraphExecDestroy(c->graph_exec));
      c->graph_exec = nullptr;
    }
    release_pipelines(c);
    c->buf_gen++;
    for (int i = 0; i < B_COUNT_; i++) {
      if (i == B_COUNTERS) continue;
      if (c->bufs[i].p) STC_CUDA(cudaFree(c->bufs[i].p));
      c->bufs[i] = DevBuf{};
    }
  });
}

stc_status stc_count(stc_ctx* c, const uint32_t* src, const uint32_t* dst, const int8_t* sign,
                     uint64_t m, const stc_opts* o, stc_counts* out) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    DeviceInput in = stage_input(c, src, dst, sign, m, o, /*defer_sign=*/true);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g, /*totals=*/true);
    wait_sign(c);
    count_triangles(c, g, cfg);
    mark(c, 5);
    end_call(c, g, out);
  });
}

stc_status stc_count_shard(stc_ctx* c, const uint32_t* src, const uint32_t* dst,
                           const int8_t* sign, uint64_t m, const stc_opts* o, uint32_t shard,
                           uint32_t shards, stc_counts* out, uint64_t* range_out) {
  if (!c || !out || shards == 0 || shards > 65535 || shard >= shards)
    return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    cfg.shard = shard;
    cfg.shards = shards;
    begin_call(c, o);
    DeviceInput in = stage_input(c, src, dst, sign, m, o);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g);
    count_triangles(c, g, cfg);
    mark(c, 5);
    end_call(c, g, out);
    if (range_out) {
      const bool split = shards > 1 && g.n && g.m_fwd;
      range_out[0] = split ? c->h_pinned[C_SHARD_LO] : (shard == 0 ? 0 : g.n);
      range_out[1] = split ? c->h_pinned[C_SHARD_HI] : (shard == 0 ? g.n : g.n);
    }
  });
}

namespace {

// Copies text (host, or device with STC_F_DEVICE_INPUT) into B_TEXT, padded
// with zero bytes to a multiple of 16, and parses it on the device.
uint64_t stage_and_parse_text(stc_ctx* c, const char* data, uint64_t size, const stc_opts* o,
                              DeviceInput* in, uint64_t* lines, uint32_t* n) {
  if (size && !data) fail(STC_ERR_INVALID_ARGUMENT, "null text");
  const uint64_t padded = (size + 15) & ~15ull;
  char* d_text = buffer<char>(c, B_TEXT, padded ? padded : 16);
  if (size) {
    const bool dev = o && (o->flags & STC_F_DEVICE_INPUT);
    STC_CUDA(cudaMemcpyAsync(d_text, data, size, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                             c->stream));
    if (padded > size) STC_CUDA(cudaMemsetAsync(d_text + size, 0, padded - size, c->stream));
  }
  uint32_t* s = nullptr;
  uint32_t* d = nullptr;
  int8_t* g = nullptr;
  const uint64_t m = parse_text_device(c, d_text, size, &s, &d, &g, lines, n);
  *in = DeviceInput{s, d, g};
  return m;
}

}  // namespace

stc_status stc_count_text(stc_ctx* c, const char* data, uint64_t size, const stc_opts* o,
                          stc_counts* out, stc_text_info* info) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    DeviceInput in;
    uint64_t lines = 0;
    uint32_t n = 0;
    const uint64_t m = stage_and_parse_text(c, data, size, o, &in, &lines, &n);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g, /*totals=*/true);
    count_triangles(c, g, cfg);
    mark(c, 5);
    end_call(c, g, out);
    if (info) *info = stc_text_info{lines, size ? n : 0u, 0u};
  });
}

stc_status stc_parse_edge_text_gpu(stc_ctx* c, const char* data, uint64_t size,
                                   const stc_opts* o, stc_edge_list* out) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  return guarded(c, [&] {
    begin_call(c, o);
    DeviceInput in;
    uint64_t lines = 0;
    uint32_t n = 0;
    const uint64_t m = stage_and_parse_text(c, data, size, o, &in, &lines, &n);
    const uint64_t cap = m ? m : 1;
    out->src = (uint32_t*)malloc(cap * sizeof(uint32_t));
    out->dst = (uint32_t*)malloc(cap * sizeof(uint32_t));
    out->sign = (int8_t*)malloc(cap);
    if (!out->src || !out->dst || !out->sign) {
      stc_free_edge_list(out);
      fail(STC_ERR_OUT_OF_MEMORY, "host allocation of the edge list failed");
    }
    if (m) {
      STC_CUDA(cudaMemcpyAsync(out->src, in.src, m * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               c->stream));
      STC_CUDA(cudaMemcpyAsync(out->dst, in.dst, m * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               c->stream));
      STC_CUDA(cudaMemcpyAsync(out->sign, in.sign, m, cudaMemcpyDeviceToHost, c->stream));
    }
    STC_CUDA(cudaStreamSynchronize(c->stream));
    out->n = size ? n : 0;
    out->lines = lines;
    out->m = m;
  });
}

stc_status stc_build_forward_csr(stc_ctx* c, const uint32_t* src, const uint32_t* dst,
                                 const int8_t* sign, uint64_t m, const stc_opts* o,
                                 stc_forward_csr* out) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  return guarded(c, [&] {
    begin_call(c, o);
    DeviceInput in = stage_input(c, src, dst, sign, m, o);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g);
    export_forward_csr(c, g, out);
    mark(c, 5);
    end_call(c, g, nullptr);
  });
}

void stc_free_forward_csr(stc_forward_csr* csr) {
  if (!csr) return;
  free(csr->offsets);
  free(csr->edges);
  free(csr->signs);
  free(csr->fdeg);
  free(csr->rank);
  memset(csr, 0, sizeof(*csr));
}

stc_status stc_count_forward_csr(stc_ctx* c, const stc_forward_csr* csr, const stc_opts* o,
                                 stc_counts* out) {
  if (!c || !csr || !out) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    const uint32_t n = csr->n;
    const uint64_t m = csr->m;
    if (!csr->offsets || (n && !csr->rank) || (m && (!csr->edges || !csr->signs)))
      fail(STC_ERR_INVALID_ARGUMENT, "null CSR array");
    if (csr->offsets[0] != 0 || csr->offsets[n] != m)
      fail(STC_ERR_INVALID_ARGUMENT, "offsets[0] must be 0 and offsets[n] must equal m");
    for (uint32_t v = 0; v < n; v++)
      if (csr->offsets[v + 1] < csr->offsets[v])
        fail(STC_ERR_INVALID_ARGUMENT, "offsets are not monotone");
    {
      std::vector<uint8_t> seen(n, 0);
      for (uint32_t v = 0; v < n; v++) {
        if (csr->rank[v] >= n || seen[csr->rank[v]])
          fail(STC_ERR_INVALID_ARGUMENT, "rank is not a permutation of [0, n)");
        seen[csr->rank[v]] = 1;
      }
    }
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    uint64_t* d_off = buffer<uint64_t>(c, B_EXPORT_OFF, (size_t)n + 1);
    uint32_t* d_edges = buffer<uint32_t>(c, B_IN_SRC, m);
    int8_t* d_signs = buffer<int8_t>(c, B_IN_SIGN, m);
    uint32_t* d_rank = buffer<uint32_t>(c, B_IN_DST, n);
    STC_CUDA(cudaMemcpyAsync(d_off, csr->offsets, ((size_t)n + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, c->stream));
    if (m) {
      STC_CUDA(cudaMemcpyAsync(d_edges, csr->edges, m * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               c->stream));
      STC_CUDA(cudaMemcpyAsync(d_signs, csr->signs, m, cudaMemcpyHostToDevice, c->stream));
    }
    if (n)
      STC_CUDA(cudaMemcpyAsync(d_rank, csr->rank, (size_t)n * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, c->stream));
    DeviceGraph g;
    graph_from_forward_csr(c, n, m, d_off, d_edges, d_signs, d_rank, g);
    count_triangles(c, g, cfg);
    mark(c, 5);
    end_call(c, g, out);
  });
}

stc_status stc_vertex_counts(stc_ctx* c, const uint32_t* src, const uint32_t* dst,
                             const int8_t* sign, uint64_t m, const stc_opts* o, uint64_t* counts,
                             uint64_t counts_len, uint32_t* n_out) {
  if (!c || !n_out) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    DeviceInput in = stage_input(c, src, dst, sign, m, o);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g);
    *n_out = g.n;
    if (!counts || counts_len < 4ull * g.n)
      fail(STC_ERR_INVALID_ARGUMENT, "counts must hold 4 * n = " + std::to_string(4ull * g.n) +
                                         " words");
    uint64_t* dv = buffer<uint64_t>(c, B_VCOUNTS, 4ull * g.n);
    if (g.n) STC_CUDA(cudaMemsetAsync(dv, 0, 4ull * g.n * sizeof(uint64_t), c->stream));
    cfg.vertex_counts = dv;
    count_triangles(c, g, cfg);
    mark(c, 5);
    if (g.n)
      STC_CUDA(cudaMemcpyAsync(counts, dv, 4ull * g.n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                               c->stream));
    end_call(c, g, nullptr);
  });
}

stc_status stc_count_batch_packed(stc_ctx* c, const uint32_t* src, const uint32_t* dst,
                                  const int8_t* sign, const uint64_t* offsets, uint32_t G,
                                  const stc_opts* o, stc_counts* outs) {
  if (!c || (G && (!offsets || !outs))) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    if (G == 0) return;
    if (offsets[0] != 0) fail(STC_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (uint32_t i = 0; i < G; i++)
      if (offsets[i + 1] < offsets[i]) fail(STC_ERR_INVALID_ARGUMENT, "offsets decrease");
    const uint64_t M = offsets[G];
    if (M && (!src || !dst || !sign)) fail(STC_ERR_INVALID_ARGUMENT, "null edge array");
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    const bool dev = o && (o->flags & STC_F_DEVICE_INPUT);
    stc_stats total{};
    uint32_t g0 = 0;
    while (g0 < G) {
      // Group of graphs whose edges fit one pass of the union pipeline.
      uint32_t g1 = g0 + 1;
      while (g1 < G && offsets[g1 + 1] - offsets[g0] <= kBatchGroupEdges) g1++;
      const uint64_t e0 = offsets[g0], me = offsets[g1] - e0;
      const uint32_t gn = g1 - g0;
      std::vector<uint64_t> eoff(gn + 1);
      for (uint32_t i = 0; i <= gn; i++) eoff[i] = offsets[g0 + i] - e0;
      DeviceInput in;
      if (dev) {
        in = DeviceInput{src + e0, dst + e0, sign + e0};
      } else {
        in = stage_input(c, src + e0, dst + e0, sign + e0, me, o);
      }
      std::vector<uint64_t> h(4ull * gn);
      const GroupOut go = count_group(c, in, me, eoff, gn, cfg, h);
      if (c->h_pinned[C_ERROR])
        fail(STC_ERR_INTERNAL, "device reported error word " + std::to_string(c->h_pinned[C_ERROR]));
      if (c->timing) {  // stage times summed over the groups
        total.ms_dedup += elapsed(c, 1, 2);
        total.ms_orient += elapsed(c, 2, 3);
        total.ms_csr += elapsed(c, 3, 4);
        total.ms_count += elapsed(c, 4, 5);
      }
      for (uint32_t i = 0; i < gn; i++) {
        stc_counts& r = outs[g0 + i];
        r.t0 = h[4ull * i + 0];
        r.t1 = h[4ull * i + 1];
        r.t2 = h[4ull * i + 2];
        r.t3 = h[4ull * i + 3];
        total.triangles += r.t0 + r.t1 + r.t2 + r.t3;
      }
      total.n += go.n;
      total.m_input += me;
      total.m_unique += go.m_unique;
      total.m_forward += go.m_unique;
      total.alg_bytes += c->h_pinned[C_ALG_BYTES];
      total.probe_bytes += c->h_pinned[C_PROBE_BYTES];
      total.groups_replayed += go.replayed ? 1 : 0;
      g0 = g1;
    }
    mark(c, 7);
    STC_CUDA(cudaStreamSynchronize(c->stream));
    total.kernel_launches = (uint32_t)c->launches;
    if (c->timing) total.ms_total = elapsed(c, 0, 7);
    c->stats = total;
  });
}

stc_status stc_count_batch(stc_ctx* c, const stc_graph* graphs, uint32_t G, const stc_opts* o,
                           stc_counts* outs) {
  if (!c || (G && (!graphs || !outs))) return STC_ERR_INVALID_ARGUMENT;
  // Gathers the graphs back to back on the device, then counts them packed.
  std::vector<uint64_t> off(G + 1, 0);
  for (uint32_t i = 0; i < G; i++) off[i + 1] = off[i] + graphs[i].m;
  const bool dev = o && (o->flags & STC_F_DEVICE_INPUT);
  stc_status s = guarded(c, [&] {
    const uint64_t M = off[G];
    cudaStream_t st = (o && o->stream) ? (cudaStream_t)o->stream : c->own_stream;
    uint32_t* ds = buffer<uint32_t>(c, B_IN_SRC, M);
    uint32_t* dd = buffer<uint32_t>(c, B_IN_DST, M);
    int8_t* dg = buffer<int8_t>(c, B_IN_SIGN, M);
    const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (uint32_t i = 0; i < G; i++) {
      const uint64_t m = graphs[i].m;
      if (!m) continue;
      if (!graphs[i].src || !graphs[i].dst || !graphs[i].sign)
        fail(STC_ERR_INVALID_ARGUMENT, "null edge array in graph " + std::to_string(i));
      STC_CUDA(cudaMemcpyAsync(ds + off[i], graphs[i].src, m * sizeof(uint32_t), kind, st));
      STC_CUDA(cudaMemcpyAsync(dd + off[i], graphs[i].dst, m * sizeof(uint32_t), kind, st));
      STC_CUDA(cudaMemcpyAsync(dg + off[i], graphs[i].sign, m, kind, st));
    }
  });
  if (s != STC_OK) return s;
  stc_opts o2 = o ? *o : stc_opts{};
  o2.flags |= STC_F_DEVICE_INPUT;
  return stc_count_batch_packed(c, static_cast<const uint32_t*>(c->bufs[B_IN_SRC].p),
                                static_cast<const uint32_t*>(c->bufs[B_IN_DST].p),
                                static_cast<const int8_t*>(c->bufs[B_IN_SIGN].p), off.data(), G,
                                &o2, outs);
}

stc_status stc_record_bucket_times(stc_ctx* c, const uint32_t* src, const uint32_t* dst,
                                   const int8_t* sign, uint64_t m, const stc_opts* o,
                                   uint64_t* cycles, uint64_t* arcs, stc_counts* out) {
  if (!c || !cycles || !arcs || !out) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    begin_call(c, o);
    uint64_t* times = buffer<uint64_t>(c, B_TIMES, 2 * kTableBytes);
    STC_CUDA(cudaMemsetAsync(times, 0, 2 * kTableBytes * sizeof(uint64_t), c->stream));
    cfg.arc_cycles = times;
    cfg.arc_counts = times + kTableBytes;
    DeviceInput in = stage_input(c, src, dst, sign, m, o);
    DeviceGraph g;
    build_graph(c, in.src, in.dst, in.sign, m, g);
    count_triangles(c, g, cfg);
    mark(c, 5);
    STC_CUDA(cudaMemcpyAsync(cycles, times, kTableBytes * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                             c->stream));
    STC_CUDA(cudaMemcpyAsync(arcs, times + kTableBytes, kTableBytes * sizeof(uint64_t),
                             cudaMemcpyDeviceToHost, c->stream));
    end_call(c, g, out);
  });
}

stc_status stc_dispatch_features(float* out) {
  if (!out) return STC_ERR_INVALID_ARGUMENT;
  dispatch_features(out);
  return STC_OK;
}

stc_status stc_dispatcher_train(stc_ctx* c, const float* features, const float* targets,
                                const float* weights, uint32_t samples, uint32_t epochs,
                                float learning_rate, float weight_decay, uint64_t seed,
                                float* params, float* loss) {
  if (!c) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->stream = c->own_stream;
    train_dispatcher(c, features, targets, weights, samples, epochs, learning_rate, weight_decay,
                     seed, params, loss);
  });
}

stc_status stc_ctx_set_dispatch_model(stc_ctx* c, const float* params, const uint8_t* support) {
  if (!c) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->stream = c->own_stream;
    load_dispatch_model(c, params, support);
  });
}

stc_status stc_dispatch_tables(stc_ctx* c, uint32_t dispatch, uint8_t* out) {
  if (!c || !out || dispatch > STC_DISPATCH_LEARNED) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->stream = c->own_stream;
    CountConfig cfg;
    cfg.dispatch = dispatch;
    const uint8_t* t = dispatch_tables(c, cfg);
    STC_CUDA(cudaMemcpyAsync(out, t, kTableBytes, cudaMemcpyDeviceToHost, c->stream));
    STC_CUDA(cudaStreamSynchronize(c->stream));
  });
}

namespace {

bool valid_tuning(const stc_tuning& t) {
  auto in = [](uint32_t v, std::initializer_list<uint32_t> ok) {
    for (uint32_t x : ok)
      if (v == x) return true;
    return false;
  };
  if (!in(t.block_threads, {128, 256, 512})) return false;
  for (int i = 0; i < 3; i++)
    if (!in(t.hash_factor[i], {2, 4, 8}) || !in(t.unroll[i], {1, 2, 4})) return false;
  return true;
}

stc_tuning to_abi(const Tuning& t) {
  stc_tuning o;
  o.block_threads = t.block_threads;
  for (int i = 0; i < 3; i++) {
    o.hash_factor[i] = t.hash_factor[i];
    o.unroll[i] = t.unroll[i];
  }
  return o;
}

Tuning from_abi(const stc_tuning& o) {
  Tuning t;
  t.block_threads = o.block_threads;
  for (int i = 0; i < 3; i++) {
    t.hash_factor[i] = o.hash_factor[i];
    t.unroll[i] = o.unroll[i];
  }
  return t;
}

}  // namespace

stc_status stc_ctx_set_tuning(stc_ctx* c, const stc_tuning* t) {
  if (!c) return STC_ERR_INVALID_ARGUMENT;
  if (!t) {
    c->tuning = Tuning{};
    return STC_OK;
  }
  if (!valid_tuning(*t)) return STC_ERR_INVALID_ARGUMENT;
  c->tuning = from_abi(*t);
  return STC_OK;
}

stc_status stc_ctx_get_tuning(const stc_ctx* c, stc_tuning* out) {
  if (!c || !out) return STC_ERR_INVALID_ARGUMENT;
  *out = to_abi(c->tuning);
  return STC_OK;
}

stc_status stc_autotune(stc_ctx* c, const uint32_t* src, const uint32_t* dst, const int8_t* sign,
                        uint64_t m, const stc_opts* o, uint32_t reps, stc_tuning* out) {
  if (!c || !out || reps == 0 || reps > 100) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    CountConfig cfg = count_config(o);
    cfg.persistent = false;
    begin_call(c, o);
    DeviceInput in = stage_input(c, src, dst, sign, m, o);
    DeviceGraph g;
    // The order counts of totals use (stc_count), whose head side takes
    // most of the count on power-law graphs.
    build_graph(c, in.src, in.dst, in.sign, m, g, /*totals=*/true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    STC_CUDA(cudaEventCreate(&e0));
    STC_CUDA(cudaEventCreate(&e1));
    Tuning best = c->tuning;
    try {
      // One class at a time; candidates of the other classes do not matter
      // to its time.  Index into the class mask: warp = 1, block = 2, large = 3.
      for (int k = 0; k < 3; k++) {
        std::vector<Tuning> cands;
        const uint32_t hfs[3] = {2, 4, 8};
        const uint32_t us[3] = {1, 2, 4};
        const uint32_t ts[3] = {128, 256, 512};
        for (uint32_t hf : hfs)
          for (uint32_t u : us)
            for (int ti = 0; ti < (k == 1 ? 3 : 1); ti++) {
              Tuning t = best;
              t.hash_factor[k] = hf;
              t.unroll[k] = u;
              if (k == 1) t.block_threads = ts[ti];
              cands.push_back(t);
            }
        // The class on both sides: the tail side's class k and the head
        // side's (bit 5 runs the head pass: its keys, sort and runs are the
        // same for every candidate, its class-k kernel is not).
        cfg.class_mask = (1u << (k + 1)) | 0x20u;
        float best_ms = 0.f;
        bool first = true;
        uint64_t want[4] = {0, 0, 0, 0};
        for (const Tuning& t : cands) {
          c->tuning = t;
          float t_min = 0.f;
          for (uint32_t r = 0; r < reps; r++) {
            STC_CUDA(cudaMemsetAsync(counters(c), 0, 4 * sizeof(uint64_t), c->stream));
            STC_CUDA(cudaEventRecord(e0, c->stream));
            count_triangles(c, g, cfg);
            STC_CUDA(cudaEventRecord(e1, c->stream));
            STC_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            STC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r == 0 || ms < t_min) t_min = ms;
          }
          uint64_t got[C_SLOTS];
          STC_CUDA(cudaMemcpy(got, counters(c), sizeof(got), cudaMemcpyDeviceToHost));
          if (got[C_ERROR])
            fail(STC_ERR_INTERNAL, "device reported error word " + std::to_string(got[C_ERROR]));
          if (first) {
            memcpy(want, got, sizeof(want));
          } else if (memcmp(want, got, sizeof(want)) != 0) {
            fail(STC_ERR_INTERNAL, "autotuner: a candidate setting changed the counts");
          }
          if (first || t_min < best_ms) {
            best_ms = t_min;
            best.hash_factor[k] = t.hash_factor[k];
            best.unroll[k] = t.unroll[k];
            if (k == 1) best.block_threads = t.block_threads;
          }
          first = false;
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tuning = best;
    *out = to_abi(best);
    STC_CUDA(cudaStreamSynchronize(c->stream));
  });
}

stc_status stc_synth_rmat_device(stc_ctx* c, uint64_t seed, uint32_t scale, uint64_t n,
                                 uint64_t samples, double a, double b, double cc, double p_pos,
                                 uint32_t* d_src, uint32_t* d_dst, int8_t* d_sign) {
  if (!c || !d_src || !d_dst || !d_sign) return STC_ERR_INVALID_ARGUMENT;
  if (scale == 0 || scale > 31 || n < 2 || n > (1ull << scale)) return STC_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    auto thr32 = [](double p) -> uint32_t {
      if (!(p > 0.0)) return 0;
      if (p >= 1.0) return UINT32_MAX;
      return (uint32_t)ldexp(p, 32);
    };
    stcgen::RmatParams rp;
    rp.scale = scale;
    rp.n = n;
    rp.t_a = thr32(a);
    rp.t_ab = thr32(a + b);
    rp.t_abc = thr32(a + b + cc);
    uint64_t thr = !(p_pos > 0.0) ? 0 : p_pos >= 1.0 ? UINT64_MAX : (uint64_t)ldexp(p_pos, 64);
    stcgen::Perm perm = stcgen::make_perm(seed, n);
    k_synth_rmat<<<kSMs * 16, 256, 0, c->own_stream>>>(seed, rp, perm, thr, samples, d_src, d_dst,
                                                       d_sign);
    STC_CUDA(cudaGetLastError());
    STC_CUDA(cudaStreamSynchronize(c->own_stream));
  });
}

}  // extern "C"
