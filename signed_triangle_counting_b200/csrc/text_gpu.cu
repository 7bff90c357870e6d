// GPU text ingest: `u v sign` lines parsed on the device, with the grammar
// of load_graph (MC/graph_io.h:72-212) that the host parser
// (text_ingest.cpp) also follows:
//   - the text is split at '\n'; a line's leading '\r' characters are
//     dropped, and an empty remainder is skipped;
//   - a line starting with '#' or '%' is a comment;
//   - otherwise it is a data line (counted in `lines`): a decimal uint32 id
//     (wrapping, no digits = 0), blanks, a second id, blanks, a sign token
//     (a leading '-' is negative, anything else positive); the rest of the
//     line is ignored;
//   - a data line with u == v is dropped; src = min, dst = max; n = max kept
//     id + 1 (1 when no edge is kept, 0 for an empty text).
// Three passes over HBM: newlines are counted per 16-byte chunk and their
// positions scanned into line starts; one thread parses each line; the kept
// edges are compacted by a scan.
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"
#include "radix_sort.cuh"
#include "stc_device.cuh"

namespace stc {
namespace {

constexpr uint32_t kNewline4 = 0x0A0A0A0Au;

// Newlines in 16-byte chunk i.
struct NewlineCount {
  const uint4* text;
  __device__ uint32_t operator()(uint64_t i) const {
    const uint4 q = text[i];
    return (__popc(__vcmpeq4(q.x, kNewline4)) + __popc(__vcmpeq4(q.y, kNewline4)) +
            __popc(__vcmpeq4(q.z, kNewline4)) + __popc(__vcmpeq4(q.w, kNewline4))) >> 3;
  }
};

// Writes the start of the line after each newline of chunk i
// (starts[0] = 0 is written separately).
struct EmitLineStarts {
  const uint4* text;
  uint64_t* starts;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t cnt) const {
    if (!cnt) return;
    const uint4 q = text[i];
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t m = __vcmpeq4(w[k], kNewline4);
      while (m) {
        const int b = (__ffs(m) - 1) >> 3;
        starts[++pos] = 16 * i + 4 * k + b + 1;
        m &= ~(0xFFu << (8 * b));
      }
    }
  }
};

// Line kinds.
constexpr uint8_t kSkip = 0, kSelfLoop = 1, kEdge = 2;

__device__ __forceinline__ uint64_t parse_uint(const char* t, uint64_t p, uint64_t e, uint32_t& out) {
  uint32_t x = 0;
  while (p < e && t[p] >= '0' && t[p] <= '9') x = x * 10u + (uint32_t)(t[p++] - '0');
  out = x;
  return p;
}

__device__ __forceinline__ uint64_t skip_blanks(const char* t, uint64_t p, uint64_t e) {
  while (p < e && (t[p] == ' ' || t[p] == '\t')) p++;
  return p;
}

// One thread per line: kind, and for data lines the ordered pair and sign.
__global__ void k_parse_lines(const char* __restrict__ text, uint64_t size,
                              const uint64_t* __restrict__ starts, uint64_t lines,
                              uint8_t* __restrict__ kind, uint32_t* __restrict__ lo,
                              uint32_t* __restrict__ hi, int8_t* __restrict__ sign,
                              unsigned long long* __restrict__ ctr) {
  uint32_t max_id = 0;
  unsigned long long data_lines = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < lines; s += stride) {
    uint64_t p = starts[s];
    const uint64_t e = s + 1 < lines ? starts[s + 1] - 1 : size;  // the line's '\n' or the end
    while (p < e && text[p] == '\r') p++;
    uint8_t k = kSkip;
    if (p < e && text[p] != '#' && text[p] != '%') {
      uint32_t u, v;
      p = parse_uint(text, p, e, u);
      p = skip_blanks(text, p, e);
      p = parse_uint(text, p, e, v);
      p = skip_blanks(text, p, e);
      const int8_t sg = (p < e && text[p] == '-') ? -1 : 1;
      data_lines++;
      if (u != v) {
        k = kEdge;
        lo[s] = u < v ? u : v;
        hi[s] = u < v ? v : u;
        sign[s] = sg;
        max_id = max(max_id, max(u, v));
      } else {
        k = kSelfLoop;
      }
    }
    kind[s] = k;
  }
  data_lines = warp_sum(data_lines);
  max_id = __reduce_max_sync(kFull, max_id);
  if (lane_id() == 0) {
    if (data_lines) atomicAdd(ctr + C_WORK + 0, data_lines);
    atomicMax(ctr + C_MAX_ID, (unsigned long long)max_id);
  }
}

struct KeptFlag {
  const uint8_t* kind;
  __device__ uint32_t operator()(uint64_t i) const { return kind[i] == kEdge; }
};
struct EmitKept {
  const uint32_t* lo;
  const uint32_t* hi;
  const int8_t* sign;
  uint32_t* src;
  uint32_t* dst;
  int8_t* osign;
  __device__ void operator()(uint64_t i, uint64_t pos, uint32_t keep) const {
    if (!keep) return;
    src[pos] = lo[i];
    dst[pos] = hi[i];
    osign[pos] = sign[i];
  }
};

}  // namespace

// Parses `size` bytes of text at `d_text` (device memory, padded to a
// multiple of 16 bytes with non-newline bytes) into device arrays; returns
// the kept edge count, and the data line count and n through the pointers.
uint64_t parse_text_device(stc_ctx* c, const char* d_text, uint64_t size, uint32_t** src,
                           uint32_t** dst, int8_t** sign, uint64_t* lines_out, uint32_t* n_out) {
  cudaStream_t st = c->stream;
  *lines_out = 0;
  *n_out = 0;
  if (size == 0) {
    *src = buffer<uint32_t>(c, B_IN_SRC, 1);
    *dst = buffer<uint32_t>(c, B_IN_DST, 1);
    *sign = buffer<int8_t>(c, B_IN_SIGN, 1);
    return 0;
  }
  uint64_t* sums = buffer<uint64_t>(c, B_SCAN_SUMS, kMaxSortGrid + 1);
  unsigned long long* ctr = (unsigned long long*)counters(c);
  const uint64_t chunks = (size + 15) / 16;
  const NewlineCount nl{(const uint4*)d_text};
  // Pass 1: newlines per chunk, scanned into line starts.
  const uint32_t grid1 = range_reduce_scan(nl, chunks, sums, st, &c->launches);
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, sums + grid1, sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  const uint64_t nlines = c->h_pinned[C_WORK] + 1;  // the last line may be empty
  uint64_t* starts = buffer<uint64_t>(c, B_KEYS_A, nlines);
  STC_CUDA(cudaMemsetAsync(starts, 0, sizeof(uint64_t), st));
  range_apply(nl, EmitLineStarts{(const uint4*)d_text, starts}, chunks, sums, st, &c->launches);
  // Pass 2: one thread per line.
  uint8_t* kind = buffer<uint8_t>(c, B_WORK2, nlines);
  uint32_t* lo = buffer<uint32_t>(c, B_DEG, nlines);
  uint32_t* hi = buffer<uint32_t>(c, B_RANK, nlines);
  int8_t* sg = buffer<int8_t>(c, B_FDEG, nlines);
  STC_CUDA(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(uint64_t), st));
  STC_CUDA(cudaMemsetAsync(ctr + C_MAX_ID, 0, sizeof(uint64_t), st));
  k_parse_lines<<<kSMs * 8, 256, 0, st>>>(d_text, size, starts, nlines, kind, lo, hi, sg, ctr);
  c->launches++;
  // Pass 3: the kept edges, compacted.
  const KeptFlag keep{kind};
  const uint32_t grid3 = range_reduce_scan(keep, nlines, sums, st, &c->launches);
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_SELF, sums + grid3, sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_WORK, ctr + C_WORK, sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaMemcpyAsync(c->h_pinned + C_MAX_ID, ctr + C_MAX_ID, sizeof(uint64_t),
                           cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  const uint64_t kept = c->h_pinned[C_SELF];
  *lines_out = c->h_pinned[C_WORK];
  *n_out = (uint32_t)c->h_pinned[C_MAX_ID] + 1u;
  *src = buffer<uint32_t>(c, B_IN_SRC, kept);
  *dst = buffer<uint32_t>(c, B_IN_DST, kept);
  *sign = buffer<int8_t>(c, B_IN_SIGN, kept);
  if (kept) range_apply(keep, EmitKept{lo, hi, sg, *src, *dst, *sign}, nlines, sums, st, &c->launches);
  STC_CUDA(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(uint64_t), st));
  STC_CUDA(cudaMemsetAsync(ctr + C_MAX_ID, 0, sizeof(uint64_t), st));
  STC_CUDA(cudaGetLastError());
  return kept;
}

}  // namespace stc
