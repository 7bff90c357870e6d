// Host text ingest: `u v sign` lines -> stc_edge_list.
//
// Same grammar as load_graph (MC/graph_io.h:72-212): lines starting with
// '#' or '%' are comments, blank lines and stray '\r' are skipped, ids are
// decimal uint32 (wrap-around, no leading blanks), a sign token starting with
// '-' is negative and anything else positive, a line with u == v is dropped,
// src = min and dst = max.  The file is split into line-aligned byte ranges;
// each thread counts its lines, then parses them into its slice of the output
// and the slices are compacted (self-loops leave no hole behind, unlike the
// reference, whose arrays are sized by line count: MC/graph_io.h:147,157-161).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "stc.h"

namespace {

constexpr uint32_t kPow10[9] = {1u, 10u, 100u, 1000u, 10000u, 100000u, 1000000u, 10000000u,
                                 100000000u};

// Decimal digits at p as a uint32 with wrap-around (x = 10 x + d per digit,
// mod 2^32), 8 bytes at a time while 8 bytes remain.  In t = bytes - '0',
// digit bytes hold 0..9; the first byte that is not a digit has its high bit
// set in t | (t + 0x76) (a borrow or carry only moves towards later bytes,
// so the bytes before it are exact).  The k leading digits are shifted to
// the top and combined pairwise by three multiply-shift steps (the
// eight-digit method of simdjson's number parser), then x = x 10^k + value,
// which equals k steps of the per-digit rule mod 2^32.
inline const char* parse_uint(const char* p, const char* end, uint32_t& out) {
  uint32_t x = 0;
  while (end - p >= 8) {
    uint64_t w;
    memcpy(&w, p, 8);
    const uint64_t t = w - 0x3030303030303030ull;
    const uint64_t nd = (t | (t + 0x7676767676767676ull)) & 0x8080808080808080ull;
    const unsigned k = nd ? (unsigned)__builtin_ctzll(nd) >> 3 : 8u;
    if (k == 0) {
      out = x;
      return p;
    }
    uint64_t v = k == 8 ? t : t << (8 * (8 - k));
    v = ((v & 0x0F0F0F0F0F0F0F0Full) * 2561u) >> 8;
    v = ((v & 0x00FF00FF00FF00FFull) * 6553601u) >> 16;
    v = ((v & 0x0000FFFF0000FFFFull) * 42949672960001ull) >> 32;
    x = x * kPow10[k] + (uint32_t)v;
    p += k;
    if (k < 8) {
      out = x;
      return p;
    }
  }
  while (p < end && *p >= '0' && *p <= '9') x = x * 10u + (uint32_t)(*p++ - '0');
  out = x;
  return p;
}

inline const char* skip_blanks(const char* p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\t')) p++;
  return p;
}

inline const char* parse_sign(const char* p, const char* end, int8_t& out) {
  int8_t s = 1;
  if (p < end && *p == '-') {
    s = -1;
    p++;
  } else if (p < end && *p == '+') {
    p++;
  }
  while (p < end && *p >= '0' && *p <= '9') p++;
  out = s;
  return p;
}

uint64_t count_lines(const char* p, const char* end) {
  uint64_t lines = 0;
  while (p < end) {
    if (*p == '\n' || *p == '\r') {
      p++;
      continue;
    }
    if (*p == '#' || *p == '%') {
      const void* nl = memchr(p, '\n', (size_t)(end - p));
      p = nl ? (const char*)nl : end;
      continue;
    }
    lines++;
    const void* nl = memchr(p, '\n', (size_t)(end - p));
    p = nl ? (const char*)nl : end;
  }
  return lines;
}

struct Slice {
  uint64_t kept = 0;
  uint32_t max_id = 0;
};

Slice parse_range(const char* p, const char* end, uint32_t* src, uint32_t* dst, int8_t* sign) {
  Slice s;
  uint64_t w = 0;
  while (p < end) {
    if (*p == '\n' || *p == '\r') {
      p++;
      continue;
    }
    if (*p == '#' || *p == '%') {
      const void* nl = memchr(p, '\n', (size_t)(end - p));
      p = nl ? (const char*)nl : end;
      continue;
    }
    uint32_t u, v;
    int8_t sg;
    p = parse_uint(p, end, u);
    p = skip_blanks(p, end);
    p = parse_uint(p, end, v);
    p = skip_blanks(p, end);
    p = parse_sign(p, end, sg);
    while (p < end && *p != '\n') p++;
    if (u == v) continue;
    src[w] = u < v ? u : v;
    dst[w] = u < v ? v : u;
    sign[w] = sg;
    w++;
    s.max_id = std::max(s.max_id, std::max(u, v));
  }
  s.kept = w;
  return s;
}

stc_status parse_buffer(const char* data, uint64_t size, stc_edge_list* out) {
  memset(out, 0, sizeof(*out));
  auto alloc = [&](uint64_t cap) -> bool {
    uint64_t c = cap ? cap : 1;
    out->src = (uint32_t*)malloc(c * sizeof(uint32_t));
    out->dst = (uint32_t*)malloc(c * sizeof(uint32_t));
    out->sign = (int8_t*)malloc(c);
    if (!out->src || !out->dst || !out->sign) {
      stc_free_edge_list(out);
      return false;
    }
    return true;
  };
  if (size == 0) return alloc(0) ? STC_OK : STC_ERR_OUT_OF_MEMORY;
  const char* end = data + size;
  unsigned T = std::max(1u, std::thread::hardware_concurrency());
  if (size < (1u << 20)) T = 1;
  std::vector<const char*> starts(T + 1);
  for (unsigned t = 0; t <= T; t++) {
    const char* p = t == T ? end : data + (size / T) * t;
    if (t > 0 && t < T)
      while (p < end && *(p - 1) != '\n') p++;
    starts[t] = p;
  }
  std::vector<uint64_t> lines(T, 0);
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++)
      th.emplace_back([&, t] { lines[t] = count_lines(starts[t], starts[t + 1]); });
    for (auto& x : th) x.join();
  }
  std::vector<uint64_t> first(T + 1, 0);
  for (unsigned t = 0; t < T; t++) first[t + 1] = first[t] + lines[t];
  const uint64_t total = first[T];
  if (!alloc(total)) return STC_ERR_OUT_OF_MEMORY;
  std::vector<Slice> slices(T);
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++)
      th.emplace_back([&, t] {
        slices[t] = parse_range(starts[t], starts[t + 1], out->src + first[t], out->dst + first[t],
                                out->sign + first[t]);
      });
    for (auto& x : th) x.join();
  }
  uint64_t w = 0;
  uint32_t max_id = 0;
  for (unsigned t = 0; t < T; t++) {
    if (w != first[t] && slices[t].kept) {
      memmove(out->src + w, out->src + first[t], slices[t].kept * sizeof(uint32_t));
      memmove(out->dst + w, out->dst + first[t], slices[t].kept * sizeof(uint32_t));
      memmove(out->sign + w, out->sign + first[t], slices[t].kept);
    }
    w += slices[t].kept;
    max_id = std::max(max_id, slices[t].max_id);
  }
  out->n = max_id + 1u;
  out->lines = total;
  out->m = w;
  return STC_OK;
}

}  // namespace

extern "C" {

stc_status stc_parse_edge_text(const char* data, uint64_t size, stc_edge_list* out) {
  if (!out || (!data && size)) return STC_ERR_INVALID_ARGUMENT;
  try {
    return parse_buffer(data, size, out);
  } catch (...) {
    return STC_ERR_OUT_OF_MEMORY;
  }
}

stc_status stc_load_edge_list(const char* path, stc_edge_list* out) {
  if (!path || !out) return STC_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  int fd = open(path, O_RDONLY);
  if (fd < 0) return STC_ERR_IO;
  struct stat st;
  if (fstat(fd, &st) < 0) {
    close(fd);
    return STC_ERR_IO;
  }
  const uint64_t size = (uint64_t)st.st_size;
  if (size == 0) {
    close(fd);
    return stc_parse_edge_text(nullptr, 0, out);
  }
  void* data = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  if (data == MAP_FAILED) {
    close(fd);
    return STC_ERR_IO;
  }
  madvise(data, size, MADV_SEQUENTIAL);
  madvise(data, size, MADV_WILLNEED);
  stc_status s = stc_parse_edge_text((const char*)data, size, out);
  munmap(data, size);
  close(fd);
  return s;
}

void stc_free_edge_list(stc_edge_list* el) {
  if (!el) return;
  free(el->src);
  free(el->dst);
  free(el->sign);
  el->src = el->dst = nullptr;
  el->sign = nullptr;
  el->n = 0;
  el->m = el->lines = 0;
}

}  // extern "C"
