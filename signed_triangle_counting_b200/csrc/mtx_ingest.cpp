// Host MatrixMarket ingest: a coordinate `.mtx` file -> stc_edge_list.
//
// The reference's GPU drivers read their graphs with Gunrock's MatrixMarket
// loader (GM/tc_split/signed_tc.cu:21-33; Gunrock itself is not vendored)
// and take an edge weight w > 0 as positive and anything else as negative
// (GM/signed_tc.hxx:317, 362).  This parser follows the published
// MatrixMarket coordinate format:
//   %%MatrixMarket matrix coordinate <real|double|integer|pattern> <general|symmetric>
//   % comment lines
//   M N nnz
//   i j [w]            (nnz entries, 1-based indices)
// Vertex i - 1 and j - 1 get an undirected edge; a diagonal entry is dropped
// (as the text loader drops self-loops); a `symmetric` entry stands for both
// directions, and in a `general` file the (i, j) and (j, i) entries fold
// into one edge when the graph is built (the first occurrence's sign wins).
// Weights are read as float, as the GPU drivers store them.  The sign rule
// is w < 0 -> negative by default (the CPU programs' rule for `u v sign`
// text), or w <= 0 -> negative with STC_MTX_ZERO_NEGATIVE (the GPU
// drivers' rule); `pattern` entries are positive.  Entry lines are parsed by
// all host threads over line-aligned byte ranges.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "stc.h"

namespace {

struct Header {
  bool pattern = false;
  bool symmetric = false;
  uint64_t rows = 0, cols = 0, nnz = 0;
  const char* entries = nullptr;  // first byte after the size line
};

std::string lower(std::string s) {
  for (char& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

const char* line_end(const char* p, const char* end) {
  const void* nl = memchr(p, '\n', (size_t)(end - p));
  return nl ? (const char*)nl : end;
}

// Parses the banner and the size line; false if the file is not a
// supported MatrixMarket coordinate matrix.
bool parse_header(const char* data, const char* end, Header& h) {
  const char* p = data;
  const char* e = line_end(p, end);
  std::string banner(p, e);
  std::vector<std::string> tok;
  {
    size_t i = 0;
    while (i < banner.size()) {
      while (i < banner.size() && std::isspace((unsigned char)banner[i])) i++;
      size_t j = i;
      while (j < banner.size() && !std::isspace((unsigned char)banner[j])) j++;
      if (j > i) tok.push_back(lower(banner.substr(i, j - i)));
      i = j;
    }
  }
  if (tok.size() < 5 || tok[0] != "%%matrixmarket" || tok[1] != "matrix" || tok[2] != "coordinate")
    return false;
  if (tok[3] == "pattern") h.pattern = true;
  else if (tok[3] != "real" && tok[3] != "double" && tok[3] != "integer") return false;
  if (tok[4] == "symmetric") h.symmetric = true;
  else if (tok[4] != "general") return false;
  p = e < end ? e + 1 : end;
  // Comment and blank lines, then the size line.
  while (p < end) {
    e = line_end(p, end);
    const char* q = p;
    while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) q++;
    if (q == e || *q == '%') {
      p = e < end ? e + 1 : end;
      continue;
    }
    std::string line(q, e);
    unsigned long long r = 0, c = 0, z = 0;
    char extra = 0;
    if (sscanf(line.c_str(), "%llu %llu %llu %c", &r, &c, &z, &extra) != 3) return false;
    h.rows = r;
    h.cols = c;
    h.nnz = z;
    h.entries = e < end ? e + 1 : end;
    return true;
  }
  return false;
}

inline const char* skip_blanks(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t')) p++;
  return p;
}

inline const char* parse_index(const char* p, const char* e, uint64_t& out, bool& ok) {
  uint64_t x = 0;
  const char* s = p;
  while (p < e && *p >= '0' && *p <= '9' && x < (1ull << 40)) x = x * 10 + (uint64_t)(*p++ - '0');
  ok = p > s && !(p < e && *p >= '0' && *p <= '9');
  out = x;
  return p;
}

struct Slice {
  uint64_t entries = 0;
  uint64_t kept = 0;
  bool bad = false;
};

bool is_entry_line(const char* p, const char* e) {
  p = skip_blanks(p, e);
  return p < e && *p != '%' && *p != '\r';
}

uint64_t count_entries(const char* p, const char* end) {
  uint64_t n = 0;
  while (p < end) {
    const char* e = line_end(p, end);
    if (is_entry_line(p, e)) n++;
    p = e < end ? e + 1 : end;
  }
  return n;
}

Slice parse_entries(const char* p, const char* end, const Header& h, bool zero_negative,
                    uint32_t* src, uint32_t* dst, int8_t* sign) {
  Slice s;
  const uint64_t dim = std::max(h.rows, h.cols);
  std::string tok;
  while (p < end) {
    const char* e = line_end(p, end);
    if (!is_entry_line(p, e)) {
      p = e < end ? e + 1 : end;
      continue;
    }
    s.entries++;
    uint64_t i = 0, j = 0;
    bool ok1 = false, ok2 = false;
    const char* q = skip_blanks(p, e);
    q = parse_index(q, e, i, ok1);
    q = skip_blanks(q, e);
    q = parse_index(q, e, j, ok2);
    if (!ok1 || !ok2 || i == 0 || j == 0 || i > h.rows || j > h.cols || dim > 0x7FFFFFFEull) {
      s.bad = true;
      return s;
    }
    int8_t sg = 1;
    if (!h.pattern) {
      q = skip_blanks(q, e);
      const char* t = q;
      while (t < e && *t != ' ' && *t != '\t' && *t != '\r') t++;
      if (t == q) {
        s.bad = true;
        return s;
      }
      tok.assign(q, t);
      char* stop = nullptr;
      const float w = strtof(tok.c_str(), &stop);
      if (stop == tok.c_str()) {
        s.bad = true;
        return s;
      }
      sg = zero_negative ? (w > 0.0f ? 1 : -1) : (w < 0.0f ? -1 : 1);
    }
    p = e < end ? e + 1 : end;
    if (i == j) continue;
    const uint32_t u = (uint32_t)(i - 1), v = (uint32_t)(j - 1);
    src[s.kept] = u < v ? u : v;
    dst[s.kept] = u < v ? v : u;
    sign[s.kept] = sg;
    s.kept++;
  }
  return s;
}

stc_status parse_mtx(const char* data, uint64_t size, uint32_t flags, stc_edge_list* out) {
  memset(out, 0, sizeof(*out));
  const char* end = data + size;
  Header h;
  if (!size || !parse_header(data, end, h)) return STC_ERR_INVALID_ARGUMENT;
  const uint64_t dim = std::max(h.rows, h.cols);
  if (dim > 0x7FFFFFFEull) return STC_ERR_LIMIT;
  const char* body = h.entries;
  const uint64_t bsize = (uint64_t)(end - body);
  unsigned T = std::max(1u, std::thread::hardware_concurrency());
  if (bsize < (1u << 20)) T = 1;
  std::vector<const char*> starts(T + 1);
  for (unsigned t = 0; t <= T; t++) {
    const char* p = t == T ? end : body + (bsize / T) * t;
    if (t > 0 && t < T)
      while (p < end && *(p - 1) != '\n') p++;
    starts[t] = p;
  }
  std::vector<uint64_t> counts(T, 0);
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++)
      th.emplace_back([&, t] { counts[t] = count_entries(starts[t], starts[t + 1]); });
    for (auto& x : th) x.join();
  }
  std::vector<uint64_t> first(T + 1, 0);
  for (unsigned t = 0; t < T; t++) first[t + 1] = first[t] + counts[t];
  const uint64_t total = first[T];
  if (total != h.nnz) return STC_ERR_INVALID_ARGUMENT;  // truncated or padded file
  if (total >= (1ull << 32)) return STC_ERR_LIMIT;
  const uint64_t cap = total ? total : 1;
  out->src = (uint32_t*)malloc(cap * sizeof(uint32_t));
  out->dst = (uint32_t*)malloc(cap * sizeof(uint32_t));
  out->sign = (int8_t*)malloc(cap);
  if (!out->src || !out->dst || !out->sign) {
    stc_free_edge_list(out);
    return STC_ERR_OUT_OF_MEMORY;
  }
  std::vector<Slice> slices(T);
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++)
      th.emplace_back([&, t] {
        slices[t] = parse_entries(starts[t], starts[t + 1], h, (flags & STC_MTX_ZERO_NEGATIVE) != 0,
                                  out->src + first[t], out->dst + first[t], out->sign + first[t]);
      });
    for (auto& x : th) x.join();
  }
  uint64_t w = 0;
  for (unsigned t = 0; t < T; t++) {
    if (slices[t].bad) {
      stc_free_edge_list(out);
      return STC_ERR_INVALID_ARGUMENT;
    }
    if (w != first[t] && slices[t].kept) {
      memmove(out->src + w, out->src + first[t], slices[t].kept * sizeof(uint32_t));
      memmove(out->dst + w, out->dst + first[t], slices[t].kept * sizeof(uint32_t));
      memmove(out->sign + w, out->sign + first[t], slices[t].kept);
    }
    w += slices[t].kept;
  }
  out->n = (uint32_t)dim;
  out->lines = total;
  out->m = w;
  return STC_OK;
}

}  // namespace

extern "C" {

stc_status stc_parse_mtx(const char* data, uint64_t size, uint32_t flags, stc_edge_list* out) {
  if (!out || (!data && size) || (flags & ~STC_MTX_ZERO_NEGATIVE)) return STC_ERR_INVALID_ARGUMENT;
  try {
    return parse_mtx(data, size, flags, out);
  } catch (...) {
    return STC_ERR_OUT_OF_MEMORY;
  }
}

stc_status stc_load_mtx(const char* path, uint32_t flags, stc_edge_list* out) {
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
    return STC_ERR_INVALID_ARGUMENT;
  }
  void* data = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  if (data == MAP_FAILED) {
    close(fd);
    return STC_ERR_IO;
  }
  madvise(data, size, MADV_SEQUENTIAL);
  const stc_status s = stc_parse_mtx((const char*)data, size, flags, out);
  munmap(data, size);
  close(fd);
  return s;
}

}  // extern "C"
