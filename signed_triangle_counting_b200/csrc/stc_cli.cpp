// stc — command-line drop-in for the reference programs
// (MC/tc_serial.cpp:172-210, MC/tc_merge_sign_enu.cpp:46-154,
// MC/tc_hash_sign_enu.cpp:76-177).
//
//   stc [--strategy auto|merge|hash|search|split|head] [--dispatch fixed|learned]
//       [--model PATH] [--zero-negative] [--host-ingest] [--device N] [--json]
//       <graph_file>
//
// <graph_file> is `u v sign` text (MC/graph_io.h:72-212), parsed on the GPU
// (--host-ingest: by the host threads instead), or, when it starts with a
// `%%MatrixMarket` banner, a coordinate .mtx file as the reference's GPU
// drivers read (--zero-negative: weight <= 0 is negative, their rule).
// --dispatch learned loads the model from --model or, by default,
// dispatch_model.json beside this executable.
//
// Prints the union of the reference outputs: tc_serial's stage lines,
// `n=.. raw_edges=..`, `forward_edges=..` and per-type block, then the
// Balanced / Unbalanced / Total lines of the merge and hash programs, then the
// total time.  Exit status 1 on a usage or I/O error, as in the reference.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "stc.h"

namespace {

struct Clock {
  std::chrono::high_resolution_clock::time_point t0 = std::chrono::high_resolution_clock::now();
  double sec() const {
    return std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  }
};

// Stage line in the reference format (MC/timer.h:24-26).
void stage(const char* label, double seconds) { std::printf("[%s] took %.4f seconds\n", label, seconds); }

int usage(const char* prog) {
  std::fprintf(stderr,
               "usage: %s [--strategy auto|merge|hash|search|split|head] [--dispatch fixed|learned] "
               "[--model PATH] [--zero-negative] [--host-ingest] [--device N] [--json] "
               "<graph_file>\n",
               prog);
  return 1;
}

bool is_mtx(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  char head[15] = {0};
  const size_t got = std::fread(head, 1, 14, f);
  std::fclose(f);
  return got == 14 && std::strncmp(head, "%%MatrixMarket", 14) == 0;
}

// The "params" array of a dispatch model file (STC_DISPATCH_MODEL_PARAMS
// floats) and its "support" cell list as a mask (all cells when absent);
// false if the file cannot be read or holds a different count.
bool read_model(const std::string& path, float* params, uint8_t* support) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::string text;
  char buf[4096];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, k);
  std::fclose(f);
  size_t at = text.find("\"params\"");
  if (at == std::string::npos) return false;
  at = text.find('[', at);
  if (at == std::string::npos) return false;
  const char* p = text.c_str() + at + 1;
  int n = 0;
  while (n < STC_DISPATCH_MODEL_PARAMS) {
    char* stop = nullptr;
    const float v = std::strtof(p, &stop);
    if (stop == p) break;
    params[n++] = v;
    p = stop;
    while (*p == ',' || *p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') p++;
  }
  if (n != STC_DISPATCH_MODEL_PARAMS || *p != ']') return false;
  size_t sat = text.find("\"support\"");
  if (sat == std::string::npos) {
    std::memset(support, 1, STC_DISPATCH_CELLS);
    return true;
  }
  sat = text.find('[', sat);
  if (sat == std::string::npos) return false;
  std::memset(support, 0, STC_DISPATCH_CELLS);
  const char* q = text.c_str() + sat + 1;
  while (true) {
    while (*q == ' ' || *q == ',' || *q == '\n' || *q == '\r' || *q == '\t') q++;
    if (*q == ']') return true;
    char* stop = nullptr;
    const long cell = std::strtol(q, &stop, 10);
    if (stop == q || cell < 0 || cell >= STC_DISPATCH_CELLS) return false;
    support[cell] = 1;
    q = stop;
  }
}

// A read-only mapping of a whole file.
struct MappedFile {
  const char* data = nullptr;
  uint64_t size = 0;
  bool open(const char* path) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) < 0) {
      ::close(fd);
      return false;
    }
    size = (uint64_t)st.st_size;
    if (size) {
      void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (p == MAP_FAILED) {
        ::close(fd);
        return false;
      }
      data = (const char*)p;
    }
    ::close(fd);
    return true;
  }
  ~MappedFile() {
    if (data) munmap((void*)data, size);
  }
};

std::string beside_executable(const char* argv0, const char* name) {
  std::string dir(argv0);
  const size_t slash = dir.rfind('/');
  dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
  return dir + "/" + name;
}

}  // namespace

int main(int argc, char** argv) {
  const char* path = nullptr;
  stc_opts opts{};
  opts.flags = STC_F_TIMING;
  int device = 0;
  bool json = false;
  bool zero_negative = false;
  bool host_ingest = false;
  std::string model_path;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--strategy" && i + 1 < argc) {
      std::string v = argv[++i];
      if (v == "auto") opts.strategy = STC_STRATEGY_AUTO;
      else if (v == "merge") opts.strategy = STC_STRATEGY_MERGE;
      else if (v == "hash") opts.strategy = STC_STRATEGY_HASH;
      else if (v == "search") opts.strategy = STC_STRATEGY_SEARCH;
      else if (v == "split") opts.strategy = STC_STRATEGY_SPLIT;
      else if (v == "head") opts.strategy = STC_STRATEGY_HEAD;
      else return usage(argv[0]);
    } else if (a == "--dispatch" && i + 1 < argc) {
      std::string v = argv[++i];
      if (v == "fixed") opts.dispatch = STC_DISPATCH_FIXED;
      else if (v == "learned") opts.dispatch = STC_DISPATCH_LEARNED;
      else return usage(argv[0]);
    } else if (a == "--model" && i + 1 < argc) {
      model_path = argv[++i];
    } else if (a == "--zero-negative") {
      zero_negative = true;
    } else if (a == "--host-ingest") {
      host_ingest = true;
    } else if (a == "--device" && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else if (a == "--json") {
      json = true;
    } else if (a == "-h" || a == "--help") {
      return usage(argv[0]);
    } else if (!path && (a.empty() || a[0] != '-')) {
      path = argv[i];
    } else {
      return usage(argv[0]);
    }
  }
  if (!path) return usage(argv[0]);

  Clock total;
  const bool mtx = is_mtx(path);
  const bool gpu_text = !mtx && !host_ingest;
  stc_edge_list el{};
  MappedFile text;
  Clock io;
  stc_status s = STC_OK;
  if (gpu_text) {
    s = text.open(path) ? STC_OK : STC_ERR_IO;
  } else {
    s = mtx ? stc_load_mtx(path, zero_negative ? STC_MTX_ZERO_NEGATIVE : 0u, &el)
            : stc_load_edge_list(path, &el);
  }
  if (s == STC_ERR_IO) {
    std::perror(path);
    return 1;
  }
  if (s != STC_OK) {
    std::fprintf(stderr, "%s: %s\n", path, stc_status_string(s));
    return 1;
  }
  const double io_s = io.sec();

  stc_ctx* ctx = nullptr;
  s = stc_ctx_create(device, &ctx);
  if (s != STC_OK) {
    std::fprintf(stderr, "stc: cannot open CUDA device %d: %s\n", device, stc_status_string(s));
    stc_free_edge_list(&el);
    return 1;
  }
  if (opts.dispatch == STC_DISPATCH_LEARNED) {
    float params[STC_DISPATCH_MODEL_PARAMS];
    uint8_t support[STC_DISPATCH_CELLS];
    const std::string mp = model_path.empty() ? beside_executable(argv[0], "dispatch_model.json")
                                              : model_path;
    if (!read_model(mp, params, support) ||
        stc_ctx_set_dispatch_model(ctx, params, support) != STC_OK) {
      std::fprintf(stderr, "stc: cannot load dispatch model %s\n", mp.c_str());
      stc_free_edge_list(&el);
      stc_ctx_destroy(ctx);
      return 1;
    }
  }
  stc_counts c{};
  stc_text_info info{};
  Clock run;
  if (gpu_text) {
    s = stc_count_text(ctx, text.data, text.size, &opts, &c, &info);
  } else {
    info.lines = el.lines;
    info.n = el.n;
    s = stc_count(ctx, el.src, el.dst, el.sign, el.m, &opts, &c);
  }
  const double run_s = run.sec();
  stc_free_edge_list(&el);
  if (s != STC_OK) {
    std::fprintf(stderr, "stc: %s: %s\n", stc_status_string(s), stc_ctx_last_error(ctx));
    stc_ctx_destroy(ctx);
    return 1;
  }
  stc_stats st{};
  stc_ctx_last_stats(ctx, &st);
  stc_ctx_destroy(ctx);

  // With GPU ingest the parse runs on the device inside the H2D stage.
  stage("Graph Load (I/O + parse)", io_s + (gpu_text ? st.ms_h2d / 1e3 : 0.0));
  std::printf("  n=%u  raw_edges=%llu\n", info.n, (unsigned long long)info.lines);
  stage("Build Forward CSR", ((gpu_text ? 0.0 : st.ms_h2d) + st.ms_dedup + st.ms_orient) / 1e3);
  stage("Algorithm-Specific Preprocessing (Adjacency List Sort)", st.ms_csr / 1e3);
  std::printf("  forward_edges=%llu\n", (unsigned long long)st.m_forward);
  stage("Triangle Counting Execution", st.ms_count / 1e3);

  std::printf("\nTriangle counts\n");
  std::printf("  T3 (+++ balanced)   : %llu\n", (unsigned long long)c.t3);
  std::printf("  T1 (+-- balanced)   : %llu\n", (unsigned long long)c.t1);
  std::printf("  T2 (++- unbalanced) : %llu\n", (unsigned long long)c.t2);
  std::printf("  T0 (--- unbalanced) : %llu\n", (unsigned long long)c.t0);
  std::printf("  --------------------------------\n");
  std::printf("  balanced total      : %llu\n", (unsigned long long)stc_balanced(&c));
  std::printf("  unbalanced total    : %llu\n", (unsigned long long)stc_unbalanced(&c));
  std::printf("  grand total         : %llu\n", (unsigned long long)stc_total(&c));
  std::printf("Balanced   = %llu\n", (unsigned long long)stc_balanced(&c));
  std::printf("Unbalanced = %llu\n", (unsigned long long)stc_unbalanced(&c));
  std::printf("Total      = %llu\n", (unsigned long long)stc_total(&c));
  stage("Total execution time", total.sec());
  if (json) {
    const double count_s = st.ms_count / 1e3;
    std::printf(
        "{\"n\": %llu, \"m_unique\": %llu, \"forward_edges\": %llu, \"t0\": %llu, \"t1\": %llu, "
        "\"t2\": %llu, \"t3\": %llu, \"balanced\": %llu, \"unbalanced\": %llu, "
        "\"ms_dedup\": %.4f, \"ms_orient\": %.4f, \"ms_csr\": %.4f, \"ms_count\": %.4f, "
        "\"ms_device_total\": %.4f, \"wall_s\": %.4f, \"alg_bytes\": %llu, "
        "\"edges_per_s_count\": %.6g}\n",
        (unsigned long long)st.n, (unsigned long long)st.m_unique, (unsigned long long)st.m_forward,
        (unsigned long long)c.t0, (unsigned long long)c.t1, (unsigned long long)c.t2,
        (unsigned long long)c.t3, (unsigned long long)stc_balanced(&c),
        (unsigned long long)stc_unbalanced(&c), st.ms_dedup, st.ms_orient, st.ms_csr, st.ms_count,
        st.ms_total, run_s, (unsigned long long)st.alg_bytes,
        count_s > 0 ? st.m_unique / count_s : 0.0);
  }
  return 0;
}
