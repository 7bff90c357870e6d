// Host implementations of the seeded synthetic signed graphs (include/stc_synth.h).
//
// The per-edge arithmetic lives in stc_gen.h and is shared with the device
// generator; this file adds what only the host does: distinct-pair ER
// sampling, the Delaunay triangulation, hub degree draws and batch recipes.
#include "stc_synth.h"
#include "stc_gen.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

using namespace stcgen;

namespace {

std::atomic<uint32_t> g_threads{0};

uint32_t host_threads() {
  uint32_t t = g_threads.load();
  if (t == 0) t = std::max(1u, std::thread::hardware_concurrency());
  return t;
}

template <class F>
void parallel_for(uint64_t count, F fn) {
  uint32_t T = host_threads();
  if (count < (1u << 16) || T == 1) {
    fn(0, count);
    return;
  }
  std::vector<std::thread> th;
  uint64_t chunk = (count + T - 1) / T;
  for (uint32_t t = 0; t < T; t++) {
    uint64_t b = t * chunk, e = std::min(count, b + chunk);
    if (b >= e) break;
    th.emplace_back([=] { fn(b, e); });
  }
  for (auto& x : th) x.join();
}

uint64_t prob_threshold(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return UINT64_MAX;
  return (uint64_t)std::ldexp(p, 64);
}

uint32_t prob_threshold32(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return UINT32_MAX;
  return (uint32_t)std::ldexp(p, 32);
}

double unit_double(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }

bool alloc_graph(stc_synth_graph* g, uint64_t n, uint64_t m) {
  g->n = n;
  g->m = m;
  size_t mm = m ? m : 1;
  g->src = (uint32_t*)std::malloc(mm * sizeof(uint32_t));
  g->dst = (uint32_t*)std::malloc(mm * sizeof(uint32_t));
  g->sign = (int8_t*)std::malloc(mm);
  if (!g->src || !g->dst || !g->sign) {
    std::free(g->src);
    std::free(g->dst);
    std::free(g->sign);
    g->src = g->dst = nullptr;
    g->sign = nullptr;
    return false;
  }
  return true;
}

// Relabels every endpoint through the seeded bijection and assigns signs from
// the final unordered pair.
void relabel_and_sign(stc_synth_graph* g, uint64_t seed, double p_pos) {
  Perm perm = make_perm(seed, g->n);
  uint64_t thr = prob_threshold(p_pos);
  parallel_for(g->m, [&](uint64_t b, uint64_t e) {
    for (uint64_t i = b; i < e; i++) {
      uint32_t u = (uint32_t)perm_apply(perm, g->src[i]);
      uint32_t v = (uint32_t)perm_apply(perm, g->dst[i]);
      g->src[i] = u;
      g->dst[i] = v;
      g->sign[i] = edge_sign(seed, u, v, thr);
    }
  });
}

// Open-addressing set of nonzero 64-bit keys.
struct KeySet {
  std::vector<uint64_t> slots;
  uint64_t mask;
  explicit KeySet(uint64_t expected) {
    uint64_t cap = 16;
    while (cap < expected * 2) cap <<= 1;
    slots.assign(cap, 0);
    mask = cap - 1;
  }
  bool insert(uint64_t key) {  // key != 0
    uint64_t pos = mix64(key) & mask;
    while (true) {
      uint64_t s = slots[pos];
      if (s == key) return false;
      if (s == 0) {
        slots[pos] = key;
        return true;
      }
      pos = (pos + 1) & mask;
    }
  }
};

// ------------------------------------------------------------ Delaunay ----
// Incremental Bowyer-Watson triangulation over integer coordinates in
// [0, 2^28) with exact orientation / in-circle predicates and "ghost"
// triangles through a vertex at infinity (so the hull needs no super
// triangle).  Points are inserted in Hilbert-curve order and located by a
// visibility walk from the most recently created triangle.
constexpr int kCoordBits = 28;
constexpr int32_t kInf = -1;

struct Pt {
  int64_t x, y;
};

inline int64_t orient(const Pt& a, const Pt& b, const Pt& c) {
  return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
}

// > 0 when d lies strictly inside the circumcircle of the CCW triangle abc.
inline int incircle(const Pt& a, const Pt& b, const Pt& c, const Pt& d) {
  int64_t adx = a.x - d.x, ady = a.y - d.y;
  int64_t bdx = b.x - d.x, bdy = b.y - d.y;
  int64_t cdx = c.x - d.x, cdy = c.y - d.y;
  __int128 al = (__int128)(adx * adx + ady * ady);
  __int128 bl = (__int128)(bdx * bdx + bdy * bdy);
  __int128 cl = (__int128)(cdx * cdx + cdy * cdy);
  __int128 det = al * (__int128)(bdx * cdy - cdx * bdy) +
                 bl * (__int128)(cdx * ady - adx * cdy) +
                 cl * (__int128)(adx * bdy - bdx * ady);
  return (det > 0) - (det < 0);
}

uint64_t hilbert_d(uint32_t order_bits, uint32_t x, uint32_t y) {
  uint64_t d = 0;
  for (uint32_t s = 1u << (order_bits - 1); s > 0; s >>= 1) {
    uint32_t rx = (x & s) > 0, ry = (y & s) > 0;
    d += (uint64_t)s * s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      std::swap(x, y);
    }
  }
  return d;
}

struct Tri {
  int32_t v[3];
  int32_t nb[3];  // nb[i]: triangle across the edge opposite v[i]
};

class Delaunay {
 public:
  explicit Delaunay(const std::vector<Pt>& pts) : P(pts) {}

  // Triangulates the points with indices in `order` (distinct points).
  bool run(std::vector<uint32_t>& order) {
    if (order.size() < 3) return false;
    // First three points must not be collinear.
    size_t k = 2;
    while (k < order.size() && orient(P[order[0]], P[order[1]], P[order[k]]) == 0) k++;
    if (k == order.size()) return false;
    std::swap(order[2], order[k]);
    int32_t a = (int32_t)order[0], b = (int32_t)order[1], c = (int32_t)order[2];
    if (orient(P[a], P[b], P[c]) < 0) std::swap(b, c);
    T.reserve(order.size() * 2 + 16);
    int32_t t0 = new_tri(a, b, c);
    int32_t g0 = new_tri(b, a, kInf), g1 = new_tri(c, b, kInf), g2 = new_tri(a, c, kInf);
    int32_t ids[4] = {t0, g0, g1, g2};
    for (int i = 0; i < 4; i++)
      for (int e = 0; e < 3; e++) {
        int32_t x = T[ids[i]].v[(e + 1) % 3], y = T[ids[i]].v[(e + 2) % 3];
        for (int j = 0; j < 4; j++) {
          if (j == i) continue;
          for (int f = 0; f < 3; f++) {
            int32_t x2 = T[ids[j]].v[(f + 1) % 3], y2 = T[ids[j]].v[(f + 2) % 3];
            if (x == y2 && y == x2) T[ids[i]].nb[e] = ids[j];
          }
        }
      }
    last = t0;
    for (size_t i = 3; i < order.size(); i++) insert((int32_t)order[i]);
    return true;
  }

  template <class F>
  void for_each_edge(F emit) const {
    for (size_t t = 0; t < T.size(); t++) {
      if (dead[t]) continue;
      const Tri& tr = T[t];
      if (tr.v[0] == kInf || tr.v[1] == kInf || tr.v[2] == kInf) continue;
      for (int e = 0; e < 3; e++) {
        int32_t o = tr.nb[e];
        bool ghost = T[o].v[0] == kInf || T[o].v[1] == kInf || T[o].v[2] == kInf;
        if (ghost || (size_t)o > t) emit(tr.v[(e + 1) % 3], tr.v[(e + 2) % 3]);
      }
    }
  }

 private:
  const std::vector<Pt>& P;
  std::vector<Tri> T;
  std::vector<uint8_t> dead;
  std::vector<uint32_t> stamp;
  std::vector<int32_t> free_list;
  uint32_t cur_stamp = 0;
  int32_t last = 0;
  uint64_t walk_rng = 0x243F6A8885A308D3ull;

  int32_t new_tri(int32_t a, int32_t b, int32_t c) {
    int32_t id;
    if (!free_list.empty()) {
      id = free_list.back();
      free_list.pop_back();
      dead[id] = 0;
    } else {
      id = (int32_t)T.size();
      T.push_back(Tri{});
      dead.push_back(0);
      stamp.push_back(0);
    }
    T[id].v[0] = a;
    T[id].v[1] = b;
    T[id].v[2] = c;
    T[id].nb[0] = T[id].nb[1] = T[id].nb[2] = -1;
    return id;
  }

  int inf_index(const Tri& t) const {
    for (int i = 0; i < 3; i++)
      if (t.v[i] == kInf) return i;
    return -1;
  }

  bool in_circle(int32_t t, const Pt& p) const {
    const Tri& tr = T[t];
    int k = inf_index(tr);
    if (k < 0) return incircle(P[tr.v[0]], P[tr.v[1]], P[tr.v[2]], p) > 0;
    const Pt& x = P[tr.v[(k + 1) % 3]];
    const Pt& y = P[tr.v[(k + 2) % 3]];
    int64_t o = orient(x, y, p);
    if (o > 0) return true;
    if (o < 0) return false;
    // Collinear with the hull edge: inside only on the open segment.
    int64_t dot = (p.x - x.x) * (y.x - x.x) + (p.y - x.y) * (y.y - x.y);
    int64_t len = (y.x - x.x) * (y.x - x.x) + (y.y - x.y) * (y.y - x.y);
    return dot > 0 && dot < len;
  }

  int32_t locate(const Pt& p) {
    int32_t t = last;
    if (dead[t]) t = 0;
    while (dead[t]) t++;
    int k = inf_index(T[t]);
    if (k >= 0) t = T[t].nb[k];
    const size_t limit = 64 + 8 * (size_t)std::sqrt((double)T.size());
    for (size_t step = 0; step < limit; step++) {
      const Tri& tr = T[t];
      if (inf_index(tr) >= 0) return t;
      walk_rng = mix64(walk_rng);
      int r = (int)(walk_rng % 3);
      bool moved = false;
      for (int e = 0; e < 3; e++) {
        int i = (r + e) % 3;
        if (orient(P[tr.v[(i + 1) % 3]], P[tr.v[(i + 2) % 3]], p) < 0) {
          t = tr.nb[i];
          moved = true;
          break;
        }
      }
      if (!moved) return t;
    }
    for (size_t s = 0; s < T.size(); s++)  // walk did not converge: exhaustive search
      if (!dead[s] && in_circle((int32_t)s, p)) return (int32_t)s;
    return t;
  }

  struct Bnd {
    int32_t a, b, outer, outer_slot;
  };
  std::vector<int32_t> cavity, stack;
  std::vector<Bnd> bnd;

  void insert(int32_t pi) {
    const Pt& p = P[pi];
    int32_t t0 = locate(p);
    cur_stamp += 2;  // stamp == cur: in cavity; stamp == cur + 1: tested, outside
    cavity.clear();
    stack.clear();
    bnd.clear();
    stamp[t0] = cur_stamp;
    stack.push_back(t0);
    while (!stack.empty()) {
      int32_t t = stack.back();
      stack.pop_back();
      cavity.push_back(t);
      for (int e = 0; e < 3; e++) {
        int32_t o = T[t].nb[e];
        if (stamp[o] == cur_stamp) continue;
        if (stamp[o] != cur_stamp + 1) {
          if (in_circle(o, p)) {
            stamp[o] = cur_stamp;
            stack.push_back(o);
            continue;
          }
          stamp[o] = cur_stamp + 1;
        }
        int32_t a = T[t].v[(e + 1) % 3], b = T[t].v[(e + 2) % 3];
        int slot = 0;
        for (int f = 0; f < 3; f++)
          if (T[o].nb[f] == t) slot = f;
        bnd.push_back(Bnd{a, b, o, slot});
      }
    }
    for (int32_t t : cavity) {
      dead[t] = 1;
      free_list.push_back(t);
    }
    const size_t K = bnd.size();
    std::vector<int32_t>& made = stack;
    made.assign(K, -1);
    for (size_t i = 0; i < K; i++) {
      int32_t id = new_tri(bnd[i].a, bnd[i].b, pi);
      made[i] = id;
      T[id].nb[2] = bnd[i].outer;
      T[bnd[i].outer].nb[bnd[i].outer_slot] = id;
    }
    // Around p: triangle (a, b, p) borders (b, c, p) across edge b-p and
    // (z, a, p) across edge p-a.
    for (size_t i = 0; i < K; i++) {
      for (size_t j = 0; j < K; j++) {
        if (bnd[j].a == bnd[i].b) T[made[i]].nb[0] = made[j];
        if (bnd[j].b == bnd[i].a) T[made[i]].nb[1] = made[j];
      }
    }
    last = made[0];
    for (size_t i = 0; i < K; i++)
      if (inf_index(T[made[i]]) < 0) {
        last = made[i];
        break;
      }
  }
};

int make_delaunay(uint64_t seed, uint64_t n, double delete_frac, double p_pos,
                  stc_synth_graph* out) {
  std::vector<Pt> pts(n);
  for (uint64_t i = 0; i < n; i++) {
    pts[i].x = (int64_t)(draw(seed, kStreamDelaunay, 2 * i) >> (64 - kCoordBits));
    pts[i].y = (int64_t)(draw(seed, kStreamDelaunay, 2 * i + 1) >> (64 - kCoordBits));
  }
  // Duplicate coordinates (probability ~n^2 / 2^57) keep their first index
  // only; later copies stay isolated vertices.
  std::vector<uint64_t> key(n);
  std::vector<uint32_t> order(n);
  const uint32_t hb = 16;
  for (uint64_t i = 0; i < n; i++) {
    key[i] = hilbert_d(hb, (uint32_t)(pts[i].x >> (kCoordBits - hb)),
                       (uint32_t)(pts[i].y >> (kCoordBits - hb)));
    order[i] = (uint32_t)i;
  }
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (key[a] != key[b]) return key[a] < key[b];
    if (pts[a].x != pts[b].x) return pts[a].x < pts[b].x;
    if (pts[a].y != pts[b].y) return pts[a].y < pts[b].y;
    return a < b;
  });
  {
    std::vector<uint32_t> uniq;
    uniq.reserve(n);
    for (uint64_t i = 0; i < n; i++) {
      if (!uniq.empty()) {
        const Pt& q = pts[uniq.back()];
        if (q.x == pts[order[i]].x && q.y == pts[order[i]].y) continue;
      }
      uniq.push_back(order[i]);
    }
    order.swap(uniq);
  }
  std::vector<uint32_t> eu, ev;
  if (n >= 3) {
    Delaunay dt(pts);
    if (dt.run(order)) {
      eu.reserve(3 * n);
      ev.reserve(3 * n);
      uint64_t del_thr = prob_threshold(delete_frac);
      dt.for_each_edge([&](int32_t a, int32_t b) {
        uint64_t lo = (uint64_t)std::min(a, b), hi = (uint64_t)std::max(a, b);
        if (draw(seed, kStreamDelete, (lo << 32) | hi) < del_thr) return;
        eu.push_back((uint32_t)a);
        ev.push_back((uint32_t)b);
      });
    }
  }
  if (!alloc_graph(out, n, eu.size())) return 4;
  std::memcpy(out->src, eu.data(), eu.size() * sizeof(uint32_t));
  std::memcpy(out->dst, ev.data(), ev.size() * sizeof(uint32_t));
  relabel_and_sign(out, seed, p_pos);
  return 0;
}

}  // namespace

extern "C" {

void stc_synth_set_threads(uint32_t threads) { g_threads.store(threads); }

void stc_synth_free(stc_synth_graph* g) {
  if (!g) return;
  std::free(g->src);
  std::free(g->dst);
  std::free(g->sign);
  g->src = g->dst = nullptr;
  g->sign = nullptr;
  g->n = g->m = 0;
}

int stc_synth_er(uint64_t seed, uint64_t n, uint64_t m, double p_pos, stc_synth_graph* out) {
  if (!out || n < 2 || n > (1ull << 31) || m > n * (n - 1) / 2) return 1;
  if (!alloc_graph(out, n, m)) return 4;
  KeySet set(m);
  uint64_t got = 0;
  for (uint64_t i = 0; got < m; i++) {
    uint32_t a, b;
    uniform_pair(seed, kStreamER, i, n, &a, &b);
    uint64_t lo = std::min(a, b), hi = std::max(a, b);
    if (!set.insert(((lo << 32) | hi) + 1)) continue;
    out->src[got] = a;
    out->dst[got] = b;
    got++;
  }
  relabel_and_sign(out, seed, p_pos);
  return 0;
}

int stc_synth_rmat(uint64_t seed, uint32_t scale, uint64_t n, uint64_t samples, double a,
                   double b, double c, double p_pos, stc_synth_graph* out) {
  if (!out || scale == 0 || scale > 31 || n < 2 || n > (1ull << scale)) return 1;
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return 1;
  if (!alloc_graph(out, n, samples)) return 4;
  RmatParams rp;
  rp.scale = scale;
  rp.n = n;
  rp.t_a = prob_threshold32(a);
  rp.t_ab = prob_threshold32(a + b);
  rp.t_abc = prob_threshold32(a + b + c);
  parallel_for(samples, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) rmat_sample(seed, i, rp, &out->src[i], &out->dst[i]);
  });
  relabel_and_sign(out, seed, p_pos);
  return 0;
}

int stc_synth_delaunay(uint64_t seed, uint64_t n, double delete_frac, double p_pos,
                       stc_synth_graph* out) {
  if (!out || n < 3 || n > (1ull << 31)) return 1;
  return make_delaunay(seed, n, delete_frac, p_pos, out);
}

int stc_synth_skew(uint64_t seed, uint64_t n, uint64_t m_total, uint32_t hubs,
                   uint64_t hub_deg_min, uint64_t hub_deg_max, double p_pos,
                   stc_synth_graph* out) {
  if (!out || n < 2 || n > (1ull << 31) || hubs >= n || hub_deg_min == 0 ||
      hub_deg_max < hub_deg_min)
    return 1;
  std::vector<uint64_t> hub_off(hubs + 1, 0);
  double lmin = std::log((double)hub_deg_min), lmax = std::log((double)hub_deg_max);
  for (uint32_t h = 0; h < hubs; h++) {
    double u = unit_double(draw(seed, kStreamHub, h));
    uint64_t d = (uint64_t)std::floor(std::exp(lmin + u * (lmax - lmin)));
    d = std::min(std::max(d, hub_deg_min), hub_deg_max);
    hub_off[h + 1] = hub_off[h] + d;
  }
  uint64_t hub_edges = hub_off[hubs];
  uint64_t backbone = m_total > hub_edges ? m_total - hub_edges : 0;
  if (!alloc_graph(out, n, hub_edges + backbone)) return 4;
  for (uint32_t h = 0; h < hubs; h++) {
    uint64_t base = hub_off[h], d = hub_off[h + 1] - hub_off[h];
    parallel_for(d, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t j = lo; j < hi; j++) hub_edge(seed, h, j, n, &out->src[base + j], &out->dst[base + j]);
    });
  }
  parallel_for(backbone, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t k = lo; k < hi; k++)
      uniform_pair(seed, kStreamBackbone, k, n, &out->src[hub_edges + k], &out->dst[hub_edges + k]);
  });
  relabel_and_sign(out, seed, p_pos);
  return 0;
}

int stc_synth_batch_specs(uint64_t seed, uint32_t G, stc_batch_spec* specs) {
  if (!specs) return 1;
  for (uint32_t g = 0; g < G; g++) {
    stc_batch_spec s;
    s.seed = draw(seed, kStreamBatch, 8ull * g);
    double u = unit_double(draw(seed, kStreamBatch, 8ull * g + 1));
    s.n = (uint64_t)std::floor(1e3 * std::pow(1e3, u));
    if (s.n < 1000) s.n = 1000;
    if (s.n > 1000000) s.n = 1000000;
    s.kind = (uint32_t)uniform(draw(seed, kStreamBatch, 8ull * g + 2), 3);
    s.p_pos = 0.3 + 0.6 * unit_double(draw(seed, kStreamBatch, 8ull * g + 3));
    s.rmat_scale = 0;
    s.m_target = 0;
    if (s.kind == STC_SYNTH_ER) {
      s.m_target = 4 * s.n;
    } else if (s.kind == STC_SYNTH_RMAT) {
      uint32_t sc = 0;
      while ((1ull << sc) < s.n) sc++;
      s.rmat_scale = sc;
      s.m_target = 8 * s.n;
    }
    specs[g] = s;
  }
  return 0;
}

int stc_synth_batch_graph(const stc_batch_spec* s, stc_synth_graph* out) {
  if (!s) return 1;
  switch (s->kind) {
    case STC_SYNTH_ER:
      return stc_synth_er(s->seed, s->n, s->m_target, s->p_pos, out);
    case STC_SYNTH_RMAT:
      return stc_synth_rmat(s->seed, s->rmat_scale, s->n, s->m_target, 0.57, 0.19, 0.19,
                            s->p_pos, out);
    case STC_SYNTH_DELAUNAY:
      return stc_synth_delaunay(s->seed, s->n, 0.2, s->p_pos, out);
    default:
      return 1;
  }
}

int stc_synth_batch_packed(const stc_batch_spec* specs, uint32_t g_begin, uint32_t g_end,
                           stc_synth_graph* out, uint64_t* offsets) {
  if (!specs || !out || !offsets || g_end < g_begin) return 1;
  const uint32_t cnt = g_end - g_begin;
  std::vector<stc_synth_graph> parts(cnt);
  std::vector<int> rc(cnt, 0);
  // Graphs in parallel, each generated single-threaded.
  const uint32_t saved = g_threads.load();
  g_threads.store(1);
  {
    std::atomic<uint32_t> next{0};
    const uint32_t T = std::max(1u, saved ? saved : std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < std::min(T, std::max(1u, cnt)); t++)
      th.emplace_back([&] {
        for (uint32_t i = next++; i < cnt; i = next++) {
          memset(&parts[i], 0, sizeof(parts[i]));
          rc[i] = stc_synth_batch_graph(&specs[g_begin + i], &parts[i]);
        }
      });
    for (auto& x : th) x.join();
  }
  g_threads.store(saved);
  int status = 0;
  uint64_t total = 0;
  for (uint32_t i = 0; i < cnt; i++) {
    if (rc[i]) status = rc[i];
    offsets[i] = total;
    total += parts[i].m;
  }
  offsets[cnt] = total;
  if (!status) {
    if (!alloc_graph(out, 0, total)) {
      status = 4;
    } else {
      uint64_t nmax = 0;
      for (uint32_t i = 0; i < cnt; i++) {
        std::memcpy(out->src + offsets[i], parts[i].src, parts[i].m * sizeof(uint32_t));
        std::memcpy(out->dst + offsets[i], parts[i].dst, parts[i].m * sizeof(uint32_t));
        std::memcpy(out->sign + offsets[i], parts[i].sign, parts[i].m);
        nmax = std::max(nmax, parts[i].n);
      }
      out->n = nmax;
    }
  }
  for (auto& pt : parts) stc_synth_free(&pt);
  return status;
}

uint64_t stc_synth_workload_seed(int workload) { return 1000ull + (uint64_t)workload; }

int stc_synth_workload(int workload, uint32_t shrink, stc_synth_graph* out) {
  uint64_t seed = stc_synth_workload_seed(workload);
  if (shrink > 12) return 1;
  switch (workload) {
    case 1:
      return stc_synth_er(seed, 10000 >> shrink, 100000 >> shrink, 0.7, out);
    case 2:
      return stc_synth_delaunay(seed, 1000000 >> shrink, 0.2, 0.6, out);
    case 3: {
      uint32_t scale = 24 - shrink;
      return stc_synth_rmat(seed, scale, 1ull << scale, 16ull << scale, 0.57, 0.19, 0.19, 0.5,
                            out);
    }
    case 5:
      return stc_synth_skew(seed, (64ull << 20) >> shrink, (128ull << 20) >> shrink, 32,
                            std::max<uint64_t>(1, 100000 >> shrink),
                            std::max<uint64_t>(1, 10000000 >> shrink), 0.8, out);
    default:
      return 1;
  }
}

}  // extern "C"
