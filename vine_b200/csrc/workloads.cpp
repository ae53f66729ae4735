// Seeded synthetic CSP workloads and file loaders (host C++).
//
// These stand in for the reference's input layer (include/io.hpp:22-93,
// include/task.hpp:10-77, include/graph.hpp:136-167) and for its benchmark
// datasets, which are not distributed with it.  Every generator draws from a
// single std::mt19937_64 stream in a fixed order, so a workload is a pure
// function of its parameters.  Budgets follow the COLA query convention the
// reference loads (cost_limit, include/task.hpp:61-76): between the smallest
// possible delay and the delay of the shortest-by-length path.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <numeric>
#include <queue>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vine.h"
#include "../../include/vine_workloads.h"
#include "common.h"

struct vine_workload {
  int32_t n = 0;
  std::vector<int64_t> row;
  std::vector<int32_t> col;
  std::vector<float> len, dly;
  std::vector<int32_t> src, dst;
  std::vector<float> budget, alpha;
};

namespace {

const float kInf = std::numeric_limits<float>::infinity();

// ---- random numbers (documented draw rules) -------------------------------
struct Rng {
  std::mt19937_64 g;
  explicit Rng(uint64_t seed) : g(seed) {}
  uint64_t u64() { return g(); }
  // uniform in [0, 1) with 53 random bits
  double uni() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform integer in [1, k]
  int uint1(int k) { return 1 + (int)(g() % (uint64_t)k); }
  // uniform integer in [0, k)
  int64_t below(int64_t k) { return (int64_t)(g() % (uint64_t)k); }
  // standard normal by Box-Muller (cosine branch only; two draws per value)
  double normal() {
    double u1 = 1.0 - uni();  // (0, 1]
    double u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  }
};

struct Arc {
  int32_t u, v;
  float len, dly;
};

// Builds CSR from arcs with a stable counting sort by source, so each
// vertex's arcs keep their generation order.
void build_csr(vine_workload *w, int32_t n, const std::vector<Arc> &arcs) {
  w->n = n;
  w->row.assign((size_t)n + 1, 0);
  for (const Arc &a : arcs) w->row[(size_t)a.u + 1]++;
  for (int32_t i = 0; i < n; ++i) w->row[(size_t)i + 1] += w->row[i];
  std::vector<int64_t> pos(w->row.begin(), w->row.end() - 1);
  w->col.resize(arcs.size());
  w->len.resize(arcs.size());
  w->dly.resize(arcs.size());
  for (const Arc &a : arcs) {
    int64_t p = pos[a.u]++;
    w->col[p] = a.v;
    w->len[p] = a.len;
    w->dly[p] = a.dly;
  }
}

int hw_threads(int req) {
  if (req > 0) return req;
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : (int)h;
}

template <typename F>
void parallel_for(int64_t count, int nthreads, F fn) {
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      int64_t i = next.fetch_add(1);
      if (i >= count) break;
      fn(i);
    }
  };
  if (nthreads <= 1 || count < 2) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < std::min<int64_t>(nthreads, count); ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}

// Lexicographic Dijkstra from s over (primary, secondary) weights, stopping
// once t is settled.  Returns (primary, secondary) distance of t.
struct LexDist {
  float a, b;
};
LexDist lex_dijkstra(const vine_workload *w, int32_t s, int32_t t, bool delay_first,
                     std::vector<float> &da, std::vector<float> &db,
                     std::vector<int32_t> &touched) {
  for (int32_t v : touched) {
    da[v] = kInf;
    db[v] = kInf;
  }
  touched.clear();
  struct Item {
    float a, b;
    int32_t v;
  };
  struct Cmp {
    bool operator()(const Item &x, const Item &y) const {
      if (x.a != y.a) return x.a > y.a;
      if (x.b != y.b) return x.b > y.b;
      return x.v > y.v;
    }
  };
  std::priority_queue<Item, std::vector<Item>, Cmp> pq;
  const float *wa = delay_first ? w->dly.data() : w->len.data();
  const float *wb = delay_first ? w->len.data() : w->dly.data();
  da[s] = 0.0f;
  db[s] = 0.0f;
  touched.push_back(s);
  pq.push({0.0f, 0.0f, s});
  while (!pq.empty()) {
    Item it = pq.top();
    pq.pop();
    if (it.a != da[it.v] || it.b != db[it.v]) continue;
    if (it.v == t) return {it.a, it.b};
    for (int64_t j = w->row[it.v]; j < w->row[(size_t)it.v + 1]; ++j) {
      int32_t x = w->col[j];
      float a = it.a + wa[j], b = it.b + wb[j];
      if (a < da[x] || (a == da[x] && b < db[x])) {
        if (da[x] == kInf) touched.push_back(x);
        da[x] = a;
        db[x] = b;
        pq.push({a, b, x});
      }
    }
  }
  return {kInf, kInf};
}

// Budget rule: floor(dmin + alpha * (dlen - dmin)); -1 when t is unreachable.
void compute_budgets(vine_workload *w, size_t first, int nthreads) {
  const int64_t count = (int64_t)(w->src.size() - first);
  w->budget.resize(w->src.size());
  struct Scratch {
    std::vector<float> a, b;
    std::vector<int32_t> touched;
  };
  const int nt = std::max(1, std::min<int>(nthreads, (int)std::max<int64_t>(count, 1)));
  std::vector<Scratch> scratch((size_t)nt);
  for (auto &s : scratch) {
    s.a.assign((size_t)w->n, kInf);
    s.b.assign((size_t)w->n, kInf);
  }
  std::atomic<int> slot{0};
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    Scratch &sc = scratch[(size_t)slot.fetch_add(1)];
    for (;;) {
      int64_t i = next.fetch_add(1);
      if (i >= count) break;
      size_t q = first + (size_t)i;
      int32_t s = w->src[q], t = w->dst[q];
      LexDist dd = lex_dijkstra(w, s, t, true, sc.a, sc.b, sc.touched);
      if (dd.a == kInf) {
        w->budget[q] = -1.0f;
        continue;
      }
      LexDist dl = lex_dijkstra(w, s, t, false, sc.a, sc.b, sc.touched);
      double dmin = dd.a, dlen = dl.b;
      w->budget[q] = (float)std::floor(dmin + (double)w->alpha[q] * (dlen - dmin));
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}

// BFS hop levels from s; returns the vertices at hop `h` (or at the farthest
// level when fewer than h levels exist).
void bfs_level(const vine_workload *w, int32_t s, int32_t h, std::vector<int32_t> &dist,
               std::vector<int32_t> &out) {
  std::fill(dist.begin(), dist.end(), -1);
  std::vector<int32_t> cur{s}, nxt;
  dist[s] = 0;
  int level = 0;
  std::vector<int32_t> last = cur;
  while (!cur.empty() && level < h) {
    nxt.clear();
    for (int32_t u : cur)
      for (int64_t j = w->row[u]; j < w->row[(size_t)u + 1]; ++j) {
        int32_t v = w->col[j];
        if (dist[v] < 0) {
          dist[v] = level + 1;
          nxt.push_back(v);
        }
      }
    ++level;
    if (!nxt.empty()) last = nxt;
    std::swap(cur, nxt);
  }
  out = cur.empty() ? last : cur;
}

// ---- graph generators -------------------------------------------------------

// 4-neighbour grid.  Vertex r*cols+c; for each vertex in id order the arcs to
// (up, down, left, right) that exist, each drawing len then delay ~ U{1..100}.
void gen_grid(vine_workload *w, Rng &rng, int rows, int cols) {
  std::vector<Arc> arcs;
  arcs.reserve((size_t)rows * cols * 4);
  const int dr[4] = {-1, 1, 0, 0}, dc[4] = {0, 0, -1, 1};
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c)
      for (int k = 0; k < 4; ++k) {
        int rr = r + dr[k], cc = c + dc[k];
        if (rr < 0 || rr >= rows || cc < 0 || cc >= cols) continue;
        float l = (float)rng.uint1(100);
        float d = (float)rng.uint1(100);
        arcs.push_back({r * cols + c, rr * cols + cc, l, d});
      }
  build_csr(w, rows * cols, arcs);
}

struct Dsu {
  std::vector<int32_t> p;
  explicit Dsu(int32_t n) : p((size_t)n) { std::iota(p.begin(), p.end(), 0); }
  int32_t find(int32_t x) {
    while (p[x] != x) {
      p[x] = p[p[x]];
      x = p[x];
    }
    return x;
  }
  bool unite(int32_t a, int32_t b) {
    a = find(a);
    b = find(b);
    if (a == b) return false;
    p[a] = b;
    return true;
  }
};

// Road-like planar graph.  Draw order: (1) jitter of every lattice point,
// row-major, x then y, each U[-0.4, 0.4); (2) one 64-bit key per candidate
// lattice edge (row-major; right neighbour then down neighbour); the edges of
// the minimum-key spanning tree (Kruskal) are always kept; (3) one U[0,1)
// per non-tree candidate, kept when below p = (m_target/2 - (n-1)) /
// (#non-tree); (4) per kept edge, in candidate order, arc u->v then v->u:
// len = max(1, round(100 * euclid)) (same both ways) and a delay per arc:
//   anticorr = 0: delay = max(1, round(len * exp(0.5 * N(0,1))))
//   anticorr = 1: delay = max(1, round(1e4 / len * U[0.5, 1.5)))
void gen_road(vine_workload *w, Rng &rng, int rows, int cols, int64_t m_target, bool anticorr) {
  const int32_t n = rows * cols;
  std::vector<double> px((size_t)n), py((size_t)n);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      int32_t v = r * cols + c;
      px[v] = c + (rng.uni() * 0.8 - 0.4);
      py[v] = r + (rng.uni() * 0.8 - 0.4);
    }
  struct Cand {
    int32_t u, v;
    uint64_t key;
  };
  std::vector<Cand> cand;
  cand.reserve((size_t)n * 2);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      int32_t v = r * cols + c;
      if (c + 1 < cols) cand.push_back({v, v + 1, rng.u64()});
      if (r + 1 < rows) cand.push_back({v, v + cols, rng.u64()});
    }
  std::vector<uint32_t> order(cand.size());
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return cand[a].key < cand[b].key || (cand[a].key == cand[b].key && a < b);
  });
  std::vector<uint8_t> keep(cand.size(), 0);
  Dsu dsu(n);
  int64_t tree = 0;
  for (uint32_t i : order)
    if (dsu.unite(cand[i].u, cand[i].v)) {
      keep[i] = 1;
      ++tree;
    }
  const int64_t nontree = (int64_t)cand.size() - tree;
  double p = nontree > 0 ? ((double)m_target / 2.0 - (double)tree) / (double)nontree : 0.0;
  p = std::min(1.0, std::max(0.0, p));
  for (size_t i = 0; i < cand.size(); ++i)
    if (!keep[i] && rng.uni() < p) keep[i] = 1;
  std::vector<Arc> arcs;
  for (size_t i = 0; i < cand.size(); ++i) {
    if (!keep[i]) continue;
    int32_t u = cand[i].u, v = cand[i].v;
    double e = std::hypot(px[u] - px[v], py[u] - py[v]);
    float l = (float)std::max(1.0, std::round(100.0 * e));
    for (int dir = 0; dir < 2; ++dir) {
      double d;
      if (anticorr)
        d = std::max(1.0, std::round(1e4 / l * (0.5 + rng.uni())));
      else
        d = std::max(1.0, std::round(l * std::exp(0.5 * rng.normal())));
      if (dir == 0)
        arcs.push_back({u, v, l, (float)d});
      else
        arcs.push_back({v, u, l, (float)d});
    }
  }
  build_csr(w, n, arcs);
}

// Chung-Lu power-law digraph.  Vertex weights w_i = (i + 1)^(-1/(gamma-1));
// m_target arcs are drawn, each as (source, target) by inverse-CDF sampling on
// the weights (two U[0,1) per arc); self loops are dropped and duplicates
// merged (sorted by source, then target).  Then len then delay ~ U{1..100}
// per arc in CSR order.
void gen_chunglu(vine_workload *w, Rng &rng, int64_t n, int64_t m_target, double gamma) {
  std::vector<double> cdf((size_t)n);
  double acc = 0.0, ex = -1.0 / (gamma - 1.0);
  for (int64_t i = 0; i < n; ++i) {
    acc += std::pow((double)(i + 1), ex);
    cdf[(size_t)i] = acc;
  }
  auto draw = [&]() -> int32_t {
    double x = rng.uni() * acc;
    auto it = std::upper_bound(cdf.begin(), cdf.end(), x);
    int64_t k = it - cdf.begin();
    return (int32_t)std::min<int64_t>(k, n - 1);
  };
  std::vector<uint64_t> keys;
  keys.reserve((size_t)m_target);
  for (int64_t k = 0; k < m_target; ++k) {
    int32_t u = draw(), v = draw();
    if (u == v) continue;
    keys.push_back(((uint64_t)(uint32_t)u << 32) | (uint32_t)v);
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  std::vector<Arc> arcs;
  arcs.reserve(keys.size());
  for (uint64_t key : keys) {
    float l = (float)rng.uint1(100);
    float d = (float)rng.uint1(100);
    arcs.push_back({(int32_t)(key >> 32), (int32_t)(key & 0xffffffffu), l, d});
  }
  build_csr(w, (int32_t)n, arcs);
}

// ---- query generators -------------------------------------------------------

// Uniform random distinct pairs; per pair either each of the fixed alphas, or
// (n_alpha == 0) one alpha ~ U[lo, hi) drawn right after the pair.
void gen_pairs(vine_workload *w, Rng &rng, int n_pairs, int n_alpha, const float *alpha,
               float lo, float hi) {
  for (int i = 0; i < n_pairs; ++i) {
    int32_t s = (int32_t)rng.below(w->n), t;
    do {
      t = (int32_t)rng.below(w->n);
    } while (t == s && w->n > 1);
    if (n_alpha > 0) {
      for (int a = 0; a < n_alpha; ++a) {
        w->src.push_back(s);
        w->dst.push_back(t);
        w->alpha.push_back(alpha[a]);
      }
    } else {
      w->src.push_back(s);
      w->dst.push_back(t);
      w->alpha.push_back((float)(lo + (hi - lo) * rng.uni()));
    }
  }
}

// Hop-sampled pairs.  Per query, in order: source ~ uniform vertex (moved to
// the next vertex id with an out-arc when it has none); hop h (log-uniform:
// round(exp(U[ln lo, ln hi))), else uniform integer in [lo, hi]); one U[0,1)
// u picking the sink as level[floor(u * |level|)] among the vertices at BFS
// hop h (the farthest level when fewer exist); alpha ~ U[alo, ahi) unless
// n_alpha > 0 (then alpha[0]).
void gen_hop_pairs(vine_workload *w, Rng &rng, int nq, int hop_lo, int hop_hi, bool log_uniform,
                   int n_alpha, const float *alpha, float alo, float ahi, int nthreads) {
  std::vector<int32_t> s(nq), h(nq);
  std::vector<double> u(nq);
  std::vector<float> al(nq);
  for (int i = 0; i < nq; ++i) {
    int32_t v = (int32_t)rng.below(w->n);
    for (int k = 0; k < w->n && w->row[(size_t)v + 1] == w->row[v]; ++k) v = (v + 1) % w->n;
    s[i] = v;
    if (log_uniform) {
      double x = std::log((double)hop_lo) + (std::log((double)hop_hi) - std::log((double)hop_lo)) * rng.uni();
      h[i] = (int32_t)std::lround(std::exp(x));
    } else {
      h[i] = hop_lo + (int32_t)rng.below(hop_hi - hop_lo + 1);
    }
    u[i] = rng.uni();
    al[i] = n_alpha > 0 ? alpha[0] : (float)(alo + (ahi - alo) * rng.uni());
  }
  std::vector<int32_t> t(nq);
  const int nt = std::max(1, std::min(nthreads, nq));
  std::vector<std::vector<int32_t>> dist((size_t)nt, std::vector<int32_t>((size_t)w->n));
  std::atomic<int> slot{0};
  std::atomic<int> next{0};
  auto worker = [&]() {
    int me = slot.fetch_add(1);
    std::vector<int32_t> level;
    for (;;) {
      int i = next.fetch_add(1);
      if (i >= nq) break;
      bfs_level(w, s[i], h[i], dist[(size_t)me], level);
      size_t k = std::min(level.size() - 1, (size_t)(u[i] * (double)level.size()));
      t[i] = level[k];
    }
  };
  std::vector<std::thread> pool;
  for (int k = 0; k < nt; ++k) pool.emplace_back(worker);
  for (auto &th : pool) th.join();
  for (int i = 0; i < nq; ++i) {
    w->src.push_back(s[i]);
    w->dst.push_back(t[i]);
    w->alpha.push_back(al[i]);
  }
}

bool weights_ok(const vine_workload *w) {
  for (size_t j = 0; j < w->col.size(); ++j) {
    if (!(w->len[j] >= 0.0f) || !(w->dly[j] >= 0.0f) || !std::isfinite(w->len[j]) ||
        !std::isfinite(w->dly[j]))
      return false;
    if (w->col[j] < 0 || w->col[j] >= w->n) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int vine_workload_default_params(int32_t config_id, vine_workload_params *p) {
  if (!p) return vine::fail(VINE_ERR_INVALID, "null params");
  std::memset(p, 0, sizeof(*p));
  p->seed = 1234u + (uint64_t)config_id;
  p->exponent = 2.2;
  p->alpha_lo = 0.1f;
  p->alpha_hi = 0.9f;
  switch (config_id) {
    case 1:  // 100x100 grid, 16 pairs, alpha = 0.5
      p->kind = VINE_WL_GRID;
      p->rows = 100;
      p->cols = 100;
      p->n_pairs = 16;
      p->n_alpha = 1;
      p->alpha[0] = 0.5f;
      break;
    case 2:  // 264k-vertex road-like graph, 300 pairs x alpha {0.2, 0.5, 0.8}
      p->kind = VINE_WL_ROAD_LOGNORMAL;
      p->rows = 500;
      p->cols = 528;
      p->m_target = 733000;
      p->n_pairs = 300;
      p->n_alpha = 3;
      p->alpha[0] = 0.2f;
      p->alpha[1] = 0.5f;
      p->alpha[2] = 0.8f;
      break;
    case 3:  // 1.5M-vertex road-like graph, anti-correlated delay, 200 queries
      p->kind = VINE_WL_ROAD_ANTICORR;
      p->rows = 1200;
      p->cols = 1250;
      p->m_target = 3900000;
      p->n_pairs = 200;
      p->n_alpha = 0;
      break;
    case 4:  // Chung-Lu, 100k vertices, ~2M arcs, 64 queries 3-6 hops apart
      p->kind = VINE_WL_CHUNGLU;
      p->n = 100000;
      p->m_target = 2000000;
      p->n_pairs = 64;
      p->n_alpha = 1;
      p->alpha[0] = 0.5f;
      p->hop_lo = 3;
      p->hop_hi = 6;
      break;
    case 5:  // the config-2 graph, 4096 queries, hops log-uniform in [10, 2000]
      p->kind = VINE_WL_ROAD_BATCH;
      p->seed = 1234u + 2u;  // same graph as config 2
      p->rows = 500;
      p->cols = 528;
      p->m_target = 733000;
      p->n_pairs = 4096;
      p->n_alpha = 0;
      p->hop_lo = 10;
      p->hop_hi = 2000;
      p->hop_log_uniform = 1;
      break;
    default:
      return vine::fail(VINE_ERR_INVALID, "config_id must be 1..5");
  }
  return VINE_OK;
}

int vine_workload_generate(const vine_workload_params *p, vine_workload **out) {
  if (!p || !out) return vine::fail(VINE_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    auto *w = new vine_workload();
    Rng rng(p->seed);
    const int nt = hw_threads(p->nthreads);
    switch (p->kind) {
      case VINE_WL_GRID:
        if (p->rows < 1 || p->cols < 1) {
          delete w;
          return vine::fail(VINE_ERR_INVALID, "grid needs rows, cols >= 1");
        }
        gen_grid(w, rng, p->rows, p->cols);
        break;
      case VINE_WL_ROAD_LOGNORMAL:
      case VINE_WL_ROAD_ANTICORR:
      case VINE_WL_ROAD_BATCH:
        if (p->rows < 1 || p->cols < 1) {
          delete w;
          return vine::fail(VINE_ERR_INVALID, "road graph needs rows, cols >= 1");
        }
        gen_road(w, rng, p->rows, p->cols, p->m_target, p->kind == VINE_WL_ROAD_ANTICORR);
        break;
      case VINE_WL_CHUNGLU:
        if (p->n < 2 || p->exponent <= 1.0) {
          delete w;
          return vine::fail(VINE_ERR_INVALID, "Chung-Lu needs n >= 2, exponent > 1");
        }
        gen_chunglu(w, rng, p->n, p->m_target, p->exponent);
        break;
      default:
        delete w;
        return vine::fail(VINE_ERR_INVALID, "unknown workload kind");
    }
    Rng qrng(p->query_seed);
    Rng &qr = p->query_seed ? qrng : rng;
    if (p->hop_hi > 0) {
      if (p->hop_lo < 1 || p->hop_hi < p->hop_lo) {
        delete w;
        return vine::fail(VINE_ERR_INVALID, "bad hop range");
      }
      gen_hop_pairs(w, qr, p->n_pairs, p->hop_lo, p->hop_hi, p->hop_log_uniform != 0,
                    p->n_alpha, p->alpha, p->alpha_lo, p->alpha_hi, nt);
    } else {
      gen_pairs(w, qr, p->n_pairs, p->n_alpha, p->alpha, p->alpha_lo, p->alpha_hi);
    }
    compute_budgets(w, 0, nt);
    *out = w;
    return VINE_OK;
  } catch (const std::exception &e) {
    return vine::fail(VINE_ERR_INTERNAL, e.what());
  }
}

int vine_workload_add_random_queries(vine_workload *w, uint64_t seed, int32_t n_pairs,
                                     int32_t n_alpha, const float *alpha) {
  if (!w || n_pairs < 0 || n_alpha < 1 || n_alpha > 4 || !alpha)
    return vine::fail(VINE_ERR_INVALID, "bad arguments");
  try {
    Rng rng(seed);
    size_t first = w->src.size();
    gen_pairs(w, rng, n_pairs, n_alpha, alpha, 0.0f, 0.0f);
    compute_budgets(w, first, hw_threads(0));
    return VINE_OK;
  } catch (const std::exception &e) {
    return vine::fail(VINE_ERR_INTERNAL, e.what());
  }
}

int vine_workload_load_mtx(const char *path, vine_workload **out) {
  if (!path || !out) return vine::fail(VINE_ERR_INVALID, "null argument");
  *out = nullptr;
  std::ifstream in(path);
  if (!in) return vine::fail(VINE_ERR_IO, std::string("cannot open ") + path);
  std::string line;
  int64_t n = -1, n2 = -1, m = -1;
  std::vector<Arc> arcs;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '%') continue;
    std::istringstream ss(line);
    if (n < 0) {
      if (!(ss >> n >> n2 >> m)) return vine::fail(VINE_ERR_IO, "bad size line");
      arcs.reserve((size_t)std::max<int64_t>(m, 0) * 2);
      continue;
    }
    int64_t eid, a, b;
    double l, d;
    if (!(ss >> eid >> a >> b >> l >> d)) return vine::fail(VINE_ERR_IO, "bad edge row: " + line);
    if (a < 0 || b < 0 || a >= n || b >= n) return vine::fail(VINE_ERR_IO, "vertex out of range");
    arcs.push_back({(int32_t)a, (int32_t)b, (float)l, (float)d});
    arcs.push_back({(int32_t)b, (int32_t)a, (float)l, (float)d});
  }
  if (n < 0) return vine::fail(VINE_ERR_IO, "missing size line");
  auto *w = new vine_workload();
  build_csr(w, (int32_t)n, arcs);
  if (!weights_ok(w)) {
    delete w;
    return vine::fail(VINE_ERR_IO, "negative or non-finite weight");
  }
  *out = w;
  return VINE_OK;
}

int vine_workload_load_cola(const char *graph_path, const char *query_path, vine_workload **out) {
  if (!graph_path || !out) return vine::fail(VINE_ERR_INVALID, "null argument");
  *out = nullptr;
  FILE *f = std::fopen(graph_path, "r");
  if (!f) return vine::fail(VINE_ERR_IO, std::string("cannot open ") + graph_path);
  int n = 0;
  if (std::fscanf(f, "%d", &n) != 1 || n < 0) {
    std::fclose(f);
    return vine::fail(VINE_ERR_IO, "missing vertex count");
  }
  std::vector<Arc> arcs;
  int u, v, len, dly;
  while (std::fscanf(f, "%d:", &u) == 1) {
    while (std::fscanf(f, "%d", &v) == 1) {
      if (v == -1) break;
      if (std::fscanf(f, "%d %d", &len, &dly) != 2 || u < 0 || u >= n || v < 0 || v >= n) {
        std::fclose(f);
        return vine::fail(VINE_ERR_IO, "bad adjacency entry");
      }
      arcs.push_back({u, v, (float)len, (float)dly});
    }
  }
  std::fclose(f);
  auto *w = new vine_workload();
  build_csr(w, n, arcs);
  if (!weights_ok(w)) {
    delete w;
    return vine::fail(VINE_ERR_IO, "negative or non-finite weight");
  }
  if (query_path) {
    FILE *q = std::fopen(query_path, "r");
    if (!q) {
      delete w;
      return vine::fail(VINE_ERR_IO, std::string("cannot open ") + query_path);
    }
    int a, b, lo, hi, lim;
    while (std::fscanf(q, "%d %d %d %d %d", &a, &b, &lo, &hi, &lim) == 5) {
      if (a < 0 || a >= n || b < 0 || b >= n) {
        std::fclose(q);
        delete w;
        return vine::fail(VINE_ERR_IO, "query vertex out of range");
      }
      w->src.push_back(a);
      w->dst.push_back(b);
      w->budget.push_back((float)lim);
      w->alpha.push_back(-1.0f);
    }
    std::fclose(q);
  }
  *out = w;
  return VINE_OK;
}

int vine_workload_graph(const vine_workload *w, int32_t *n, int64_t *m, const int64_t **row_ptr,
                        const int32_t **col, const float **len, const float **delay) {
  if (!w) return vine::fail(VINE_ERR_INVALID, "null workload");
  if (n) *n = w->n;
  if (m) *m = (int64_t)w->col.size();
  if (row_ptr) *row_ptr = w->row.data();
  if (col) *col = w->col.data();
  if (len) *len = w->len.data();
  if (delay) *delay = w->dly.data();
  return VINE_OK;
}

int vine_workload_queries(const vine_workload *w, int32_t *nq, const int32_t **src,
                          const int32_t **dst, const float **budget, const float **alpha) {
  if (!w) return vine::fail(VINE_ERR_INVALID, "null workload");
  if (nq) *nq = (int32_t)w->src.size();
  if (src) *src = w->src.data();
  if (dst) *dst = w->dst.data();
  if (budget) *budget = w->budget.data();
  if (alpha) *alpha = w->alpha.data();
  return VINE_OK;
}

void vine_workload_destroy(vine_workload *w) { delete w; }

}  // extern "C"
