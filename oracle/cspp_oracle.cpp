// CPU ORACLE FOR THE EXACT CSP QUERY PATH -- TEST INFRASTRUCTURE ONLY.
//
// This file is the checker, never the product.  Only the test-suite, the smoke
// check in __graft_entry__.py and the cpu_baseline leg of bench.py load it.
// The shipped engine (vine_b200/libvine.so) never links or calls it.
//
// Three routines live here:
//
//   oracle_solve_reference_rules
//       A restatement of the reference CPU solver RUN_CSPP_CPU
//       (algorithm/cspp_cpu.hpp:44-125) and its helper add_new_frontier
//       (algorithm/cspp_cpu.hpp:16-42): round-synchronous label correcting,
//       per-vertex linear Pareto stores with erase, next frontier deduplicated
//       per vertex and emitted in vertex-id order (std::map iteration).
//       Label arithmetic follows the *device* c_label::expand
//       (include/label.hpp:214-222: d += len, delay += e.delay); the shipped
//       host twin expand_cpu multiplies (include/label.hpp:224-232), which
//       makes every CPU cost 0, so it is not followed.  dominate is
//       `a.d <= b.d && a.delay <= b.delay` (include/label.hpp:234-236,244-246);
//       the constraint is `!(delay > delay_L)` (include/constraint.hpp:99-104).
//       Unlike the reference it also returns what the reference never
//       extracts: the sink's Pareto set, the lexicographically smallest
//       feasible (cost, delay) label and its path, plus work counters.
//
//   oracle_solve_label_setting
//       A sequential label-setting search that applies exactly the pruning
//       rules of the GPU engine (constraint with optional delay lower bounds,
//       Pareto dominance, optional incumbent pruning with optional A* cost
//       lower bounds) in strict lexicographic (f, delay) order.  Its counters
//       are the minimal work under those rules and define the algorithmic
//       bytes per query used for the roofline.
//
//   oracle_dijkstra
//       Lexicographic single-source shortest paths (primary, secondary
//       weight); used by the tests to compute exact lower bounds and budgets.
//
// Exactness: all weights used by the workloads are integers whose path sums
// stay below 2^24, so every FP32 addition here is exact and order-free.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <queue>
#include <vector>

namespace {

const float kInf = std::numeric_limits<float>::infinity();

// Optional wall-clock limit of the next label-setting searches on this thread
// (oracle_set_time_limit); a search that passes it stops and returns 2.
thread_local double tl_limit_s = 0.0;

struct Lab {
  int vid;
  float d;
  float delay;
  int node;  // index into the parent arena
};

struct Node {
  int vid;
  int parent;
};

// include/label.hpp:234-236 (device) and :244-246 (host): weak dominance.
inline bool dominate(const Lab &a, const Lab &b) {
  return a.d <= b.d && a.delay <= b.delay;
}

inline bool lex_less(float d0, float l0, float d1, float l1) {
  return d0 < d1 || (d0 == d1 && l0 < l1);
}

struct Csr {
  int n;
  const int64_t *row;
  const int32_t *col;
  const float *len;
  const float *dly;
};

struct Counters {
  int64_t P = 0, R = 0, S = 0, I = 0, dom_calls = 0, rounds = 0;
};

// Walks the parent arena from `node` back to the source and writes the vertex
// sequence source -> sink into path[0..len).  Returns the path length, or -1
// when the caller's buffer is too small.
int write_path(const std::vector<Node> &arena, int node, int32_t *path, int cap) {
  int len = 0;
  for (int k = node; k >= 0; k = arena[k].parent) ++len;
  if (path == nullptr) return len;
  if (len > cap) return -1;
  int pos = len - 1;
  for (int k = node; k >= 0; k = arena[k].parent) path[pos--] = arena[k].vid;
  return len;
}

int write_pareto(std::vector<Lab> labs, float *pd, float *pl, int cap) {
  std::sort(labs.begin(), labs.end(), [](const Lab &a, const Lab &b) {
    return lex_less(a.d, a.delay, b.d, b.delay);
  });
  std::vector<Lab> front;
  float best_delay = kInf;
  for (const Lab &l : labs) {
    if (l.delay < best_delay) {
      front.push_back(l);
      best_delay = l.delay;
    }
  }
  int n = (int)front.size();
  if (pd != nullptr && pl != nullptr) {
    for (int i = 0; i < n && i < cap; ++i) {
      pd[i] = front[i].d;
      pl[i] = front[i].delay;
    }
  }
  return n;
}

// algorithm/cspp_cpu.hpp:16-42
void add_new_frontier(std::map<int, std::vector<Lab>> &next_round, const Lab &nl,
                      Counters &c) {
  auto it = next_round.find(nl.vid);
  if (it == next_round.end()) {
    next_round[nl.vid] = std::vector<Lab>{nl};
    return;
  }
  std::vector<Lab> &vec = it->second;
  for (size_t k = 0; k < vec.size();) {
    c.dom_calls++;
    if (dominate(vec[k], nl)) return;  // new label is dominated
    c.dom_calls++;
    if (dominate(nl, vec[k])) {
      vec.erase(vec.begin() + (long)k);  // new label dominates a queued one
    } else {
      ++k;
    }
  }
  vec.push_back(nl);
}

}  // namespace

extern "C" {

// Output record shared by the oracle entry points (mirrored in oracle/oracle.py).
typedef struct {
  float cost;      // lexicographically smallest feasible (cost, delay): cost
  float delay;     //   ... and its delay
  int32_t found;   // 1 when a feasible path exists
  int32_t path_len;
  int32_t pareto_n;
  int32_t pad;
  int64_t P;       // labels popped and expanded
  int64_t R;       // edges relaxed (expand calls)
  int64_t S;       // stored labels read by dominance tests
  int64_t I;       // labels inserted into a store
  int64_t dom_calls;
  int64_t rounds;
} oracle_result;

// Restatement of RUN_CSPP_CPU (algorithm/cspp_cpu.hpp:44-125) for one query.
// path/pareto buffers may be null.  Returns 0, or -1 when a buffer was short.
int oracle_solve_reference_rules(int32_t n, const int64_t *row_ptr, const int32_t *col,
                                 const float *len, const float *delay, int32_t src,
                                 int32_t dst, float budget, int32_t *path, int32_t path_cap,
                                 float *pareto_d, float *pareto_delay, int32_t pareto_cap,
                                 oracle_result *out) {
  Csr g{n, row_ptr, col, len, delay};
  Counters c;
  std::vector<Node> arena;
  arena.push_back({src, -1});
  Lab source{src, 0.0f, 0.0f, 0};

  float best_d = kInf, best_l = kInf;
  int best_node = -1;
  if (src == dst && !(0.0f > budget)) {  // the source label is a feasible sink label
    best_d = 0.0f;
    best_l = 0.0f;
    best_node = 0;
  }

  std::vector<Lab> frontiers;                      // cspp_cpu.hpp:63
  std::map<int, std::vector<Lab>> dominance_list;  // cspp_cpu.hpp:64
  std::map<int, std::vector<Lab>> next_round;      // cspp_cpu.hpp:65
  frontiers.push_back(source);
  while (!frontiers.empty()) {  // cspp_cpu.hpp:72
    c.rounds++;
    for (size_t ff = 0; ff < frontiers.size(); ++ff) {  // cspp_cpu.hpp:74
      const Lab frontier = frontiers[ff];
      c.P++;
      for (int64_t j = g.row[frontier.vid]; j < g.row[frontier.vid + 1]; ++j) {  // :77
        c.R++;
        Lab nl;  // expand (label.hpp:214-222): additive
        nl.vid = g.col[j];
        nl.d = frontier.d + g.len[j];
        nl.delay = frontier.delay + g.dly[j];
        nl.node = (int)arena.size();
        arena.push_back({nl.vid, frontier.node});
        if (nl.delay > budget) continue;  // pass_constraints_check_cpu, :80
        if (nl.vid == dst && lex_less(nl.d, nl.delay, best_d, best_l)) {
          best_d = nl.d;
          best_l = nl.delay;
          best_node = nl.node;
        }
        auto it = dominance_list.find(nl.vid);
        if (it != dominance_list.end()) {  // :83-108
          std::vector<Lab> &vec = it->second;
          bool dominated = false;
          for (size_t k = 0; k < vec.size();) {
            c.S++;
            c.dom_calls++;
            if (dominate(vec[k], nl)) {
              dominated = true;
              break;
            }
            c.dom_calls++;
            if (dominate(nl, vec[k])) {
              vec.erase(vec.begin() + (long)k);
            } else {
              ++k;
            }
          }
          if (dominated) continue;
          vec.push_back(nl);
          c.I++;
          add_new_frontier(next_round, nl, c);
        } else {
          dominance_list[nl.vid] = std::vector<Lab>{nl};
          c.I++;
          add_new_frontier(next_round, nl, c);
        }
      }
    }
    frontiers.clear();  // :111-115, next frontier in vertex-id order
    for (auto &kv : next_round) frontiers.insert(frontiers.end(), kv.second.begin(), kv.second.end());
    next_round.clear();
  }

  out->P = c.P;
  out->R = c.R;
  out->S = c.S;
  out->I = c.I;
  out->dom_calls = c.dom_calls;
  out->rounds = c.rounds;
  out->found = best_node >= 0 ? 1 : 0;
  out->cost = best_d;
  out->delay = best_l;
  out->path_len = 0;
  int rc = 0;
  if (best_node >= 0) {
    int pl = write_path(arena, best_node, path, path_cap);
    if (pl < 0) {
      rc = -1;
      pl = write_path(arena, best_node, nullptr, 0);
    }
    out->path_len = pl;
  }
  std::vector<Lab> sink_labels;
  auto it = dominance_list.find(dst);
  if (it != dominance_list.end()) sink_labels = it->second;
  if (src == dst && !(0.0f > budget)) sink_labels.push_back(source);
  out->pareto_n = write_pareto(sink_labels, pareto_d, pareto_delay, pareto_cap);
  if (out->pareto_n > pareto_cap && pareto_d != nullptr) rc = -1;
  return rc;
}

// Sequential label setting under the GPU engine's pruning rules.
//   h_len, h_del : optional lower bounds on the remaining cost / delay to dst
//                  (null = 0).  They must be consistent (exact reverse
//                  shortest-path distances are).
//   use_incumbent: prune labels whose lower-bound vector is lexicographically
//                  no better than the best feasible sink label found so far.
// With h_len = h_del = null and use_incumbent = 0 the popped sink labels are
// the full sink Pareto set, identical to the reference's final store.
int oracle_solve_label_setting(int32_t n, const int64_t *row_ptr, const int32_t *col,
                               const float *len, const float *delay, int32_t src, int32_t dst,
                               float budget, const float *h_len, const float *h_del,
                               int32_t use_incumbent, int32_t *path, int32_t path_cap,
                               float *pareto_d, float *pareto_delay, int32_t pareto_cap,
                               oracle_result *out) {
  Csr g{n, row_ptr, col, len, delay};
  Counters c;
  auto hl = [&](int v) { return h_len ? h_len[v] : 0.0f; };
  auto hd = [&](int v) { return h_del ? h_del[v] : 0.0f; };

  struct Item {
    float f, l;
    int64_t seq;
    int lab;
  };
  struct Cmp {
    bool operator()(const Item &a, const Item &b) const {
      if (a.f != b.f) return a.f > b.f;
      if (a.l != b.l) return a.l > b.l;
      return a.seq > b.seq;
    }
  };
  std::priority_queue<Item, std::vector<Item>, Cmp> pq;
  std::vector<Lab> labs;
  std::vector<Node> arena;
  std::vector<float> sdel((size_t)n, kInf);
  std::vector<Lab> sink_popped;
  int64_t seq = 0;

  float inc_d = kInf, inc_l = kInf;
  int inc_node = -1;
  out->path_len = 0;
  out->pareto_n = 0;

  if (!(0.0f + hd(src) > budget) && std::isfinite(hd(src)) && std::isfinite(hl(src))) {
    arena.push_back({src, -1});
    labs.push_back({src, 0.0f, 0.0f, 0});
    pq.push({hl(src), hd(src), seq++, 0});
    c.I++;
    if (src == dst) {
      inc_d = 0.0f;
      inc_l = 0.0f;
      inc_node = 0;
    }
  }
  const auto t_start = std::chrono::steady_clock::now();
  int64_t pops = 0;
  while (!pq.empty()) {
    if (tl_limit_s > 0.0 && (++pops & 4095) == 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count() >
            tl_limit_s) {
      out->found = 0;
      out->P = c.P;
      out->R = c.R;
      out->S = c.S;
      out->I = c.I;
      out->path_len = 0;
      out->pareto_n = 0;
      return 2;  // stopped at the time limit: no result
    }
    Item it = pq.top();
    pq.pop();
    const Lab lab = labs[it.lab];
    const int v = lab.vid;
    c.S++;
    if (lab.delay >= sdel[v]) continue;  // dominated by a popped label at v
    if (use_incumbent && inc_node >= 0 && !lex_less(it.f, lab.delay + hd(v), inc_d, inc_l))
      continue;
    sdel[v] = lab.delay;
    if (v == dst) sink_popped.push_back(lab);
    c.P++;
    for (int64_t j = g.row[v]; j < g.row[v + 1]; ++j) {
      c.R++;
      const int w = g.col[j];
      const float nd = lab.d + g.len[j];
      const float nl = lab.delay + g.dly[j];
      const float lbl = nl + hd(w);
      if (lbl > budget || !std::isfinite(lbl)) continue;
      c.S++;
      if (nl >= sdel[w]) continue;
      const float nf = nd + hl(w);
      if (!std::isfinite(nf)) continue;
      if (use_incumbent && inc_node >= 0 && !lex_less(nf, lbl, inc_d, inc_l)) continue;
      const int node = (int)arena.size();
      arena.push_back({w, lab.node});
      labs.push_back({w, nd, nl, node});
      pq.push({nf, lbl, seq++, (int)labs.size() - 1});
      c.I++;
      if (w == dst && lex_less(nd, nl, inc_d, inc_l)) {
        inc_d = nd;
        inc_l = nl;
        inc_node = node;
      }
    }
  }
  out->P = c.P;
  out->R = c.R;
  out->S = c.S;
  out->I = c.I;
  out->dom_calls = 0;
  out->rounds = 0;
  out->found = inc_node >= 0 ? 1 : 0;
  out->cost = inc_d;
  out->delay = inc_l;
  int rc = 0;
  if (inc_node >= 0) {
    int pl = write_path(arena, inc_node, path, path_cap);
    if (pl < 0) {
      rc = -1;
      pl = write_path(arena, inc_node, nullptr, 0);
    }
    out->path_len = pl;
  }
  out->pareto_n = write_pareto(sink_popped, pareto_d, pareto_delay, pareto_cap);
  if (out->pareto_n > pareto_cap && pareto_d != nullptr) rc = -1;
  return rc;
}

// Sets the wall-clock limit (seconds, 0 = none) of the label-setting searches
// that the calling thread runs next.
void oracle_set_time_limit(double seconds) { tl_limit_s = seconds > 0.0 ? seconds : 0.0; }

// Lexicographic Dijkstra over (w1, w2) from src.  dist1/dist2 receive the
// primary distance and the secondary weight of the lexicographically shortest
// path (+inf when unreachable).  parent (optional) receives the predecessor.
int oracle_dijkstra(int32_t n, const int64_t *row_ptr, const int32_t *col, const float *w1,
                    const float *w2, int32_t src, float *dist1, float *dist2, int32_t *parent) {
  for (int i = 0; i < n; ++i) {
    dist1[i] = kInf;
    dist2[i] = kInf;
    if (parent) parent[i] = -1;
  }
  struct Item {
    float a, b;
    int v;
  };
  struct Cmp {
    bool operator()(const Item &x, const Item &y) const {
      if (x.a != y.a) return x.a > y.a;
      if (x.b != y.b) return x.b > y.b;
      return x.v > y.v;
    }
  };
  std::priority_queue<Item, std::vector<Item>, Cmp> pq;
  dist1[src] = 0.0f;
  dist2[src] = 0.0f;
  pq.push({0.0f, 0.0f, src});
  while (!pq.empty()) {
    Item it = pq.top();
    pq.pop();
    if (it.a != dist1[it.v] || it.b != dist2[it.v]) continue;
    for (int64_t j = row_ptr[it.v]; j < row_ptr[it.v + 1]; ++j) {
      const int w = col[j];
      const float a = it.a + w1[j];
      const float b = it.b + w2[j];
      if (lex_less(a, b, dist1[w], dist2[w])) {
        dist1[w] = a;
        dist2[w] = b;
        if (parent) parent[w] = it.v;
        pq.push({a, b, w});
      }
    }
  }
  return 0;
}

}  // extern "C"
