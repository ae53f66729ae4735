// vine/cspp.hpp -- header-only C++ drop-in for the reference's CSP query API.
//
// Keeps the names and argument meanings of the reference's problem types and
// query class so that a caller written against them (main.cu:61-81) compiles
// with a changed include:
//
//   c_edge                      include/edge.hpp:16-26
//   c_label (CSP=1)             include/label.hpp:170-247
//   c_constraint<Label_t>       include/constraint.hpp:81-105
//   Graph<Edge_t>               include/graph.hpp:90-195 (CSR part + make_gpu_graph)
//   cspp<Label_t, Edge_t>       algorithm/cspp.hpp:11-69
//
// Everything is forwarded to the C ABI in vine.h; the GPU work happens in
// libvine.so.  Differences from the reference, all additive:
//   * solve() fills path_l / size_of_result_l (the reference left them
//     empty) and cost_l / delay_l / found_l; it uses C_l[i] for task i (the
//     reference's GPU driver applied C_l[0] to every task, cspp.cuh:196,234);
//   * it returns the vine_status of the call instead of always 0;
//   * the single-query constructor keeps its own constraint (the reference's
//     one bound a reference member to nothing, cspp.hpp:28-34).
#ifndef VINE_CSPP_HPP_
#define VINE_CSPP_HPP_

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../vine.h"

class c_edge {
 public:
  float len;
  float delay;
  c_edge() {}
  c_edge(float l, float d) : len(l), delay(d) {}
};

class c_label {
 public:
  int vid;
  float d;
  float delay;
  c_label() {}
  explicit c_label(int v) : vid(v), d(0), delay(0) {}
  c_label(int v, float d_, float delay_) : vid(v), d(d_), delay(delay_) {}
  // additive expansion, as the reference's device expand (label.hpp:214-222)
  template <typename Edge_t>
  void expand(int next_v, const Edge_t &e, c_label *son) const {
    son->vid = next_v;
    son->d = d + e.len;
    son->delay = delay + e.delay;
  }
  static bool dominate(const c_label &a, const c_label &b) {
    return a.d <= b.d && a.delay <= b.delay;
  }
  static bool equal(const c_label &a, const c_label &b) {
    return a.vid == b.vid && a.d == b.d && a.delay == b.delay;
  }
};

template <typename Label_t>
class c_constraint {
 public:
  float delay_L;
  c_constraint() : delay_L(0) {}
  c_constraint(float d) : delay_L(d) {}
  void set_constraints(int d) { delay_L = (float)d; }
  bool pass_constraints_check(const Label_t &l) const { return !(l.delay > delay_L); }
  bool pass_constraints_check_cpu(const Label_t &l) const { return !(l.delay > delay_L); }
};

// CSR graph (the reference's Graph CSR arrays without the edge-id
// indirection).  Fill N, M, _count_row, _vid_col, _len, _delay (the
// reference's names for row pointers, heads and weights), then call
// make_gpu_graph().
template <typename Edge_t>
class Graph {
 public:
  int N = 0, M = 0;
  std::vector<int64_t> _count_row;  // N + 1
  std::vector<int32_t> _vid_col;    // M
  std::vector<float> _len, _delay;  // M
  vine_graph *gg = nullptr;         // device graph
  int device = 0;

  Graph() {}
  Graph(int n, int m) : N(n), M(m), _count_row((size_t)n + 1, 0) {}
  ~Graph() { vine_graph_destroy(gg); }
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;

  // Builds CSR from an arc list (u, v, len, delay) in the given order.
  void from_arcs(int n, const std::vector<int> &u, const std::vector<int> &v,
                 const std::vector<float> &len, const std::vector<float> &delay) {
    N = n;
    M = (int)u.size();
    _count_row.assign((size_t)n + 1, 0);
    for (int x : u) _count_row[(size_t)x + 1]++;
    for (int i = 0; i < n; ++i) _count_row[(size_t)i + 1] += _count_row[i];
    std::vector<int64_t> pos(_count_row.begin(), _count_row.end() - 1);
    _vid_col.resize(M);
    _len.resize(M);
    _delay.resize(M);
    for (int j = 0; j < M; ++j) {
      const int64_t p = pos[u[j]]++;
      _vid_col[p] = v[j];
      _len[p] = len[j];
      _delay[p] = delay[j];
    }
  }
  int adj_to_csr() { return 0; }  // the CSR is built by from_arcs
  int make_gpu_graph() {
    if (gg) return 0;
    return vine_graph_create(device, N, M, _count_row.data(), _vid_col.data(), _len.data(),
                             _delay.data(), &gg);
  }
};

template <typename Label_t, typename Edge_t>
class cspp {
  using Graph_t = Graph<Edge_t>;
  using Constraint_t = c_constraint<Label_t>;

 public:
  std::vector<Label_t> init_state;
  std::vector<int> sink_l;
  int ntask = 0;
  std::vector<std::vector<int>> path_l;
  std::vector<int> size_of_result_l;
  std::vector<float> cost_l, delay_l;
  std::vector<int> found_l, status_l;
  Graph_t *g = nullptr;
  std::vector<Constraint_t> C_l;
  vine_config config;

  // one query (algorithm/cspp.hpp:28-34)
  cspp(Graph_t *g_, Label_t source_state, int sink, Constraint_t C) : g(g_) {
    ntask = 1;
    init_state.push_back(source_state);
    sink_l.push_back(sink);
    C_l.push_back(C);
    vine_config_default(&config);
  }
  // ntask queries (algorithm/cspp.hpp:36-46)
  cspp(Graph_t *g_, int ntask_, std::vector<Label_t> &source_state, std::vector<int> &sinks,
       std::vector<Constraint_t> &C)
      : init_state(source_state), sink_l(sinks), ntask(ntask_), g(g_), C_l(C) {
    vine_config_default(&config);
  }

  // algorithm/cspp.hpp:48-53: runs the GPU engine and fills the results.
  int solve() {
    if (int rc = g->make_gpu_graph()) return rc;
    std::vector<int32_t> src(ntask), dst(ntask);
    std::vector<float> bud(ntask);
    for (int i = 0; i < ntask; ++i) {
      src[i] = init_state[i].vid;
      dst[i] = sink_l[i];
      bud[i] = C_l[i].delay_L;
    }
    cost_l.assign(ntask, 0.0f);
    delay_l.assign(ntask, 0.0f);
    found_l.assign(ntask, 0);
    status_l.assign(ntask, 0);
    std::vector<int64_t> off((size_t)ntask + 1, 0);
    std::vector<int32_t> path((size_t)ntask * 64 + 1024);
    vine_results r = {};
    r.cost = cost_l.data();
    r.delay = delay_l.data();
    r.found = found_l.data();
    r.status = status_l.data();
    r.path_offsets = off.data();
    r.path = path.data();
    r.path_capacity = (int64_t)path.size();
    int rc = vine_solve(g->gg, ntask, src.data(), dst.data(), bud.data(), &config, &r);
    if (rc == VINE_ERR_CAPACITY && off[ntask] > r.path_capacity) {
      path.resize((size_t)off[ntask]);
      r.path = path.data();
      r.path_capacity = (int64_t)path.size();
      rc = vine_solve(g->gg, ntask, src.data(), dst.data(), bud.data(), &config, &r);
    }
    path_l.assign(ntask, {});
    size_of_result_l.assign(ntask, 0);
    for (int i = 0; i < ntask && off[ntask] <= r.path_capacity; ++i) {
      path_l[i].assign(path.begin() + off[i], path.begin() + off[i + 1]);
      size_of_result_l[i] = (int)path_l[i].size();
    }
    return rc;
  }

  int self_validate() { return 0; }
};

#endif  // VINE_CSPP_HPP_
