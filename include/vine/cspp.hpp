// vine/cspp.hpp -- header-only C++ drop-in for the reference's CSP query API.
//
// Keeps the names, members and argument meanings of the reference's problem
// types, graph model and query class, so that a caller written against them
// (main.cu:17-83: read_graph -> adj_to_csr -> el = create_edge_list(g) ->
// make_gpu_graph -> cspp(...) -> solve()) compiles with its includes replaced
// by this one header:
//
//   c_edge                      include/edge.hpp:16-26
//   c_label (CSP=1)             include/label.hpp:170-247
//   c_constraint<Label_t>       include/constraint.hpp:81-105
//   Edge, Vertex<Graph_t>       include/graph.hpp:25-88
//   Graph<Edge_t>               include/graph.hpp:90-195 (adjacency + CSR + make_gpu_graph)
//   read_graph                  include/io.hpp:22-93     (vine/io.hpp)
//   task                        include/task.hpp:10-77   (vine/io.hpp)
//   cuda_err_chk                include/util.hpp:14-20   (vine/io.hpp)
//   cspp<Label_t, Edge_t>       algorithm/cspp.hpp:11-69
//
// Everything is forwarded to the C ABI in vine.h; the GPU work happens in
// libvine.so.  Differences from the reference, all additive or fixes:
//   * make_gpu_graph() uploads through vine_graph_create (gg is the engine's
//     graph handle, not a gpuGraph); arc weights come from el[_eid_col[j]]
//     when the caller set el, as the reference's kernels read them
//     (algorithm/bucket.cuh:73), else from _len / _delay;
//   * solve() fills path_l / size_of_result_l (the reference left them
//     empty) and cost_l / delay_l / found_l / status_l; it uses C_l[i] for
//     task i (the reference's GPU driver applied C_l[0] to every task,
//     algorithm/cspp.cuh:196,234);
//   * solve() returns the vine_status of the call instead of always 0;
//   * cspp keeps its own copy of the constraints (the reference held a
//     reference, which its single-query constructor left unbound,
//     algorithm/cspp.hpp:25-34), and path_l points into one block sized by
//     the answers (the reference reserved N ints per task);
//   * the graph's CSR arrays and device graph are freed with the Graph.
#ifndef VINE_CSPP_HPP_
#define VINE_CSPP_HPP_

#include <cstdint>
#include <cstdlib>
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
  static bool dominate_vid(const c_label &a, const c_label &b) {
    return a.vid == b.vid && dominate(a, b);
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

template <typename Edge_t>
class Graph;

// One arc of the adjacency model (include/graph.hpp:25-61).
class Edge {
 public:
  int id;
  int src, snk;
  float len, delay;
  Edge() {}
  Edge(int id_) : id(id_) {}
  int assign(int id_, int src_, int snk_, float len_ = 0.0f, float delay_ = 0.0f) {
    id = id_;
    src = src_;
    snk = snk_;
    len = len_;
    delay = delay_;
    return 0;
  }
  int getOwner() const { return src; }
};

// One vertex with its out-arcs (edges, next) and in-arcs (edges_r, pre)
// (include/graph.hpp:63-88).
template <typename Graph_t>
class Vertex {
 public:
  int id;
  std::vector<Edge *> edges;
  std::vector<int> next;
  std::vector<Edge *> edges_r;
  std::vector<int> pre;
  Vertex() {}
  Vertex(int id_) : id(id_) {}
  int assign(Edge *e, Graph_t *g) {
    edges.push_back(e);
    next.push_back(e->snk);
    Vertex *son = &(g->v_l[e->snk]);
    son->edges_r.push_back(e);
    son->pre.push_back(id);
    return 0;
  }
};

// The reference's graph: adjacency lists (v_l, e_l) filled by the caller or
// by read_graph, then adj_to_csr() and make_gpu_graph().
template <typename Edge_t>
class Graph {
 public:
  using MyV = Vertex<Graph<Edge_t>>;
  std::vector<MyV> v_l;
  std::vector<Edge *> e_l;
  int N = 0, M = 0;

  // CSR part (include/graph.hpp:99-107), malloc'd by adj_to_csr
  int *_count_row = nullptr;  // CSR row pointer [N + 1]
  int *_eid_col = nullptr;    // edge id of each CSR slot [M]
  int *_vid_col = nullptr;    // head vertex of each CSR slot [M]
  int *e_sink = nullptr;      // edge id -> its tail vertex (the reference's naming) [M]
  int *e_csr = nullptr;       // edge id -> CSR slot [M]
  float *_len = nullptr;      // CSR arc length [M]
  float *_delay = nullptr;    // CSR arc delay [M]

  Edge_t *el = nullptr;  // per edge id {len, delay}; set by the caller (main.cu:62)

  vine_graph *gg = nullptr;  // the engine's device graph (make_gpu_graph)
  int device = 0;

  Graph() {}
  Graph(int n, int m) : e_l(m), N(n), M(m) {
    v_l.reserve(n);
    for (int i = 0; i < n; i++) v_l.push_back(MyV(i));
    for (int i = 0; i < m; i++) e_l[i] = new Edge(i);
  }
  ~Graph() {
    vine_graph_destroy(gg);
    free_csr();
  }
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;

  // Fills the adjacency model from an arc list (u, v, len, delay), arcs of a
  // vertex in list order.  A helper of this header; the reference's callers
  // fill v_l / e_l themselves or through read_graph.
  void from_arcs(int n, const std::vector<int> &u, const std::vector<int> &v,
                 const std::vector<float> &len, const std::vector<float> &delay) {
    N = n;
    M = (int)u.size();
    v_l.clear();
    v_l.reserve(n);
    for (int i = 0; i < n; i++) v_l.push_back(MyV(i));
    e_l.assign((size_t)M, nullptr);
    for (int j = 0; j < M; j++) {
      e_l[j] = new Edge(j);
      e_l[j]->assign(j, u[j], v[j], len[j], delay[j]);
      v_l[u[j]].assign(e_l[j], this);
    }
  }

  // CSR from the adjacency lists: slot order = each vertex's edges in
  // insertion order (include/graph.hpp:136-167).
  int adj_to_csr() {
    free_csr();
    _count_row = (int *)std::malloc(sizeof(int) * ((size_t)N + 1));
    const size_t mb = (size_t)(M > 0 ? M : 1);
    _eid_col = (int *)std::malloc(sizeof(int) * mb);
    _vid_col = (int *)std::malloc(sizeof(int) * mb);
    e_sink = (int *)std::malloc(sizeof(int) * mb);
    e_csr = (int *)std::malloc(sizeof(int) * mb);
    _len = (float *)std::malloc(sizeof(float) * mb);
    _delay = (float *)std::malloc(sizeof(float) * mb);
    if (!_count_row || !_eid_col || !_vid_col || !e_sink || !e_csr || !_len || !_delay) {
      free_csr();
      return VINE_ERR_INVALID;
    }
    _count_row[0] = 0;
    for (int i = 0; i < N; i++) {
      const int deg = (int)v_l[i].edges.size();
      _count_row[i + 1] = _count_row[i] + deg;
      if (_count_row[i + 1] > M) {  // more arcs in v_l than M says
        free_csr();
        return VINE_ERR_INVALID;
      }
      for (int t = 0; t < deg; t++) {
        const Edge *e = v_l[i].edges[t];
        const int j = _count_row[i] + t;
        e_csr[e->id] = j;
        e_sink[e->id] = e->src;
        _eid_col[j] = e->id;
        _vid_col[j] = e->snk;
        _len[j] = e->len;
        _delay[j] = e->delay;
      }
    }
    return 0;
  }

  // Uploads the CSR to the device (vine_graph_create); builds it first when
  // adj_to_csr() was not called.  Weights: el[_eid_col[j]] when el is set.
  int make_gpu_graph() {
    if (gg) return 0;
    if (_count_row == nullptr) {
      if (int rc = adj_to_csr()) return rc;
    }
    const int m = _count_row[N];
    std::vector<int64_t> row((size_t)N + 1);
    for (int i = 0; i <= N; ++i) row[i] = _count_row[i];
    std::vector<float> len((size_t)m), dly((size_t)m);
    for (int j = 0; j < m; ++j) {
      if (el != nullptr) {
        const Edge_t &e = el[_eid_col[j]];
        len[j] = e.len;
        dly[j] = e.delay;
      } else {
        len[j] = _len[j];
        dly[j] = _delay[j];
      }
    }
    return vine_graph_create(device, N, m, row.data(), _vid_col, len.data(), dly.data(), &gg);
  }

 private:
  void free_csr() {
    std::free(_count_row);
    std::free(_eid_col);
    std::free(_vid_col);
    std::free(e_sink);
    std::free(e_csr);
    std::free(_len);
    std::free(_delay);
    _count_row = _eid_col = _vid_col = e_sink = e_csr = nullptr;
    _len = _delay = nullptr;
  }
};

template <typename Label_t, typename Edge_t>
class cspp {
  using Graph_t = Graph<Edge_t>;
  using Constraint_t = c_constraint<Label_t>;

 public:
  int *path = nullptr;  // the block path_l points into
  std::vector<Label_t> init_state;
  std::vector<int> sink_l;
  int ntask = 0;
  std::vector<int *> path_l;          // path of task i: path_l[i][0 .. size_of_result_l[i])
  std::vector<int> size_of_result_l;  // 0 when task i has no feasible path
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
  ~cspp() { std::free(path); }
  cspp(const cspp &) = delete;
  cspp &operator=(const cspp &) = delete;

  // algorithm/cspp.hpp:48-53: runs the GPU engine and fills the results.
  int solve() {
    if (int rc = g->make_gpu_graph()) return rc;
    if ((int)init_state.size() < ntask || (int)sink_l.size() < ntask || (int)C_l.size() < ntask)
      return VINE_ERR_INVALID;
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
    std::free(path);
    int64_t cap = (int64_t)ntask * 64 + 1024;
    path = (int *)std::malloc(sizeof(int) * (size_t)cap);
    vine_results r = {};
    r.cost = cost_l.data();
    r.delay = delay_l.data();
    r.found = found_l.data();
    r.status = status_l.data();
    r.path_offsets = off.data();
    r.path = path;
    r.path_capacity = cap;
    int rc = vine_solve(g->gg, ntask, src.data(), dst.data(), bud.data(), &config, &r);
    if (rc == VINE_ERR_CAPACITY && off[ntask] > cap) {  // paths longer than guessed
      cap = off[ntask];
      std::free(path);
      path = (int *)std::malloc(sizeof(int) * (size_t)cap);
      r.path = path;
      r.path_capacity = cap;
      rc = vine_solve(g->gg, ntask, src.data(), dst.data(), bud.data(), &config, &r);
    }
    path_l.assign(ntask, nullptr);
    size_of_result_l.assign(ntask, 0);
    if (off[ntask] <= cap) {
      for (int i = 0; i < ntask; ++i) {
        path_l[i] = path + off[i];
        size_of_result_l[i] = (int)(off[i + 1] - off[i]);
      }
    }
    return rc;
  }

  // algorithm/cspp.hpp:55-61: the race-free multi-core CPU engine
  // (vine_solve_host) on one thread / on all cores; same results as solve().
  int solve_cpu() { return solve_host(1); }
  int solve_omp() { return solve_host(0); }

  int self_validate() { return 0; }

 private:
  int solve_host(int nthreads) {
    if (g->_count_row == nullptr) {
      if (int rc = g->adj_to_csr()) return rc;
    }
    if ((int)init_state.size() < ntask || (int)sink_l.size() < ntask || (int)C_l.size() < ntask)
      return VINE_ERR_INVALID;
    const int n = g->N, m = g->_count_row[n];
    std::vector<int64_t> row((size_t)n + 1);
    for (int i = 0; i <= n; ++i) row[i] = g->_count_row[i];
    std::vector<float> len((size_t)m), dly((size_t)m);
    for (int j = 0; j < m; ++j) {
      len[j] = g->el ? g->el[g->_eid_col[j]].len : g->_len[j];
      dly[j] = g->el ? g->el[g->_eid_col[j]].delay : g->_delay[j];
    }
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
    std::free(path);
    const int64_t cap = (int64_t)ntask * (int64_t)(n + 1);  // a path visits each vertex once
    path = (int *)std::malloc(sizeof(int) * (size_t)std::max<int64_t>(cap, 1));
    vine_results r = {};
    r.cost = cost_l.data();
    r.delay = delay_l.data();
    r.found = found_l.data();
    r.status = status_l.data();
    r.path_offsets = off.data();
    r.path = path;
    r.path_capacity = cap;
    const int rc = vine_solve_host(n, m, row.data(), g->_vid_col, len.data(), dly.data(), ntask,
                                   src.data(), dst.data(), bud.data(), nthreads, 0, &r);
    path_l.assign(ntask, nullptr);
    size_of_result_l.assign(ntask, 0);
    for (int i = 0; i < ntask; ++i) {
      path_l[i] = path + off[i];
      size_of_result_l[i] = (int)(off[i + 1] - off[i]);
    }
    return rc;
  }
};

#include "io.hpp"

#endif  // VINE_CSPP_HPP_
