// REFERENCE CPU SOLVER, INSTANTIATED UNMODIFIED -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile against the reference's own headers
// (algorithm/cspp_cpu.hpp and the include/ tree it pulls in) into
// oracle/_ref/libvine_ref.so.  Nothing here is shipped; the tests use it to
// pin the restatement in cspp_oracle.cpp, and bench.py times it as the CPU
// baseline.
//
// RUN_CSPP_CPU (algorithm/cspp_cpu.hpp:44-125) is a template over the label
// type.  The shipped CSP=1 c_label cannot be used: its expand_cpu multiplies
// (include/label.hpp:224-232), so every host label stays (0, 0).  OracleLabel
// below supplies the members the template uses -- vid, d, delay, expand_cpu,
// dominate_cpu -- with expand_cpu adding exactly like the device expand
// (include/label.hpp:214-222) and dominate_cpu as in include/label.hpp:244-246.
// The template returns no result (path_l / size_of_result_l are never
// written), so expand_cpu also records, in thread-local state, every label it
// creates at the sink that satisfies the budget and keeps the
// lexicographically smallest (cost, delay) one, plus an optional parent arena
// from which that label's path is rebuilt.  Every feasible sink label the
// search can produce passes through expand_cpu, so the minimum over those is
// the optimum the reference's search reaches.

#define CSP 1
#include "algorithm/cspp_cpu.hpp"

#include <unistd.h>
#include <fcntl.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <algorithm>
#include <limits>
#include <string>
#include <thread>
#include <vector>

namespace {

struct ArenaNode {
  int vid;
  int parent;
};

thread_local int tl_sink = -1;
thread_local float tl_budget = 0.0f;
thread_local bool tl_record = false;
thread_local std::vector<ArenaNode> *tl_arena = nullptr;
thread_local float tl_best_d = 0.0f;
thread_local float tl_best_l = 0.0f;
thread_local int tl_best_node = -1;
thread_local bool tl_found = false;
thread_local long long tl_expand_calls = 0;
thread_local long long tl_dom_calls = 0;
// optional per-query time cap: expand_cpu checks the clock every 1024 calls
// and unwinds out of the template (its state is all in std containers)
thread_local bool tl_capped = false;
thread_local std::chrono::steady_clock::time_point tl_deadline;
struct DeadlineExceeded {};

inline bool lex_less(float d0, float l0, float d1, float l1) {
  return d0 < d1 || (d0 == d1 && l0 < l1);
}

}  // namespace

class OracleLabel {
 public:
  int vid;
  float d;
  float delay;
  int node;

  OracleLabel() {}
  OracleLabel(int v) : vid(v), d(0), delay(0), node(-1) {}

  template <typename Edge_t>
  void expand_cpu(int next_v, Edge_t e, OracleLabel *son) {
    son->vid = next_v;
    son->d = this->d + e.len;
    son->delay = this->delay + e.delay;
    son->node = -1;
    tl_expand_calls++;
    if (tl_capped && (tl_expand_calls & 1023) == 0 &&
        std::chrono::steady_clock::now() > tl_deadline)
      throw DeadlineExceeded{};
    if (tl_record) {
      son->node = (int)tl_arena->size();
      tl_arena->push_back({next_v, this->node});
    }
    if (next_v == tl_sink && !(son->delay > tl_budget)) {
      if (!tl_found || lex_less(son->d, son->delay, tl_best_d, tl_best_l)) {
        tl_found = true;
        tl_best_d = son->d;
        tl_best_l = son->delay;
        tl_best_node = son->node;
      }
    }
  }

  static bool dominate_cpu(OracleLabel a, OracleLabel b) {
    tl_dom_calls++;
    return a.d <= b.d && a.delay <= b.delay;
  }
};

namespace {

struct RefGraph {
  Graph<c_edge> *g;
};

// Runs one query through RUN_CSPP_CPU on the calling thread.
void run_one(Graph<c_edge> *g, int src, int dst, float budget, bool record, float *cost,
             float *delay, int32_t *found, int32_t *path, int path_cap, int32_t *path_len,
             long long *calls) {
  std::vector<ArenaNode> arena;
  tl_sink = dst;
  tl_budget = budget;
  tl_record = record;
  tl_arena = &arena;
  tl_found = false;
  tl_best_node = -1;
  tl_expand_calls = 0;
  tl_dom_calls = 0;

  OracleLabel source(src);
  if (record) {
    source.node = 0;
    arena.push_back({src, -1});
  }
  if (src == dst && !(0.0f > budget)) {  // the source label is feasible at the sink
    tl_found = true;
    tl_best_d = 0.0f;
    tl_best_l = 0.0f;
    tl_best_node = source.node;
  }
  std::vector<OracleLabel> init{source};
  std::vector<int> sinks{dst};
  std::vector<int *> path_l;
  std::vector<int> size_of_result_l;
  std::vector<c_constraint<OracleLabel>> C_l{c_constraint<OracleLabel>(budget)};
  RUN_CSPP_CPU<OracleLabel, c_edge>(g, 1, init, sinks, path_l, size_of_result_l, C_l);

  *found = tl_found ? 1 : 0;
  *cost = tl_found ? tl_best_d : std::numeric_limits<float>::infinity();
  *delay = tl_found ? tl_best_l : std::numeric_limits<float>::infinity();
  if (calls) {
    calls[0] = tl_expand_calls;
    calls[1] = tl_dom_calls;
  }
  if (path_len) *path_len = 0;
  if (record && tl_found && path && path_len) {
    int n = 0;
    for (int k = tl_best_node; k >= 0; k = arena[k].parent) ++n;
    *path_len = n;
    if (n <= path_cap) {
      int pos = n - 1;
      for (int k = tl_best_node; k >= 0; k = arena[k].parent) path[pos--] = arena[k].vid;
    }
  }
  tl_arena = nullptr;
}

}  // namespace

extern "C" {

// Builds the reference's Graph<c_edge> (include/graph.hpp:90-134) from CSR,
// inserting each vertex's out-edges in CSR order so the template visits them
// in the same order as the restatement.
void *ref_graph_create(int32_t n, const int64_t *row_ptr, const int32_t *col, const float *len,
                       const float *delay) {
  const int64_t m = row_ptr[n];
  auto *g = new Graph<c_edge>((int)n, (int)m);
  for (int u = 0; u < n; ++u) {
    for (int64_t j = row_ptr[u]; j < row_ptr[u + 1]; ++j) {
      g->e_l[j]->assign((int)j, u, col[j], len[j], delay[j]);
      g->v_l[u].assign(g->e_l[j], g);
    }
  }
  return new RefGraph{g};
}

void ref_graph_destroy(void *h) {
  auto *rg = static_cast<RefGraph *>(h);
  if (!rg) return;
  for (Edge *e : rg->g->e_l) delete e;
  delete rg->g;
  delete rg;
}

// Solves nq queries with `nthreads` host threads (one query per thread at a
// time).  RUN_CSPP_CPU prints timings to stdout; the process's stdout is sent
// to /dev/null for the duration of the call.  When record_paths is set, query
// q's path is written to paths[q * path_stride ...] and path_len[q] is set.
// calls (optional) receives per query {expand_cpu calls, dominate_cpu calls}.
// Timing variant for the CPU baseline: like ref_solve without paths, but
// each query stops after cap_seconds of wall time.  seconds[q] receives the
// query's wall time (at most about cap_seconds) and finished[q] whether it
// ran to completion (cost / delay / found are only meaningful then).
int ref_solve_capped(void *h, int32_t nq, const int32_t *src, const int32_t *dst,
                     const float *budget, int32_t nthreads, double cap_seconds, float *cost,
                     float *delay, int32_t *found, double *seconds, int32_t *finished) {
  auto *rg = static_cast<RefGraph *>(h);
  if (!rg || nq < 0 || !(cap_seconds > 0.0)) return -1;
  if (nthreads < 1) nthreads = 1;
  fflush(stdout);
  std::cout.flush();
  int saved = dup(1);
  int devnull = open("/dev/null", O_WRONLY);
  if (saved >= 0 && devnull >= 0) dup2(devnull, 1);
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      int q = next.fetch_add(1);
      if (q >= nq) break;
      const auto t0 = std::chrono::steady_clock::now();
      tl_capped = true;
      tl_deadline = t0 + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                             std::chrono::duration<double>(cap_seconds));
      finished[q] = 1;
      try {
        run_one(rg->g, src[q], dst[q], budget[q], false, &cost[q], &delay[q], &found[q],
                nullptr, 0, nullptr, nullptr);
      } catch (const DeadlineExceeded &) {
        finished[q] = 0;
        found[q] = 0;
        cost[q] = delay[q] = std::numeric_limits<float>::quiet_NaN();
        tl_arena = nullptr;
      }
      tl_capped = false;
      seconds[q] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
  std::cout.flush();
  fflush(stdout);
  if (saved >= 0 && devnull >= 0) dup2(saved, 1);
  if (saved >= 0) close(saved);
  if (devnull >= 0) close(devnull);
  return 0;
}

int ref_solve(void *h, int32_t nq, const int32_t *src, const int32_t *dst, const float *budget,
              int32_t nthreads, int32_t record_paths, float *cost, float *delay, int32_t *found,
              int32_t *paths, int32_t path_stride, int32_t *path_len, int64_t *calls) {
  auto *rg = static_cast<RefGraph *>(h);
  if (!rg || nq < 0) return -1;
  if (nthreads < 1) nthreads = 1;
  fflush(stdout);
  std::cout.flush();
  int saved = dup(1);
  int devnull = open("/dev/null", O_WRONLY);
  if (saved >= 0 && devnull >= 0) dup2(devnull, 1);

  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      int q = next.fetch_add(1);
      if (q >= nq) break;
      long long c2[2];
      run_one(rg->g, src[q], dst[q], budget[q], record_paths != 0, &cost[q], &delay[q],
              &found[q], paths ? paths + (int64_t)q * path_stride : nullptr, path_stride,
              path_len ? &path_len[q] : nullptr, c2);
      if (calls) {
        calls[2 * (int64_t)q] = c2[0];
        calls[2 * (int64_t)q + 1] = c2[1];
      }
    }
  };
  if (nthreads == 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
  }

  std::cout.flush();
  fflush(stdout);
  if (saved >= 0 && devnull >= 0) {
    dup2(saved, 1);
  }
  if (saved >= 0) close(saved);
  if (devnull >= 0) close(devnull);
  return 0;
}

// ---------------------------------------------------------------------------
// Label variants (include/label.hpp:46-465, include/constraint.hpp:21-187).
//
// The reference selects its label type with the CSP macro; this library is
// built with CSP=1, so the other variants are supplied here as label types
// with the members RUN_CSPP_CPU uses (vid, expand_cpu, dominate_cpu), their
// arithmetic restated from the reference's device code, and with explicit
// specialisations of c_constraint<Label_t> for their constraints.  The
// template itself is instantiated unmodified for each.  As for OracleLabel,
// expand_cpu records the best feasible sink label it creates: for the hop and
// max-cost labels the lexicographically smallest (d, delay, hop, maxcost),
// for the QoS label the smallest d, then the largest bandwidth.

}  // extern "C"

namespace {
thread_local int tl_v_sink = -1;
thread_local bool tl_v_found = false;
thread_local float tl_v_best[4];
thread_local int tl_v_best_node = -1;
thread_local std::vector<ArenaNode> *tl_v_arena = nullptr;
thread_local long long tl_v_calls = 0;
thread_local bool tl_v_capped = false;
thread_local std::chrono::steady_clock::time_point tl_v_deadline;

inline bool lex4_less(const float *a, const float *b, int k) {
  for (int i = 0; i < k; ++i) {
    if (a[i] < b[i]) return true;
    if (a[i] > b[i]) return false;
  }
  return false;
}

inline void v_tick() {
  tl_v_calls++;
  if (tl_v_capped && (tl_v_calls & 1023) == 0 && std::chrono::steady_clock::now() > tl_v_deadline)
    throw DeadlineExceeded{};
}

inline int v_node(int next_v, int parent) {
  if (!tl_v_arena) return -1;
  tl_v_arena->push_back({next_v, parent});
  return (int)tl_v_arena->size() - 1;
}

// Offers a feasible sink label's key (k components, smaller is better).
inline void v_offer(int next_v, const float *key, int k, int node) {
  if (next_v != tl_v_sink) return;
  if (!tl_v_found || lex4_less(key, tl_v_best, k)) {
    tl_v_found = true;
    for (int i = 0; i < k; ++i) tl_v_best[i] = key[i];
    tl_v_best_node = node;
  }
}
}  // namespace

// CSP=2 (include/label.hpp:46-105): (d, delay, hop); constraint delay <= L and hop <= H.
class HopLabel {
 public:
  int vid;
  float d, delay;
  int hop;
  int node;
  HopLabel() {}
  HopLabel(int v) : vid(v), d(0), delay(0), hop(0), node(-1) {}
  template <typename Edge_t>
  void expand_cpu(int next_v, Edge_t e, HopLabel *son);
  static bool dominate_cpu(HopLabel a, HopLabel b) {
    return a.d <= b.d && a.delay <= b.delay && a.hop <= b.hop;
  }
};

// CSP=3 (include/label.hpp:106-168): (d, delay, hop, maxcost = largest arc length).
class MaxLabel {
 public:
  int vid;
  float d, delay;
  int hop;
  float maxcost;
  int node;
  MaxLabel() {}
  MaxLabel(int v) : vid(v), d(0), delay(0), hop(0), maxcost(0), node(-1) {}
  template <typename Edge_t>
  void expand_cpu(int next_v, Edge_t e, MaxLabel *son);
  static bool dominate_cpu(MaxLabel a, MaxLabel b) {
    return a.d <= b.d && a.delay <= b.delay && a.hop <= b.hop && a.maxcost <= b.maxcost;
  }
};

// Network QoS (include/label.hpp:382-464): d adds lengths, delay is the
// bottleneck bandwidth min(delay, arc delay), starting at 21474836;
// constraint bandwidth >= L.
class QosLabel {
 public:
  int vid;
  float d, delay;
  int node;
  QosLabel() {}
  QosLabel(int v) : vid(v), d(0), delay(21474836), node(-1) {}
  template <typename Edge_t>
  void expand_cpu(int next_v, Edge_t e, QosLabel *son);
  static bool dominate_cpu(QosLabel a, QosLabel b) { return a.d <= b.d && a.delay >= b.delay; }
};

// include/constraint.hpp:21-50
template <>
class c_constraint<HopLabel> {
 public:
  float delay_L;
  int hop_L;
  c_constraint() {}
  c_constraint(float d, int h = 100) : delay_L(d), hop_L(h) {}
  bool pass_constraints_check_cpu(const HopLabel &l) {
    return !(l.delay > delay_L || l.hop > hop_L);
  }
};

// include/constraint.hpp:50-80
template <>
class c_constraint<MaxLabel> {
 public:
  float delay_L;
  int hop_L;
  float maxcost_L;
  c_constraint() {}
  c_constraint(float d, int h = 100, float m = 10000) : delay_L(d), hop_L(h), maxcost_L(m) {}
  bool pass_constraints_check_cpu(const MaxLabel &l) {
    return !(l.delay > delay_L || l.hop > hop_L || l.maxcost > maxcost_L);
  }
};

// include/constraint.hpp:162-186
template <>
class c_constraint<QosLabel> {
 public:
  float delay_L;
  c_constraint() {}
  c_constraint(float d) : delay_L(d) {}
  bool pass_constraints_check_cpu(const QosLabel &l) { return !(l.delay < delay_L); }
};

namespace {
thread_local c_constraint<HopLabel> tl_c_hop;
thread_local c_constraint<MaxLabel> tl_c_max;
thread_local c_constraint<QosLabel> tl_c_qos;
}  // namespace

template <typename Edge_t>
void HopLabel::expand_cpu(int next_v, Edge_t e, HopLabel *son) {
  son->vid = next_v;
  son->d = d + e.len;
  son->delay = delay + e.delay;
  son->hop = hop + 1;
  v_tick();
  son->node = v_node(next_v, node);
  if (tl_c_hop.pass_constraints_check_cpu(*son)) {
    const float key[3] = {son->d, son->delay, (float)son->hop};
    v_offer(next_v, key, 3, son->node);
  }
}

template <typename Edge_t>
void MaxLabel::expand_cpu(int next_v, Edge_t e, MaxLabel *son) {
  son->vid = next_v;
  son->d = d + e.len;
  son->delay = delay + e.delay;
  son->hop = hop + 1;
  son->maxcost = std::max(maxcost, (float)e.len);
  v_tick();
  son->node = v_node(next_v, node);
  if (tl_c_max.pass_constraints_check_cpu(*son)) {
    const float key[4] = {son->d, son->delay, (float)son->hop, son->maxcost};
    v_offer(next_v, key, 4, son->node);
  }
}

template <typename Edge_t>
void QosLabel::expand_cpu(int next_v, Edge_t e, QosLabel *son) {
  son->vid = next_v;
  son->d = d + e.len;
  son->delay = std::min(delay, (float)e.delay);
  v_tick();
  son->node = v_node(next_v, node);
  if (tl_c_qos.pass_constraints_check_cpu(*son)) {
    const float key[2] = {son->d, -son->delay};
    v_offer(next_v, key, 2, son->node);
  }
}

namespace {

// One variant query through RUN_CSPP_CPU; returns false when stopped at the cap.
template <typename L>
bool run_variant(Graph<c_edge> *g, int src, int dst, c_constraint<L> C, bool record,
                 const float *src_key, int k, float *best, int32_t *found, int32_t *path,
                 int path_cap, int32_t *path_len, long long *calls) {
  std::vector<ArenaNode> arena;
  tl_v_sink = dst;
  tl_v_found = false;
  tl_v_best_node = -1;
  tl_v_calls = 0;
  tl_v_arena = record ? &arena : nullptr;
  L source(src);
  if (record) {
    source.node = 0;
    arena.push_back({src, -1});
  }
  std::vector<c_constraint<L>> C_l{C};
  // the source label itself answers src == dst when it is feasible
  if (src == dst && C_l[0].pass_constraints_check_cpu(source)) {
    tl_v_found = true;
    for (int i = 0; i < k; ++i) tl_v_best[i] = src_key[i];
    tl_v_best_node = source.node;
  }
  std::vector<L> init{source};
  std::vector<int> sinks{dst};
  std::vector<int *> path_l;
  std::vector<int> size_of_result_l;
  bool done = true;
  try {
    RUN_CSPP_CPU<L, c_edge>(g, 1, init, sinks, path_l, size_of_result_l, C_l);
  } catch (const DeadlineExceeded &) {
    done = false;
  }
  *found = done && tl_v_found ? 1 : 0;
  for (int i = 0; i < k; ++i) best[i] = tl_v_best[i];
  if (calls) *calls = tl_v_calls;
  if (path_len) *path_len = 0;
  if (done && record && tl_v_found && path && path_len) {
    int n = 0;
    for (int q = tl_v_best_node; q >= 0; q = arena[q].parent) ++n;
    *path_len = n;
    if (n <= path_cap) {
      int pos = n - 1;
      for (int q = tl_v_best_node; q >= 0; q = arena[q].parent) path[pos--] = arena[q].vid;
    }
  }
  tl_v_arena = nullptr;
  return done;
}

}  // namespace

extern "C" {

// Label-variant queries through RUN_CSPP_CPU, one query per thread.
// kind 2: hop-constrained (limits delay_L[q], hop_L[q]); kind 3: max-cost
// (delay_L, hop_L, max_L); kind 6: QoS (delay_L[q] = minimum bandwidth).
// out[q * 4 + i] receives the best label's (d, delay, hop, maxcost) (QoS:
// (d, bandwidth)).  A query still running after cap_seconds (0 = no cap)
// stops with finished[q] = 0.
int ref_solve_variant(void *h, int32_t kind, int32_t nq, const int32_t *src, const int32_t *dst,
                      const float *delay_L, const int32_t *hop_L, const float *max_L,
                      int32_t nthreads, double cap_seconds, float *out, int32_t *found,
                      int32_t *finished, int32_t *paths, int32_t path_stride, int32_t *path_len,
                      int64_t *calls) {
  auto *rg = static_cast<RefGraph *>(h);
  if (!rg || nq < 0 || (kind != 2 && kind != 3 && kind != 6)) return -1;
  if (nthreads < 1) nthreads = 1;
  fflush(stdout);
  std::cout.flush();
  int saved = dup(1);
  int devnull = open("/dev/null", O_WRONLY);
  if (saved >= 0 && devnull >= 0) dup2(devnull, 1);
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int q = next.fetch_add(1);
      if (q >= nq) break;
      tl_v_capped = cap_seconds > 0.0;
      tl_v_deadline = std::chrono::steady_clock::now() +
                      std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                          std::chrono::duration<double>(cap_seconds > 0.0 ? cap_seconds : 1.0));
      float best[4] = {0, 0, 0, 0};
      int32_t *pq = paths ? paths + (int64_t)q * path_stride : nullptr;
      int32_t *pl = path_len ? &path_len[q] : nullptr;
      long long nc = 0;
      bool done;
      if (kind == 2) {
        tl_c_hop = c_constraint<HopLabel>(delay_L[q], hop_L[q]);
        const float k0[3] = {0, 0, 0};
        done = run_variant<HopLabel>(rg->g, src[q], dst[q], tl_c_hop, paths != nullptr, k0, 3,
                                     best, &found[q], pq, path_stride, pl, &nc);
      } else if (kind == 3) {
        tl_c_max = c_constraint<MaxLabel>(delay_L[q], hop_L[q], max_L[q]);
        const float k0[4] = {0, 0, 0, 0};
        done = run_variant<MaxLabel>(rg->g, src[q], dst[q], tl_c_max, paths != nullptr, k0, 4,
                                     best, &found[q], pq, path_stride, pl, &nc);
      } else {
        tl_c_qos = c_constraint<QosLabel>(delay_L[q]);
        const float k0[2] = {0, -21474836.0f};
        done = run_variant<QosLabel>(rg->g, src[q], dst[q], tl_c_qos, paths != nullptr, k0, 2,
                                     best, &found[q], pq, path_stride, pl, &nc);
        best[1] = -best[1];
      }
      tl_v_capped = false;
      finished[q] = done ? 1 : 0;
      for (int i = 0; i < 4; ++i) out[(int64_t)q * 4 + i] = best[i];
      if (calls) calls[q] = nc;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
  std::cout.flush();
  fflush(stdout);
  if (saved >= 0 && devnull >= 0) dup2(saved, 1);
  if (saved >= 0) close(saved);
  if (devnull >= 0) close(devnull);
  return 0;
}

}  // extern "C"

// The seeded workload generator (vine_b200/csrc/workloads.cpp, compiled into
// this library by oracle/Makefile) reports errors through vine::set_error;
// this library keeps the text for ref_last_error().  With the generator in
// here, the CPU reference timing builds its input without loading the GPU
// engine's library.
namespace vine {
thread_local std::string g_ref_last_error;
void set_error(const std::string &msg) { g_ref_last_error = msg; }
}  // namespace vine

extern "C" const char *ref_last_error(void) { return vine::g_ref_last_error.c_str(); }
