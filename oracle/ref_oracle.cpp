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
