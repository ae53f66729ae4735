// Multi-core CPU engine: the reference's OpenMP solver RUN_CSPP_OMP
// (algorithm/cspp_cpu.hpp:127-213) with its data races removed.
//
// The reference expands a round's frontier in parallel while every thread
// reads, erases from and appends to the shared per-vertex dominance lists
// (cspp_cpu.hpp:171-192: iteration races with erase / push_back in other
// threads), and prints the labels of vertex N-1 instead of the sink
// (:203-205).  Here one round has two phases separated by a barrier:
//
//   1. expand   thread t expands frontier labels t, t+T, ...: children that
//               pass the constraint go to outbox[t][owner(v)], owner(v) =
//               v mod T (no shared writes);
//   2. merge    thread o owns the vertices with owner o: it takes the
//               children addressed to it (outboxes 0..T-1 in order) and
//               applies the reference's per-label rule against v's list --
//               dropped when a stored label dominates it, stored labels it
//               dominates are erased, otherwise appended to v's list and to
//               the next frontier (cspp_cpu.hpp:170-193).
//
// Every list is touched by its owner only, so the run is race-free and the
// result does not depend on the thread count: the sink list ends as the set
// of non-dominated feasible sink labels.
//
// One change of the reference's rule: a label erased from its vertex's list
// (dominated by a later arrival) is marked dead and not expanded when its
// round comes.  The reference expands it all the same, and how many such
// labels a round holds depends on the order children arrive in; on a 100x100
// grid one thread (breadth-first order) expanded some 20x more labels than
// two.  Skipping them is exact: the dominating label is in the frontier too,
// and its child over each arc dominates the dead label's child over it.  Labels carry their parent (a
// (thread, index) arena reference), so the answer's path is returned too.
// The answer is the lexicographically smallest (cost, delay) label of the
// sink's list, as for the GPU engines.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <unistd.h>

#include "../../include/vine.h"
#include "common.h"

namespace vine {
namespace {

// A label of the host engine; parent = (arena << 40) | index, -1 for the source.
struct HLabel {
  int32_t vid;
  float d;
  float dl;
  int64_t ref;  // this label's own arena reference
};

inline bool hdom(const HLabel &a, const HLabel &b) {  // include/label.hpp:244-246
  return a.d <= b.d && a.dl <= b.dl;
}

struct Node {
  int32_t vid;
  int64_t parent;
  bool dead;  // erased from its vertex's list: dominated, not expanded
};

// Runs fn(t) on T threads and waits for all of them (threads kept between rounds).
class RoundPool {
 public:
  explicit RoundPool(int T) : T_(T) {
    for (int t = 1; t < T_; ++t) threads_.emplace_back([this, t] { loop(t); });
  }
  ~RoundPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto &th : threads_) th.join();
  }
  void run(const std::function<void(int)> &fn) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      pending_ = T_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }

 private:
  void loop(int t) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)> *fn;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        fn = fn_;
      }
      (*fn)(t);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }
  int T_;
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)> *fn_ = nullptr;
  int pending_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

struct HostGraph {
  int32_t n;
  const int64_t *row;
  const int32_t *col;
  const float *len;
  const float *dly;
};

struct QueryOut {
  bool found = false;
  float cost = INFINITY, delay = INFINITY;
  std::vector<int32_t> path;
  std::vector<std::pair<float, float>> pareto;
};

// One query with T threads (pool may be null when T == 1).  Returns
// VINE_ERR_CAPACITY, with no answer, once the query holds more than
// max_labels labels (checked after every round), else VINE_OK.
int solve_one(const HostGraph &g, int32_t s, int32_t t, float L, int T, RoundPool *pool,
              int64_t max_labels, QueryOut *out) {
  const int32_t n = g.n;
  std::vector<std::vector<HLabel>> lists((size_t)n);
  std::vector<std::vector<Node>> arena((size_t)T);
  std::vector<HLabel> frontier, next;
  auto node = [&arena](int64_t r) -> Node & {
    return arena[(size_t)(r >> 40)][(size_t)(r & ((int64_t(1) << 40) - 1))];
  };
  // outbox[producer][owner]: children with their parent references
  std::vector<std::vector<std::vector<std::pair<HLabel, int64_t>>>> outbox(
      (size_t)T, std::vector<std::vector<std::pair<HLabel, int64_t>>>((size_t)T));
  std::vector<std::vector<HLabel>> next_part((size_t)T);

  // every label at v lives in the arena of v's owner, which alone writes it
  const int so = (int)(s % T);
  arena[(size_t)so].push_back({s, -1, false});
  HLabel src{s, 0.0f, 0.0f, (int64_t)so << 40};
  frontier.push_back(src);
  // the source label is stored at s, as a label of the search (a later
  // label at s with cost and delay >= 0 is dominated by it)
  lists[(size_t)s].push_back(src);
  std::function<void(int)> expand = [&](int th) {
    for (auto &box : outbox[(size_t)th]) box.clear();
    for (size_t i = (size_t)th; i < frontier.size(); i += (size_t)T) {
      const HLabel &f = frontier[i];
      if (node(f.ref).dead) continue;  // dominated since it joined the frontier
      for (int64_t j = g.row[f.vid]; j < g.row[f.vid + 1]; ++j) {
        const int32_t v = g.col[j];
        HLabel c{v, f.d + g.len[j], f.dl + g.dly[j], -1};  // include/label.hpp:214-222
        if (c.dl > L) continue;                            // include/constraint.hpp:99-101
        outbox[(size_t)th][(size_t)(v % T)].push_back({c, f.ref});
      }
    }
  };
  std::function<void(int)> merge = [&](int o) {
    next_part[(size_t)o].clear();
    for (int p = 0; p < T; ++p) {
      for (auto &item : outbox[(size_t)p][(size_t)o]) {
        HLabel c = item.first;
        auto &lst = lists[(size_t)c.vid];
        bool dominated = false;
        for (auto it = lst.begin(); it != lst.end();) {
          if (hdom(*it, c)) {
            dominated = true;
            break;
          }
          if (hdom(c, *it)) {
            node(it->ref).dead = true;  // v's owner is this thread: its own arena
            it = lst.erase(it);
          } else {
            ++it;
          }
        }
        if (dominated) continue;
        c.ref = ((int64_t)o << 40) | (int64_t)arena[(size_t)o].size();
        arena[(size_t)o].push_back({c.vid, item.second, false});
        lst.push_back(c);
        next_part[(size_t)o].push_back(c);
      }
    }
  };
  while (!frontier.empty()) {
    if (pool) {
      pool->run(expand);
      pool->run(merge);
    } else {
      expand(0);
      merge(0);
    }
    next.clear();
    for (int o = 0; o < T; ++o) next.insert(next.end(), next_part[(size_t)o].begin(), next_part[(size_t)o].end());
    frontier.swap(next);
    int64_t held = 0;
    for (const auto &a : arena) held += (int64_t)a.size();
    if (held > max_labels) return VINE_ERR_CAPACITY;
  }
  // answer: lexicographically smallest (cost, delay) of the sink's list
  const auto &sl = lists[(size_t)t];
  const HLabel *best = nullptr;
  for (const HLabel &l : sl) {
    if (l.dl > L) continue;  // only the source label can be stored unchecked (L < 0)
    out->pareto.push_back({l.d, l.dl});
    if (!best || l.d < best->d || (l.d == best->d && l.dl < best->dl)) best = &l;
  }
  std::sort(out->pareto.begin(), out->pareto.end());
  if (!best) return VINE_OK;
  out->found = true;
  out->cost = best->d;
  out->delay = best->dl;
  for (int64_t r = best->ref; r >= 0;) {
    const Node &nd = arena[(size_t)(r >> 40)][(size_t)(r & ((int64_t(1) << 40) - 1))];
    out->path.push_back(nd.vid);
    r = nd.parent;
  }
  std::reverse(out->path.begin(), out->path.end());
  return VINE_OK;
}

// Labels one query may hold: a quarter of physical memory shared by the
// queries in flight, at about 96 bytes a label (arena node, list entry,
// frontier and outbox copies).  VINE_HOST_MAX_LABELS overrides it.
int64_t label_cap(int in_flight) {
  if (const char *e = std::getenv("VINE_HOST_MAX_LABELS")) {
    const long long v = std::atoll(e);
    if (v > 0) return (int64_t)v;
  }
  const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
  const double bytes = pages > 0 && page > 0 ? (double)pages * (double)page : 16e9;
  return std::max<int64_t>(int64_t(1) << 20, (int64_t)(bytes / 4.0 / std::max(1, in_flight) / 96.0));
}

}  // namespace
}  // namespace vine

using namespace vine;

extern "C" {

int vine_solve_host(int32_t n, int64_t m, const int64_t *row_ptr, const int32_t *col,
                    const float *len, const float *delay, int32_t nq, const int32_t *src,
                    const int32_t *dst, const float *budget, int32_t nthreads,
                    int32_t across_queries, vine_results *out) {
  if (n < 1 || m < 0 || !row_ptr || (m > 0 && (!col || !len || !delay)) || nq < 0 || !out)
    return fail(VINE_ERR_INVALID, "bad arguments");
  if (row_ptr[0] != 0 || row_ptr[n] != m) return fail(VINE_ERR_INVALID, "row_ptr must run 0..m");
  for (int64_t j = 0; j < m; ++j)
    if (col[j] < 0 || col[j] >= n || !(len[j] >= 0.0f) || !(delay[j] >= 0.0f))
      return fail(VINE_ERR_INVALID, "bad arc");
  if (nq > 0 && (!src || !dst || !budget || !out->cost || !out->delay || !out->found))
    return fail(VINE_ERR_INVALID, "missing input/output buffers");
  int T = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  const HostGraph g{n, row_ptr, col, len, delay};
  std::vector<QueryOut> res((size_t)nq);
  std::vector<int32_t> status((size_t)nq, VINE_OK);
  const int64_t cap = label_cap(across_queries ? std::min<int>(T, std::max(nq, 1)) : 1);
  auto one = [&](int32_t q, int threads, RoundPool *pool) {
    const int32_t s = src[q], t = dst[q];
    const float L = budget[q];
    if (s < 0 || s >= n || t < 0 || t >= n || std::isnan(L)) {
      status[(size_t)q] = VINE_ERR_INVALID;
      return;
    }
    if (0.0f > L) return;  // even the source label violates the budget
    const int rc = solve_one(g, s, t, L, threads, pool, cap, &res[(size_t)q]);
    if (rc != VINE_OK) {
      res[(size_t)q] = QueryOut();  // no partial answer
      status[(size_t)q] = rc;
    }
  };
  if (across_queries) {
    // one query per thread at a time, each expanded by that thread alone
    std::atomic<int32_t> next{0};
    std::vector<std::thread> th;
    for (int k = 0; k < std::min<int>(T, std::max(nq, 1)); ++k)
      th.emplace_back([&] {
        for (int32_t q; (q = next.fetch_add(1)) < nq;) one(q, 1, nullptr);
      });
    for (auto &x : th) x.join();
  } else {
    RoundPool pool(T);
    for (int32_t q = 0; q < nq; ++q) one(q, T, T > 1 ? &pool : nullptr);
  }
  int rc = VINE_OK;
  int64_t run = 0;
  int32_t n_invalid = 0, n_capacity = 0;
  for (int32_t q = 0; q < nq; ++q) {
    n_invalid += status[(size_t)q] == VINE_ERR_INVALID;
    n_capacity += status[(size_t)q] == VINE_ERR_CAPACITY;
  }
  if (n_invalid || n_capacity)
    set_error(std::to_string(n_invalid) + " of " + std::to_string(nq) + " queries are invalid, " +
              std::to_string(n_capacity) + " exceeded the label cap of " + std::to_string(cap));
  for (int32_t q = 0; q < nq; ++q) {
    const QueryOut &r = res[(size_t)q];
    out->cost[q] = r.found ? r.cost : INFINITY;
    out->delay[q] = r.found ? r.delay : INFINITY;
    out->found[q] = r.found ? 1 : 0;
    if (out->status) out->status[q] = status[(size_t)q];
    if (status[(size_t)q] != VINE_OK && rc == VINE_OK) rc = status[(size_t)q];
    if (out->pareto_n) {
      out->pareto_n[q] = (int32_t)r.pareto.size();
      for (int32_t k = 0; k < std::min<int32_t>((int32_t)r.pareto.size(), out->pareto_stride); ++k) {
        out->pareto_d[(size_t)q * out->pareto_stride + k] = r.pareto[(size_t)k].first;
        out->pareto_delay[(size_t)q * out->pareto_stride + k] = r.pareto[(size_t)k].second;
      }
    }
    if (out->path_offsets) {
      out->path_offsets[q] = run;
      if (out->path && run + (int64_t)r.path.size() <= out->path_capacity)
        std::memcpy(out->path + run, r.path.data(), sizeof(int32_t) * r.path.size());
      run += (int64_t)r.path.size();
    }
  }
  if (out->path_offsets) {
    out->path_offsets[nq] = run;
    if (run > out->path_capacity && rc == VINE_OK)
      rc = fail(VINE_ERR_CAPACITY, "path buffer too small (need " + std::to_string(run) + ")");
  }
  return rc;
}

}  // extern "C"
