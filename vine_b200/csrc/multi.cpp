// Query sharding over several GPUs (one graph handle per device).
//
// Queries are independent, so a batch splits across devices with no
// exchange between them: the graph is replicated (one vine_graph per
// device), each device solves its share with vine_solve on its own host
// thread, and the results are scattered back into the caller's arrays in
// query order.  The share of each device is picked by longest-processing-
// time-first: queries in decreasing budget (the batch engine's own proxy for
// a query's cost) each go to the device with the least budget assigned so
// far, so every device gets a similar mix of heavy and light queries.

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vine.h"
#include "common.h"

using namespace vine;

namespace {
constexpr int32_t kUnset = INT32_MIN;  // per-query status not written by the call
}

extern "C" {

int vine_solve_multi(vine_graph **graphs, int32_t ngraphs, int32_t nq, const int32_t *src,
                     const int32_t *dst, const float *budget, const vine_config *cfg,
                     vine_results *out) {
  if (!graphs || ngraphs < 1 || nq < 0 || !out) return fail(VINE_ERR_INVALID, "bad arguments");
  for (int32_t k = 0; k < ngraphs; ++k)
    if (!graphs[k]) return fail(VINE_ERR_INVALID, "null graph handle");
  if (nq == 0) {
    if (out->path_offsets) out->path_offsets[0] = 0;
    return VINE_OK;
  }
  if (!src || !dst || !budget || !out->cost || !out->delay || !out->found)
    return fail(VINE_ERR_INVALID, "missing input/output buffers");
  // longest-processing-time-first assignment by budget
  std::vector<int32_t> order((size_t)nq);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    const float fa = budget[a] == budget[a] ? budget[a] : -1.0f;
    const float fb = budget[b] == budget[b] ? budget[b] : -1.0f;
    return fa > fb;
  });
  std::vector<std::vector<int32_t>> part((size_t)ngraphs);
  std::vector<double> load((size_t)ngraphs, 0.0);
  for (int32_t q : order) {
    const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
    part[k].push_back(q);
    load[k] += std::max(1.0, (double)(budget[q] == budget[q] ? budget[q] : 0.0f));
  }
  for (auto &p : part) std::sort(p.begin(), p.end());  // each share in query order

  const bool want_paths = out->path_offsets != nullptr;
  const bool want_pareto = out->pareto_d && out->pareto_delay && out->pareto_n && out->pareto_stride > 0;
  const int32_t stride = want_pareto ? out->pareto_stride : 0;
  struct Share {
    std::vector<int32_t> s, t;
    std::vector<float> b, cost, delay, pd, pl;
    std::vector<int32_t> found, status, pn, path;
    std::vector<int64_t> off, stats;
    int rc = VINE_OK, retried = 0;
    std::string err;
  };
  std::vector<Share> sh((size_t)ngraphs);
  std::vector<std::thread> th;
  for (int32_t k = 0; k < ngraphs; ++k) {
    th.emplace_back([&, k]() {
      Share &x = sh[(size_t)k];
      const auto &idx = part[(size_t)k];
      const int32_t n = (int32_t)idx.size();
      if (n == 0) return;
      x.s.resize(n);
      x.t.resize(n);
      x.b.resize(n);
      for (int32_t i = 0; i < n; ++i) {
        x.s[i] = src[idx[i]];
        x.t[i] = dst[idx[i]];
        x.b[i] = budget[idx[i]];
      }
      // a call that fails before it writes the per-query outputs leaves
      // these: not found, and (below) the call's own status
      x.cost.assign(n, INFINITY);
      x.delay.assign(n, INFINITY);
      x.found.assign(n, 0);
      x.status.assign(n, kUnset);
      vine_results r = {};
      r.cost = x.cost.data();
      r.delay = x.delay.data();
      r.found = x.found.data();
      r.status = x.status.data();
      if (out->stats) {
        x.stats.resize((size_t)n * VINE_STAT_COUNT);
        r.stats = x.stats.data();
      }
      if (want_pareto) {
        x.pd.resize((size_t)n * stride);
        x.pl.resize((size_t)n * stride);
        x.pn.resize(n);
        r.pareto_d = x.pd.data();
        r.pareto_delay = x.pl.data();
        r.pareto_n = x.pn.data();
        r.pareto_stride = stride;
      }
      int64_t cap = (int64_t)n * 256 + 4096;
      for (int attempt = 0; attempt < 2; ++attempt) {
        if (want_paths) {
          x.off.assign((size_t)n + 1, 0);
          x.path.resize((size_t)cap);
          r.path_offsets = x.off.data();
          r.path = x.path.data();
          r.path_capacity = cap;
        }
        x.rc = vine_solve(graphs[k], n, x.s.data(), x.t.data(), x.b.data(), cfg, &r);
        if (!(want_paths && x.rc == VINE_ERR_CAPACITY && x.off[n] > cap)) break;
        cap = x.off[n];  // the library reported the size the paths need
      }
      x.retried = r.retried;
      if (x.rc != VINE_OK) x.err = vine_last_error();
      for (int32_t &st : x.status)
        if (st == kUnset) st = x.rc;
    });
  }
  for (auto &t : th) t.join();

  int rc = VINE_OK;
  std::string err;
  std::vector<int64_t> plen(want_paths ? (size_t)nq : 0, 0);
  std::vector<const int32_t *> psrc(want_paths ? (size_t)nq : 0, nullptr);
  out->retried = 0;
  for (int32_t k = 0; k < ngraphs; ++k) {
    const Share &x = sh[(size_t)k];
    const auto &idx = part[(size_t)k];
    if (x.rc != VINE_OK && rc == VINE_OK) {
      rc = x.rc;
      err = "device share " + std::to_string(k) + ": " + x.err;
    }
    out->retried += x.retried;
    for (size_t i = 0; i < idx.size(); ++i) {
      const int32_t q = idx[i];
      out->cost[q] = x.cost[i];
      out->delay[q] = x.delay[i];
      out->found[q] = x.found[i];
      if (out->status) out->status[q] = x.status[i];
      if (out->stats)
        std::memcpy(out->stats + (size_t)q * VINE_STAT_COUNT, x.stats.data() + i * VINE_STAT_COUNT,
                    sizeof(int64_t) * VINE_STAT_COUNT);
      if (want_pareto) {
        out->pareto_n[q] = x.pn[i];
        std::memcpy(out->pareto_d + (size_t)q * stride, x.pd.data() + i * stride, sizeof(float) * stride);
        std::memcpy(out->pareto_delay + (size_t)q * stride, x.pl.data() + i * stride, sizeof(float) * stride);
      }
      if (want_paths && !x.off.empty()) {
        plen[q] = x.off[i + 1] - x.off[i];
        psrc[q] = x.path.data() + x.off[i];
      }
    }
  }
  if (want_paths) {
    int64_t run = 0;
    for (int32_t q = 0; q < nq; ++q) {
      out->path_offsets[q] = run;
      run += plen[q];
    }
    out->path_offsets[nq] = run;
    if (run > out->path_capacity || out->path == nullptr) {
      if (rc == VINE_OK) {
        rc = VINE_ERR_CAPACITY;
        err = "path buffer too small (need " + std::to_string(run) + ")";
      }
    } else {
      for (int32_t q = 0; q < nq; ++q)
        if (plen[q]) std::memcpy(out->path + out->path_offsets[q], psrc[q], sizeof(int32_t) * plen[q]);
    }
  }
  if (rc != VINE_OK) set_error(err);
  return rc;
}

}  // extern "C"
