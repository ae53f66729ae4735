// Autotuner for the batch engine: picks the bucket-table size, the bucket
// granularity (initial width; the far band's width in buckets) and the block
// shape by timing candidates on a sample of queries with CUDA events.
// The reference fixes these at compile time (BLOCK_SIZE, TABLE_SIZE, VSIZE,
// algorithm/bucket.cuh:9-13; SearchSpace, algorithm/dominance.cuh:11) and
// sizes its split from free memory (algorithm/cspp.cuh:43-47, 136-138).
// Results are cached in a text file keyed by the graph fingerprint and the
// search mode, so a graph is tuned once.

#include "engine_host.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

using namespace vine;

namespace {

struct Candidate {
  int block_threads, table_log2, split;
  float width_mult;
  int band_mult;
};

std::string cache_key(const vine_graph *g, const vine_config &c) {
  std::ostringstream ss;
  ss << "v2 " << std::hex << g->fingerprint << std::dec << " m" << c.mode << " b" << c.use_bounds << " p"
     << c.policy;
  return ss.str();
}

bool cache_lookup(const char *path, const std::string &key, Candidate *out) {
  if (!path) return false;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    if (line.compare(0, key.size(), key) != 0 || line.size() <= key.size() || line[key.size()] != '|')
      continue;
    Candidate c;
    if (std::sscanf(line.c_str() + key.size() + 1, "%d %d %d %f %d", &c.block_threads,
                    &c.table_log2, &c.split, &c.width_mult, &c.band_mult) == 5) {
      *out = c;
      return true;
    }
  }
  return false;
}

void cache_store(const char *path, const std::string &key, const Candidate &c) {
  if (!path) return;
  std::ofstream out(path, std::ios::app);
  out << key << '|' << c.block_threads << ' ' << c.table_log2 << ' ' << c.split << ' '
      << c.width_mult << ' ' << c.band_mult << '\n';
}

void apply(const Candidate &k, const vine_graph *g, vine_config *c) {
  c->block_threads = k.block_threads;
  c->table_log2 = k.table_log2;
  c->split_threshold = k.split;
  c->bucket_width = k.width_mult * g->mean_len;
  c->band_mult = k.band_mult;
}

}  // namespace

extern "C" int vine_autotune(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
                             const float *budget, const vine_config *base,
                             const char *cache_path, vine_config *best) {
  if (!g || nq <= 0 || !src || !dst || !budget || !best)
    return fail(VINE_ERR_INVALID, "bad arguments");
  vine_config b0;
  if (base) b0 = *base;
  else vine_config_default(&b0);
  b0.engine = VINE_ENGINE_BATCH;
  b0.trace = 0;
  const std::string key = cache_key(g, b0);
  Candidate hit;
  if (cache_lookup(cache_path, key, &hit)) {
    *best = b0;
    apply(hit, g, best);
    return VINE_OK;
  }
  VINE_CUDA_TRY(cudaSetDevice(g->device));
  int32_t *d_src = nullptr, *d_dst = nullptr, *d_found = nullptr, *d_status = nullptr;
  float *d_budget = nullptr, *d_cost = nullptr, *d_delay = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_src);
    cudaFree(d_dst);
    cudaFree(d_found);
    cudaFree(d_status);
    cudaFree(d_budget);
    cudaFree(d_cost);
    cudaFree(d_delay);
  };
  if (cudaMalloc(&d_src, 4 * (size_t)nq) != cudaSuccess || cudaMalloc(&d_dst, 4 * (size_t)nq) != cudaSuccess ||
      cudaMalloc(&d_found, 4 * (size_t)nq) != cudaSuccess || cudaMalloc(&d_status, 4 * (size_t)nq) != cudaSuccess ||
      cudaMalloc(&d_budget, 4 * (size_t)nq) != cudaSuccess || cudaMalloc(&d_cost, 4 * (size_t)nq) != cudaSuccess ||
      cudaMalloc(&d_delay, 4 * (size_t)nq) != cudaSuccess) {
    cleanup();
    return fail(VINE_ERR_CUDA, "autotune allocation failed");
  }
  cudaMemcpy(d_src, src, 4 * (size_t)nq, cudaMemcpyHostToDevice);
  cudaMemcpy(d_dst, dst, 4 * (size_t)nq, cudaMemcpyHostToDevice);
  cudaMemcpy(d_budget, budget, 4 * (size_t)nq, cudaMemcpyHostToDevice);
  // one CTA of 512 threads per SM (smaller blocks co-resident on an SM
  // slow each other down), table of 2^12 or 2^13 slots, initial width and
  // band width around the values that measured best on road graphs
  std::vector<Candidate> cands;
  for (int tl : {12, 13})
    for (float wm : {0.2f, 0.3f, 0.5f})
      for (int bm : {8, 16}) cands.push_back({512, tl, 0, wm, bm});
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  Candidate best_c = cands[0];
  int rc = VINE_OK;
  for (const Candidate &k : cands) {
    vine_config c = b0;
    apply(k, g, &c);
    Resolved r;
    if (resolve_config(g, &c, &r) != VINE_OK) continue;  // does not fit: skip
    DeviceOutputs o;
    o.cost = d_cost;
    o.delay = d_delay;
    o.found = d_found;
    o.status = d_status;
    float ms_total = 0.0f;
    bool ok = true;
    for (int rep = 0; rep < 2 && ok; ++rep) {
      cudaEventRecord(e0, g->stream);
      if (batch_run(g, r, nq, d_src, d_dst, d_budget, o, g->stream, nullptr) != VINE_OK) ok = false;
      cudaEventRecord(e1, g->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(VINE_ERR_CUDA, "autotune run failed");
        ok = false;
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep == 1) ms_total = ms;  // first run warms the workspace
    }
    if (rc != VINE_OK) break;
    if (!ok) continue;
    std::vector<int32_t> st((size_t)nq);
    cudaMemcpy(st.data(), d_status, 4 * (size_t)nq, cudaMemcpyDeviceToHost);
    bool all_ok = true;
    for (int32_t v : st) all_ok = all_ok && v == VINE_OK;
    if (all_ok && ms_total < best_ms) {
      best_ms = ms_total;
      best_c = k;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cleanup();
  if (rc != VINE_OK) return rc;
  if (best_ms >= 1e30f) return fail(VINE_ERR_CAPACITY, "no autotune candidate solved the sample");
  *best = b0;
  apply(best_c, g, best);
  cache_store(cache_path, key, best_c);
  return VINE_OK;
}
