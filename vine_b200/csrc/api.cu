// C ABI of the engine: graph upload, configuration, solve entry points.
//
// vine_graph_create replaces Graph::adj_to_csr + Graph::make_gpu_graph
// (include/graph.hpp:136-195): the CSR is uploaded as SoA arrays with the two
// arc weights interleaved ({len, delay} per arc, one 8-byte load) and without
// the reference's edge-id indirection (el_d[_eid_col_d[l]],
// algorithm/bucket.cuh:73), plus a reverse CSR for the lower-bound searches.
// vine_solve replaces cspp::solve -> RUN_CSPP (algorithm/cspp.hpp:48-53,
// algorithm/cspp.cuh:69-325) and, unlike it, returns cost, delay, path and
// status per query.

#include "engine_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace vine {

thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

int batch_slots(const vine_graph *g, const vine_config &c, int round_cap, int *slots);

namespace {

uint64_t fnv1a(uint64_t h, const void *data, size_t bytes) {
  const unsigned char *p = static_cast<const unsigned char *>(data);
  for (size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Device buffers for one host-buffer solve call.
struct IoBuffers {
  int32_t *src = nullptr, *dst = nullptr, *found = nullptr, *status = nullptr,
          *pareto_n = nullptr;
  float *budget = nullptr, *cost = nullptr, *delay = nullptr, *pareto_d = nullptr,
        *pareto_dl = nullptr;
  int64_t *stats = nullptr, *offsets = nullptr;
  int32_t *path = nullptr;
  void release() {
    cudaFree(src);
    cudaFree(dst);
    cudaFree(found);
    cudaFree(status);
    cudaFree(pareto_n);
    cudaFree(budget);
    cudaFree(cost);
    cudaFree(delay);
    cudaFree(pareto_d);
    cudaFree(pareto_dl);
    cudaFree(stats);
    cudaFree(offsets);
    cudaFree(path);
    *this = IoBuffers();
  }
};

// vine_solve's device buffers, kept with the graph handle between calls
// (allocating and freeing them on every call cost a device-wide sync each).
// They follow the calls' needs: the statistics and Pareto buffers exist only
// while calls ask for them, and a call that needs less than a quarter of the
// held capacity gets right-sized buffers, so one large call does not keep
// its memory for the handle's whole life.
struct IoCache {
  IoBuffers b;
  int64_t cap_q = 0;
  bool stats = false;
  size_t stride = 0;
  int64_t path_cap = 0;
};

IoCache &io_cache(vine_graph *g) {
  if (!g->io_cache) g->io_cache = new IoCache();
  return *static_cast<IoCache *>(g->io_cache);
}

int io_reserve(IoCache &c, int32_t k, bool stats, size_t stride) {
  const size_t cap = std::max<size_t>((size_t)k, 1024);
  if ((size_t)k <= (size_t)c.cap_q && 4 * cap > (size_t)c.cap_q && stats == c.stats &&
      stride == c.stride)
    return VINE_OK;
  c.b.release();
  c.cap_q = 0;
  c.path_cap = 0;
  const bool want_stats = stats;
  const size_t want_stride = stride;
  IoBuffers &io = c.b;
  if (cudaMalloc(&io.src, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&io.dst, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&io.budget, sizeof(float) * cap) != cudaSuccess ||
      cudaMalloc(&io.cost, sizeof(float) * cap) != cudaSuccess ||
      cudaMalloc(&io.delay, sizeof(float) * cap) != cudaSuccess ||
      cudaMalloc(&io.found, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&io.status, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&io.offsets, sizeof(int64_t) * (cap + 1)) != cudaSuccess ||
      (want_stats && cudaMalloc(&io.stats, sizeof(int64_t) * VINE_STAT_COUNT * cap) != cudaSuccess) ||
      (want_stride > 0 && (cudaMalloc(&io.pareto_d, sizeof(float) * want_stride * cap) != cudaSuccess ||
                           cudaMalloc(&io.pareto_dl, sizeof(float) * want_stride * cap) != cudaSuccess ||
                           cudaMalloc(&io.pareto_n, sizeof(int32_t) * cap) != cudaSuccess))) {
    c.b.release();
    return fail(VINE_ERR_CUDA, "result allocation failed");
  }
  c.cap_q = (int64_t)cap;
  c.stats = want_stats;
  c.stride = want_stride;
  return VINE_OK;
}

int io_reserve_path(IoCache &c, int64_t n) {
  if (n <= c.path_cap && 4 * (n + 1024) > c.path_cap) return VINE_OK;
  cudaFree(c.b.path);
  c.b.path = nullptr;
  c.path_cap = 0;
  const int64_t cap = n + n / 4 + 1024;
  if (cudaMalloc(&c.b.path, sizeof(int32_t) * (size_t)cap) != cudaSuccess)
    return fail(VINE_ERR_CUDA, "path allocation failed");
  c.path_cap = cap;
  return VINE_OK;
}

}  // namespace

int resolve_config(const vine_graph *g, const vine_config *in, Resolved *out) {
  vine_config c;
  if (in) {
    c = *in;
  } else {
    vine_config_default(&c);
  }
  if (c.engine != VINE_ENGINE_BATCH && c.engine != VINE_ENGINE_PLAIN)
    return fail(VINE_ERR_INVALID, "unknown engine");
  if (c.mode != VINE_MODE_OPTIMAL && c.mode != VINE_MODE_PARETO)
    return fail(VINE_ERR_INVALID, "unknown mode");
  if (c.policy < VINE_POLICY_FIXED || c.policy > VINE_POLICY_MLP)
    return fail(VINE_ERR_INVALID, "unknown policy");
  if (c.policy == VINE_POLICY_MLP && c.mlp == nullptr)
    return fail(VINE_ERR_INVALID, "VINE_POLICY_MLP needs cfg.mlp");
  if (c.use_bounds && c.mode == VINE_MODE_PARETO)
    return fail(VINE_ERR_INVALID, "lower bounds prune the Pareto set; use VINE_MODE_OPTIMAL");
  if (c.use_bounds && !g->integral)
    return fail(VINE_ERR_INVALID, "lower bounds need integral weights below 2^24");
  if (c.block_threads == 0) c.block_threads = 512;
  if (c.block_threads < 64 || c.block_threads > 512 || c.block_threads % 32)
    return fail(VINE_ERR_INVALID, "block_threads must be a multiple of 32 in [64, 512]");
  if (c.table_log2 == 0) c.table_log2 = 11;
  if (c.table_log2 < 6 || c.table_log2 > 13) return fail(VINE_ERR_INVALID, "table_log2 in [6, 13]");
  if (c.spill_log2 == 0) c.spill_log2 = 16;
  if (c.spill_log2 < 8 || c.spill_log2 > 24) return fail(VINE_ERR_INVALID, "spill_log2 in [8, 24]");
  if (!(c.bucket_width >= 0.0f) || !std::isfinite(c.bucket_width))
    return fail(VINE_ERR_INVALID, "bucket_width must be finite and >= 0");
  if (c.max_workers < 0) return fail(VINE_ERR_INVALID, "max_workers must be >= 0");
  if (c.band_mult == 0) c.band_mult = 16;
  if (c.ar_scale == 0.0f) c.ar_scale = 1.0f;
  if (!(c.ar_scale >= 1.0f / 64.0f && c.ar_scale <= 64.0f))
    return fail(VINE_ERR_INVALID, "ar_scale in [1/64, 64]");
  if (c.band_mult < 1 || c.band_mult > 1024) return fail(VINE_ERR_INVALID, "band_mult in [1, 1024]");
  if (c.wait_limit == 0) c.wait_limit = 1 << 26;
  if (c.wait_limit < 1) return fail(VINE_ERR_INVALID, "wait_limit must be >= 0");
  if (c.time_limit_ms == 0) c.time_limit_ms = 600000;
  const bool far_auto = c.far_capacity == 0;
  if (far_auto) c.far_capacity = int64_t(1) << 20;  // sized below once the worker count is known
  if (c.far_capacity < 1024 || c.far_capacity > (int64_t(1) << 30))
    return fail(VINE_ERR_INVALID, "far_capacity out of range");
  if (c.pool_labels == 0) {
    // keep the arena the engine already holds (resizing it would release and
    // rebuild the whole workspace between calls)
    const int64_t held = c.engine == VINE_ENGINE_BATCH ? g->batch.pool_cap : g->plain.pool_cap;
    if (held > 0) c.pool_labels = held;
  }
  if (c.pool_labels == 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    // arena + chain links: 20 bytes per label; workers keep the chunks of
    // their largest query, so the arena is sized for one heavy query each
    int64_t want = (int64_t)(free_b * 2 / 5 / (sizeof(Label) + sizeof(uint32_t)));
    c.pool_labels = std::min<int64_t>(want, (int64_t(1) << 31) - (int64_t(1) << 20));
  }
  if (c.pool_labels < 1024 || c.pool_labels > (int64_t(1) << 31) - (int64_t(1) << 20))
    return fail(VINE_ERR_INVALID, "pool_labels out of range");
  int round_cap = std::min(1024, 4 * c.block_threads);
  if (c.split_threshold < 0) return fail(VINE_ERR_INVALID, "split_threshold must be >= 0");
  if (c.split_threshold > 0) round_cap = std::max(32, std::min(round_cap, c.split_threshold));
  out->width0 = c.bucket_width > 0.0f ? c.bucket_width : std::max(1.0f, g->mean_len);
  out->round_cap = round_cap;
  out->slots = 0;
  if (c.engine == VINE_ENGINE_BATCH) VINE_TRY(batch_slots(g, c, round_cap, &out->slots));
  if (far_auto && out->slots > 0) {
    // every worker holds far_capacity x 160 bytes of piles (band bins and
    // rest pile, 4 x far_capacity labels + keys each): keep them within a
    // quarter of the device's memory, at most 2^20 per worker
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const int64_t per_worker = (int64_t)(total_b / 4 / (size_t)out->slots / 160);
    int64_t cap = int64_t(1) << 20;
    while (cap > 4096 && cap > per_worker) cap >>= 1;
    c.far_capacity = cap;
  }
  out->cfg = c;
  return VINE_OK;
}

}  // namespace vine

using namespace vine;

extern "C" {

const char *vine_last_error(void) { return g_last_error.c_str(); }
const char *vine_version(void) { return "vine-b200 0.1 (sm_100a)"; }

void vine_config_default(vine_config *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->engine = VINE_ENGINE_BATCH;
  cfg->mode = VINE_MODE_OPTIMAL;
  cfg->policy = VINE_POLICY_FIXED;
  cfg->use_bounds = 0;
  cfg->block_threads = 512;
  cfg->table_log2 = 11;
  cfg->spill_log2 = 16;
  cfg->use_cuda_graph = 0;
  cfg->order_queries = 1;
}

int vine_graph_create(int32_t device, int32_t n, int64_t m, const int64_t *row_ptr,
                      const int32_t *col, const float *len, const float *delay, vine_graph **out) {
  if (!out) return fail(VINE_ERR_INVALID, "null output handle");
  *out = nullptr;
  if (n < 1 || m < 0 || !row_ptr || (m > 0 && (!col || !len || !delay)))
    return fail(VINE_ERR_INVALID, "bad graph arrays");
  if (m >= (int64_t(1) << 31)) return fail(VINE_ERR_INVALID, "more than 2^31-1 arcs");
  if (row_ptr[0] != 0 || row_ptr[n] != m) return fail(VINE_ERR_INVALID, "row_ptr must run 0..m");
  for (int32_t u = 0; u < n; ++u)
    if (row_ptr[u + 1] < row_ptr[u]) return fail(VINE_ERR_INVALID, "row_ptr not monotone");
  bool integral = true;
  double sum_len = 0.0, sum_delay = 0.0;
  for (int64_t j = 0; j < m; ++j) {
    if (col[j] < 0 || col[j] >= n) return fail(VINE_ERR_INVALID, "arc head out of range");
    if (!(len[j] >= 0.0f) || !(delay[j] >= 0.0f) || !std::isfinite(len[j]) ||
        !std::isfinite(delay[j]))
      return fail(VINE_ERR_INVALID, "weights must be finite and >= 0");
    if (len[j] != std::floor(len[j]) || delay[j] != std::floor(delay[j]) || len[j] >= 16777216.0f ||
        delay[j] >= 16777216.0f)
      integral = false;
    sum_len += len[j];
    sum_delay += delay[j];
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(VINE_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(VINE_ERR_INVALID, "device out of range");
  VINE_CUDA_TRY(cudaSetDevice(device));

  std::vector<int32_t> row32((size_t)n + 1);
  for (int32_t i = 0; i <= n; ++i) row32[i] = (int32_t)row_ptr[i];
  std::vector<float2> w((size_t)m);
  for (int64_t j = 0; j < m; ++j) w[j] = make_float2(len[j], delay[j]);
  // reverse CSR (in-arcs), stable by source
  std::vector<int32_t> rrow((size_t)n + 1, 0), rcol((size_t)m);
  std::vector<float2> rw((size_t)m);
  for (int64_t j = 0; j < m; ++j) rrow[(size_t)col[j] + 1]++;
  for (int32_t i = 0; i < n; ++i) rrow[i + 1] += rrow[i];
  std::vector<int32_t> pos(rrow.begin(), rrow.end() - 1);
  for (int32_t u = 0; u < n; ++u)
    for (int64_t j = row_ptr[u]; j < row_ptr[u + 1]; ++j) {
      const int32_t p = pos[col[j]]++;
      rcol[p] = u;
      rw[p] = w[j];
    }

  auto *g = new vine_graph();
  g->device = device;
  g->n = n;
  g->m = m;
  g->integral = integral ? 1 : 0;
  g->mean_len = m > 0 ? (float)(sum_len / (double)m) : 1.0f;
  g->mean_delay = m > 0 ? (float)(sum_delay / (double)m) : 1.0f;
  uint64_t fp = 1469598103934665603ull;
  fp = fnv1a(fp, &n, sizeof(n));
  fp = fnv1a(fp, row32.data(), row32.size() * sizeof(int32_t));
  fp = fnv1a(fp, col, (size_t)m * sizeof(int32_t));
  fp = fnv1a(fp, w.data(), w.size() * sizeof(float2));
  g->fingerprint = fp;
  auto cleanup = [&](int st) {
    vine_graph_destroy(g);
    return st;
  };
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    return cleanup(fail(VINE_ERR_CUDA, "cudaGetDeviceProperties failed"));
  g->sm_count = prop.multiProcessorCount;
  const size_t mb = std::max<size_t>(1, (size_t)m);
  if (cudaMalloc(&g->row, sizeof(int32_t) * ((size_t)n + 1)) != cudaSuccess ||
      cudaMalloc(&g->col, sizeof(int32_t) * mb) != cudaSuccess ||
      cudaMalloc(&g->w, sizeof(float2) * mb) != cudaSuccess ||
      cudaMalloc(&g->rrow, sizeof(int32_t) * ((size_t)n + 1)) != cudaSuccess ||
      cudaMalloc(&g->rcol, sizeof(int32_t) * mb) != cudaSuccess ||
      cudaMalloc(&g->rw, sizeof(float2) * mb) != cudaSuccess)
    return cleanup(fail(VINE_ERR_CUDA, "graph allocation failed"));
  if (cudaMemcpy(g->row, row32.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      (m > 0 && cudaMemcpy(g->col, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice) != cudaSuccess) ||
      (m > 0 && cudaMemcpy(g->w, w.data(), sizeof(float2) * (size_t)m, cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(g->rrow, rrow.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      (m > 0 && cudaMemcpy(g->rcol, rcol.data(), sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice) != cudaSuccess) ||
      (m > 0 && cudaMemcpy(g->rw, rw.data(), sizeof(float2) * (size_t)m, cudaMemcpyHostToDevice) != cudaSuccess))
    return cleanup(fail(VINE_ERR_CUDA, "graph upload failed"));
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(VINE_ERR_CUDA, "stream creation failed"));
  *out = g;
  return VINE_OK;
}

void vine_graph_destroy(vine_graph *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  g->batch.release();
  g->plain.release();
  if (g->io_cache) {
    static_cast<IoCache *>(g->io_cache)->b.release();
    delete static_cast<IoCache *>(g->io_cache);
    g->io_cache = nullptr;
  }
  cudaFree(g->row);
  cudaFree(g->col);
  cudaFree(g->w);
  cudaFree(g->rrow);
  cudaFree(g->rcol);
  cudaFree(g->rw);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int vine_graph_info(const vine_graph *g, int32_t *n, int64_t *m, int32_t *integral) {
  if (!g) return fail(VINE_ERR_INVALID, "null graph");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (integral) *integral = g->integral;
  return VINE_OK;
}

static int run_engine(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
                      const int32_t *d_dst, const float *d_budget, const int32_t *h_src,
                      const int32_t *h_dst, const float *h_budget, const DeviceOutputs &o,
                      cudaStream_t s, PathOut *paths) {
  if (r.cfg.engine == VINE_ENGINE_BATCH)
    return batch_run(g, r, nq, d_src, d_dst, d_budget, o, s, paths);
  return plain_run(g, r, nq, h_src, h_dst, h_budget, o, s, paths);
}

int vine_solve_device(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
                      const float *budget, const vine_config *cfg, vine_results *out,
                      void *stream) {
  if (!g || !out || nq < 0) return fail(VINE_ERR_INVALID, "bad arguments");
  if (nq == 0) return VINE_OK;
  if (!src || !dst || !budget || !out->cost || !out->delay || !out->found || !out->status)
    return fail(VINE_ERR_INVALID, "missing input/output buffers");
  std::lock_guard<std::mutex> lk(g->mu);
  VINE_CUDA_TRY(cudaSetDevice(g->device));
  Resolved r;
  VINE_TRY(resolve_config(g, cfg, &r));
  if (r.cfg.engine != VINE_ENGINE_BATCH)
    return fail(VINE_ERR_INVALID, "vine_solve_device runs the batch engine only");
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream
  DeviceOutputs o;
  o.cost = out->cost;
  o.delay = out->delay;
  o.found = out->found;
  o.status = out->status;
  o.stats = out->stats;
  o.pareto_d = out->pareto_d;
  o.pareto_delay = out->pareto_delay;
  o.pareto_n = out->pareto_n;
  o.pareto_stride = out->pareto_d ? out->pareto_stride : 0;
  VINE_TRY(batch_prepare(g, r, nq, s));
  auto enqueue = [&]() -> int {
    PathOut paths;
    VINE_TRY(batch_enqueue(g, r, nq, src, dst, budget, o, s, &paths));
    if (out->path_offsets && out->path) {
      VINE_TRY(path_offsets(paths, nq, out->path_offsets, s));
      // packs the paths; the caller sizes `path` (path_capacity) for the total
      VINE_TRY(path_gather(paths, nq, out->path_offsets, out->path, s));
    }
    return VINE_OK;
  };
  if (!r.cfg.use_cuda_graph) return enqueue();
  // Replay the captured launch sequence when the call has the same shape,
  // buffers and configuration as the captured one; otherwise capture anew.
  BatchWorkspace &w = g->batch;
  uint64_t key = 1469598103934665603ull;
  const void *ptrs[] = {src, dst, budget, out->cost, out->delay, out->found, out->status,
                        out->stats, out->path_offsets, out->path, out->pareto_d,
                        out->pareto_delay, out->pareto_n, stream};
  key = fnv1a(key, &nq, sizeof(nq));
  key = fnv1a(key, ptrs, sizeof(ptrs));
  key = fnv1a(key, &r.cfg, sizeof(r.cfg));
  key = fnv1a(key, &r.width0, sizeof(r.width0));
  if (w.graph_exec == nullptr || w.graph_key != key) {
    if (w.graph_exec) {
      cudaGraphExecDestroy(w.graph_exec);
      w.graph_exec = nullptr;
    }
    VINE_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int st = enqueue();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (st != VINE_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess) return fail(VINE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&w.graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
      w.graph_exec = nullptr;
      return fail(VINE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    }
    w.graph_key = key;
  }
  VINE_CUDA_TRY(cudaGraphLaunch(w.graph_exec, s));
  return VINE_OK;
}

int vine_solve(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
               const float *budget, const vine_config *cfg, vine_results *out) {
  if (!g || !out || nq < 0) return fail(VINE_ERR_INVALID, "bad arguments");
  if (nq == 0) {
    if (out->path_offsets) out->path_offsets[0] = 0;
    return VINE_OK;
  }
  if (!src || !dst || !budget || !out->cost || !out->delay || !out->found)
    return fail(VINE_ERR_INVALID, "missing input/output buffers");
  std::lock_guard<std::mutex> lk(g->mu);
  VINE_CUDA_TRY(cudaSetDevice(g->device));
  Resolved r;
  VINE_TRY(resolve_config(g, cfg, &r));
  cudaStream_t s = g->stream;
  const bool want_pareto = out->pareto_d && out->pareto_delay && out->pareto_n && out->pareto_stride > 0;
  const bool want_paths = out->path_offsets != nullptr;

  out->retried = 0;
  constexpr int kMaxRetries = 4;
  std::vector<int32_t> status((size_t)nq, VINE_OK);
  std::vector<int32_t> todo((size_t)nq);
  for (int32_t i = 0; i < nq; ++i) todo[i] = i;
  int attempt = 0;
  std::vector<int64_t> all_len((size_t)nq, 0);
  std::vector<std::vector<int32_t>> all_paths(want_paths ? (size_t)nq : 0);
  int rc = VINE_OK;
  while (!todo.empty()) {
    const int32_t k = (int32_t)todo.size();
    std::vector<int32_t> hs(k), hd(k);
    std::vector<float> hb(k);
    for (int32_t i = 0; i < k; ++i) {
      hs[i] = src[todo[i]];
      hd[i] = dst[todo[i]];
      hb[i] = budget[todo[i]];
    }
    auto bail = [&](int st) {
      cudaStreamSynchronize(s);
      return st;
    };
    const size_t stride = want_pareto ? (size_t)out->pareto_stride : 0;
    IoCache &cache = io_cache(g);
    VINE_TRY(io_reserve(cache, k, out->stats != nullptr, stride));
    IoBuffers &io = cache.b;
    if (cudaMemcpyAsync(io.src, hs.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(io.dst, hd.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(io.budget, hb.data(), sizeof(float) * k, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return bail(fail(VINE_ERR_CUDA, "input upload failed"));
    DeviceOutputs o;
    o.cost = io.cost;
    o.delay = io.delay;
    o.found = io.found;
    o.status = io.status;
    o.stats = out->stats ? io.stats : nullptr;
    o.pareto_d = want_pareto ? io.pareto_d : nullptr;
    o.pareto_delay = want_pareto ? io.pareto_dl : nullptr;
    o.pareto_n = want_pareto ? io.pareto_n : nullptr;
    o.pareto_stride = (int32_t)stride;
    PathOut paths;
    int st = run_engine(g, r, k, io.src, io.dst, io.budget, hs.data(), hd.data(), hb.data(), o, s, &paths);
    if (st != VINE_OK) return bail(st);
    std::vector<int64_t> off;
    std::vector<int32_t> path;
    if (want_paths) {
      if ((st = path_offsets(paths, k, io.offsets, s)) != VINE_OK) return bail(st);
      off.resize((size_t)k + 1);
      if (cudaMemcpyAsync(off.data(), io.offsets, sizeof(int64_t) * (k + 1), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return bail(fail(VINE_ERR_CUDA, std::string("engine failed: ") + cudaGetErrorString(cudaGetLastError())));
      if (off[k] > 0) {
        if ((st = io_reserve_path(cache, off[k])) != VINE_OK) return bail(st);
        if ((st = path_gather(paths, k, io.offsets, io.path, s)) != VINE_OK) return bail(st);
        path.resize((size_t)off[k]);
        if (cudaMemcpyAsync(path.data(), io.path, sizeof(int32_t) * (size_t)off[k], cudaMemcpyDeviceToHost, s) != cudaSuccess)
          return bail(fail(VINE_ERR_CUDA, "path download failed"));
      }
    }
    std::vector<float> hc(k), hdl(k), pd, pl;
    std::vector<int32_t> hf(k), hst(k), pn;
    std::vector<int64_t> hstats;
    if (cudaMemcpyAsync(hc.data(), io.cost, sizeof(float) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(hdl.data(), io.delay, sizeof(float) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(hf.data(), io.found, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(hst.data(), io.status, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return bail(fail(VINE_ERR_CUDA, "result download failed"));
    if (out->stats) {
      hstats.resize((size_t)k * VINE_STAT_COUNT);
      if (cudaMemcpyAsync(hstats.data(), io.stats, sizeof(int64_t) * hstats.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return bail(fail(VINE_ERR_CUDA, "stats download failed"));
    }
    if (want_pareto) {
      pd.resize(stride * k);
      pl.resize(stride * k);
      pn.resize(k);
      if (cudaMemcpyAsync(pd.data(), io.pareto_d, sizeof(float) * pd.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaMemcpyAsync(pl.data(), io.pareto_dl, sizeof(float) * pl.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaMemcpyAsync(pn.data(), io.pareto_n, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return bail(fail(VINE_ERR_CUDA, "pareto download failed"));
    }
    if (cudaStreamSynchronize(s) != cudaSuccess)
      return bail(fail(VINE_ERR_CUDA, std::string("engine failed: ") + cudaGetErrorString(cudaGetLastError())));
    if (r.cfg.trace && r.cfg.engine == VINE_ENGINE_BATCH && g->batch.trace) {
      unsigned long long rows = 0;
      cudaMemcpy(&rows, g->batch.counters + 3, sizeof(rows), cudaMemcpyDeviceToHost);
      rows = std::min<unsigned long long>(rows, (unsigned long long)g->batch.trace_cap);
      g->last_trace.resize((size_t)rows * VINE_TRACE_COLS);
      if (rows)
        cudaMemcpy(g->last_trace.data(), g->batch.trace, sizeof(float) * g->last_trace.size(), cudaMemcpyDeviceToHost);
      // trace rows carry the engine's local query index; map back
      for (size_t i = 0; i < (size_t)rows; ++i) {
        float &qq = g->last_trace[i * VINE_TRACE_COLS + 16];
        const int32_t li = (int32_t)qq;
        if (li >= 0 && li < k) qq = (float)todo[li];
      }
    }
    std::vector<int32_t> retry;
    for (int32_t i = 0; i < k; ++i) {
      const int32_t q = todo[i];
      out->cost[q] = hc[i];
      out->delay[q] = hdl[i];
      out->found[q] = hf[i];
      status[q] = hst[i];
      if (out->stats)
        std::memcpy(out->stats + (size_t)q * VINE_STAT_COUNT, hstats.data() + (size_t)i * VINE_STAT_COUNT,
                    sizeof(int64_t) * VINE_STAT_COUNT);
      if (want_pareto) {
        out->pareto_n[q] = pn[i];
        const int32_t cnt = std::min<int32_t>(pn[i], out->pareto_stride);
        std::memcpy(out->pareto_d + (size_t)q * stride, pd.data() + (size_t)i * stride, sizeof(float) * cnt);
        std::memcpy(out->pareto_delay + (size_t)q * stride, pl.data() + (size_t)i * stride, sizeof(float) * cnt);
      }
      if (want_paths) {
        all_len[q] = off[i + 1] - off[i];
        all_paths[q].assign(path.begin() + off[i], path.begin() + off[i + 1]);
      }
      if (hst[i] == VINE_ERR_CAPACITY) retry.push_back(q);
    }
    if (retry.empty() || attempt >= kMaxRetries) break;
    if (attempt == 0) out->retried = (int32_t)retry.size();
    // retry the overflowing queries with roomier per-worker structures: the
    // first retry gives each of them its own worker with 8x piles and the
    // largest label arena; later ones halve the number of workers running
    // at once, so that fewer heavy queries share the arena (workers keep
    // the arena chunks of their largest query)
    ++attempt;
    if (attempt == 1) {
      r.cfg.far_capacity = std::min<int64_t>(r.cfg.far_capacity * 8, int64_t(1) << 24);
      r.cfg.pool_labels = (int64_t(1) << 31) - (int64_t(1) << 20);
      r.cfg.max_workers = (int32_t)std::min<size_t>(retry.size(), 1u << 16);
    } else {
      r.cfg.far_capacity = std::min<int64_t>(r.cfg.far_capacity * 2, int64_t(1) << 24);
      r.cfg.max_workers = std::max(1, std::min(r.cfg.max_workers, (int32_t)retry.size()) / 2);
    }
    r.cfg.spill_log2 = std::min(r.cfg.spill_log2 + 3, 22);
    r.cfg.ctas_per_sm = 1;
    r.cfg.trace = 0;
    {
      // the retried workers' piles (160 bytes per far_capacity unit each)
      // stay within a third of the device's memory
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      const int64_t workers = std::max<int64_t>(1, std::min<int64_t>(r.cfg.max_workers, (int64_t)g->sm_count));
      while (r.cfg.far_capacity > (int64_t(1) << 20) &&
             workers * r.cfg.far_capacity * 160 > (int64_t)(total_b / 3))
        r.cfg.far_capacity >>= 1;
    }
    VINE_TRY(resolve_config(g, &r.cfg, &r));
    r.chunk_log2 = 20;  // 4096 chunks of 2^20 labels per worker: room for any query the arena holds
    todo = retry;
  }
  int32_t n_failed = 0;
  for (int32_t q = 0; q < nq; ++q) {
    if (out->status) out->status[q] = status[q];
    if (status[q] != VINE_OK) {
      ++n_failed;
      if (rc == VINE_OK) rc = status[q];
    }
  }
  // this call's own message (the thread's text may still hold an older one)
  if (rc != VINE_OK)
    set_error(std::to_string(n_failed) + " of " + std::to_string(nq) +
              " queries failed; first status " + std::to_string(rc) +
              (rc == VINE_ERR_CAPACITY ? " (engine capacity, also after the retry)" : ""));
  if (want_paths) {
    int64_t run = 0;
    for (int32_t q = 0; q < nq; ++q) {
      out->path_offsets[q] = run;
      run += all_len[q];
    }
    out->path_offsets[nq] = run;
    if (run > out->path_capacity || out->path == nullptr) {
      if (rc == VINE_OK) rc = fail(VINE_ERR_CAPACITY, "path buffer too small (need " + std::to_string(run) + ")");
      else set_error(vine_last_error() + std::string("; path buffer too small (need ") + std::to_string(run) + ")");
    } else {
      for (int32_t q = 0; q < nq; ++q)
        std::memcpy(out->path + out->path_offsets[q], all_paths[q].data(), sizeof(int32_t) * all_len[q]);
    }
  }
  return rc;
}

int vine_trace_fetch(vine_graph *g, int64_t *rows, float *buf, int64_t capacity) {
  if (!g || !rows) return fail(VINE_ERR_INVALID, "bad arguments");
  const int64_t n = (int64_t)(g->last_trace.size() / VINE_TRACE_COLS);
  *rows = n;
  if (buf) {
    const int64_t c = std::min(n, capacity);
    std::memcpy(buf, g->last_trace.data(), sizeof(float) * (size_t)c * VINE_TRACE_COLS);
  }
  return VINE_OK;
}

}  // extern "C"
