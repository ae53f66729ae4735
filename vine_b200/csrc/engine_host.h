// Host-side state of a graph handle and the launch interfaces of the two
// engines.  Shared by api.cu, batch.cu, plain.cu and mlp.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/vine.h"
#include "common.h"
#include "engine.cuh"

namespace vine {

// Device buffers owned by one graph handle for the batch engine; reused
// between calls while the shape fits.
struct BatchWorkspace {
  int slots = 0;
  int block_threads = 0;
  int table_log2 = 0;
  int64_t far_cap = 0;
  int64_t near_cap = 0;
  int sink_cap = 0;
  int64_t pool_cap = 0;
  VState *vs = nullptr;
  uint32_t *nearq = nullptr;
  Label *far = nullptr;
  uint32_t *sinklist = nullptr;
  uint32_t *bctr = nullptr;     // per worker bucket counter
  uint32_t *next = nullptr;     // arena-parallel chain links
  Label *rest = nullptr;        // per worker rest pile
  float *far_key = nullptr;     // keys beside the band bins
  float *rest_key = nullptr;    // keys beside the rest pile
  int64_t rest_cap = 0;
  uint2 *chunks = nullptr;      // per worker arena chunk lists
  int max_chunks = 0;
  int32_t *path_arena = nullptr;
  int64_t path_cap = 0;
  int64_t *path_start = nullptr;
  int32_t *path_len = nullptr;
  Label *pool = nullptr;
  unsigned long long *counters = nullptr;  // [0]=pool_top [1]=queue [2]=path_top [3]=trace_top
  int32_t *order = nullptr;
  int64_t q_cap = 0;
  float *trace = nullptr;
  int64_t trace_cap = 0;
  uint32_t epoch_next = 1;
  // captured launch sequence (CUDA graph) for the current shape
  cudaGraphExec_t graph_exec = nullptr;
  uint64_t graph_key = 0;
  void release();
};

// Device buffers of the plain (whole-GPU, one query at a time) engine.
struct PlainWorkspace {
  int32_t n = 0;
  int64_t far_cap = 0;
  int64_t pool_cap = 0;
  VState *vs = nullptr;
  uint32_t *nearq = nullptr;
  Label *far[2] = {nullptr, nullptr};
  int *locks = nullptr;
  Label *pool = nullptr;
  uint32_t *next = nullptr;
  uint32_t *sinklist = nullptr;
  int64_t q_cap = 0;
  int32_t *path_arena = nullptr;
  int64_t path_cap = 0;
  int64_t *path_start = nullptr;
  int32_t *path_len = nullptr;
  unsigned long long *path_top = nullptr;
  void *st = nullptr;       // device query state
  void *st_host = nullptr;  // pinned host mirror
  uint32_t bctr = 0;
  uint32_t epoch_next = 1;
  void release();
};

}  // namespace vine

struct vine_graph {
  int device = 0;
  int sm_count = 0;
  int32_t n = 0;
  int64_t m = 0;
  int32_t integral = 0;
  float mean_len = 1.0f;
  float mean_delay = 1.0f;
  int32_t *row = nullptr, *col = nullptr, *rrow = nullptr, *rcol = nullptr;
  float2 *w = nullptr, *rw = nullptr;
  uint64_t fingerprint = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;  // one solve at a time per handle
  vine::BatchWorkspace batch;
  vine::PlainWorkspace plain;
  std::vector<float> last_trace;  // host copy of the last trace
  void *io_cache = nullptr;       // device in/out buffers of vine_solve, kept between calls
  vine::DevGraph dev() const {
    vine::DevGraph g;
    g.n = n;
    g.m = m;
    g.row = row;
    g.col = col;
    g.w = w;
    g.rrow = rrow;
    g.rcol = rcol;
    g.rw = rw;
    return g;
  }
};

struct vine_mlp {
  int device = 0;
  float *params = nullptr;  // device, kMlpParams floats
  float *adam_m = nullptr;
  float *adam_v = nullptr;
  int64_t step = 0;
};

namespace vine {

// Per-call outputs on the device (all device pointers; pareto/stats optional).
struct DeviceOutputs {
  float *cost = nullptr;
  float *delay = nullptr;
  int32_t *found = nullptr;
  int32_t *status = nullptr;
  int64_t *stats = nullptr;
  float *pareto_d = nullptr;
  float *pareto_delay = nullptr;
  int32_t *pareto_n = nullptr;
  int32_t pareto_stride = 0;
};

// Where an engine left the answer paths of the last call: query q's path is
// arena[start[q] .. start[q] + len[q]) (device pointers).
struct PathOut {
  const int32_t *arena = nullptr;
  const int64_t *start = nullptr;
  const int32_t *len = nullptr;
};

// Resolved configuration (defaults filled in).
struct Resolved {
  vine_config cfg;
  int slots;
  float width0;
  int round_cap;
  int chunk_log2 = 16;  // arena chunk size a worker takes at a time (2^16 labels;
                        // capacity retries use larger chunks, since a worker
                        // holds at most 4096 of them)
};

int resolve_config(const vine_graph *g, const vine_config *in, Resolved *out);

// Batch engine: solves nq queries whose inputs are on the device.
int batch_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
              const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
              cudaStream_t stream, PathOut *paths);

// The two halves of batch_run: workspace / epoch bookkeeping (host work,
// never captured) and the stream work (capturable in a CUDA graph).
int batch_prepare(vine_graph *g, const Resolved &r, int32_t nq, cudaStream_t stream);
int batch_enqueue(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
                  const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
                  cudaStream_t stream, PathOut *paths);

// Plain engine: solves the queries one at a time with the whole GPU.
int plain_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *h_src,
              const int32_t *h_dst, const float *h_budget, const DeviceOutputs &out,
              cudaStream_t stream, PathOut *paths);

// Orders queries by decreasing budget class (largest first).
int order_queries(int32_t nq, const float *d_budget, int32_t *d_order, cudaStream_t stream);

// Packs the paths of `p` in query order: offsets[q] = exclusive prefix sum of
// the lengths (offsets[nq] = total), then path[offsets[q] ..] = path of q.
int path_offsets(const PathOut &p, int32_t nq, int64_t *d_offsets, cudaStream_t stream);
int path_gather(const PathOut &p, int32_t nq, const int64_t *d_offsets, int32_t *d_path,
                cudaStream_t stream);

}  // namespace vine
