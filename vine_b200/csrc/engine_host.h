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
  int spill_log2 = 0;
  int64_t far_cap = 0;
  int64_t near_cap = 0;
  int sink_cap = 0;
  int64_t pool_cap = 0;
  VState *vs = nullptr;
  uint32_t *nearq = nullptr;
  Label *far = nullptr;
  TEntry *spill = nullptr;
  TEntry *rebuild = nullptr;  // per worker: table entries kept across a rebalance
  Label *retry = nullptr;     // per worker: 2 lists of deferred low-key candidates
  int64_t retry_cap = 0;
  uint32_t *spill_used = nullptr;
  uint32_t *sinklist = nullptr;
  Label *pool = nullptr;
  unsigned long long *counters = nullptr;  // [0]=pool_top [1]=queue [2]=path_top [3]=trace_top
  int32_t *best_idx = nullptr;             // per query, capacity q_cap
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
  int table_log2 = 0;
  int64_t far_cap = 0;
  int64_t near_cap = 0;
  int64_t pool_cap = 0;
  VState *vs = nullptr;
  uint32_t *nearq = nullptr;
  Label *far[2] = {nullptr, nullptr};
  TEntry *table = nullptr;
  uint32_t *table_used = nullptr;
  int *locks = nullptr;
  Label *pool = nullptr;
  uint32_t *sinklist = nullptr;
  int sink_cap = 0;
  unsigned long long *ctl = nullptr;  // device control block (see plain.cu)
  unsigned long long *ctl_host = nullptr;  // pinned mirror
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
  int32_t *row = nullptr, *col = nullptr, *rrow = nullptr, *rcol = nullptr;
  float2 *w = nullptr, *rw = nullptr;
  uint64_t fingerprint = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;  // one solve at a time per handle
  vine::BatchWorkspace batch;
  vine::PlainWorkspace plain;
  std::vector<float> last_trace;  // host copy of the last trace
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
  int32_t *best_idx = nullptr;  // arena index of the answer label per query
};

// Resolved configuration (defaults filled in).
struct Resolved {
  vine_config cfg;
  int slots;
  float width0;
  int round_cap;
};

int resolve_config(const vine_graph *g, const vine_config *in, Resolved *out);

// Batch engine: solves nq queries whose inputs are on the device.
int batch_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
              const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
              cudaStream_t stream, Label **pool_out);

// Plain engine: solves the queries one at a time with the whole GPU.
int plain_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *h_src,
              const int32_t *h_dst, const float *h_budget, const DeviceOutputs &out,
              cudaStream_t stream, Label **pool_out);

// Path extraction from an arena: lengths (pass 1) then vertices (pass 2).
int path_lengths(const Label *pool, int32_t nq, const int32_t *d_best_idx, int64_t *d_offsets,
                 cudaStream_t stream);
int path_write(const Label *pool, int32_t nq, const int32_t *d_best_idx,
               const int64_t *d_offsets, int32_t *d_path, cudaStream_t stream);

}  // namespace vine
