// Plain engine: one query at a time on the whole GPU, host-driven rounds.
//
// This is the baseline the batch engine is measured against, with the same
// structure as the reference's GPU driver RUN_CSPP (algorithm/cspp.cuh:69-325):
// per round the host launches an expansion kernel over the whole frontier,
// copies the control state back (the reference copies the scanned frontier
// size, cspp.cuh:245-248), runs the bucket policy on the host in FP64 (the
// reference's AR step, cspp.cuh:254-284) and launches the split of the far
// pile (the reference's recheck / fill, cspp.cuh:205-213, 291).  The device
// side reuses the batch engine's search functions; the bucket store is the
// per-vertex overflow chains alone (no shared-memory level, since blocks of
// one round do not share memory), with striped locks in global memory.

#include "engine_host.h"
#include "search.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace vine {

namespace {

constexpr int kPlainThreads = 256;
constexpr int kPlainRound = 1024;       // near labels per block and round
constexpr int kPlainLockLog2 = 20;
constexpr int64_t kPlainNear = int64_t(1) << 24;

struct PlainArgs {
  SearchParams P;
  QueryState *st;
  int *locks;
  Label *far_cur;
  Label *far_next;
};

__device__ void plain_ctx(Ctx &c, const PlainArgs &A) {
  const SearchParams &P = A.P;
  c.vs = P.vs;
  c.nearq = P.nearq;
  c.far = A.far_cur;
  c.sinks = P.sinklist;
  c.bt.tv = nullptr;
  c.bt.tw = nullptr;
  c.bt.ti = nullptr;
  c.bt.log2h = 0;
  c.bt.probe = 0;  // no shared-memory level: every label lives in a chain
  c.bt.locks = A.locks;
  c.bt.lock_mask = (1 << kPlainLockLog2) - 1;
  c.bt.vs = P.vs;
  c.bt.next = P.next;
  c.bt.chain_steps = nullptr;
  c.bt.spin_limit = P.wait_limit;
  c.bt.epoch = A.st->epoch;
  c.bt.qbase = A.st->qbase;
  c.bt.bcur = A.st->bcur;
}

__device__ void flush_counters(Ctx &c) {
  QueryState &st = c.st;
  if (c.c_dominated) atomicAdd(&st.b_dominated, c.c_dominated);
  if (c.c_candidates) atomicAdd(&st.b_candidates, c.c_candidates);
  if (c.c_spills) atomicAdd(&st.b_spilled, c.c_spills);
  if (c.c_near) atomicAdd(&st.b_labels, c.c_near);
  if (c.c_dominated)
    atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
  if (c.c_near + c.c_far)
    atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
  if (c.c_spills) atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
  c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
}

// Expansion round: block b expands near items [first + b*R, ...).
__global__ void __launch_bounds__(kPlainThreads) plain_round_kernel(PlainArgs A, uint32_t first,
                                                                    uint32_t n) {
  __shared__ uint32_t s_idx[kPlainRound];
  __shared__ int s_vid[kPlainRound], s_beg[kPlainRound], s_off[kPlainRound];
  __shared__ float s_d[kPlainRound], s_dl[kPlainRound];
  __shared__ int s_scan[kScanScratch];
  Ctx c(A.P, *A.st);
  plain_ctx(c, A);
  const RoundBuf rb{s_idx, s_vid, s_d, s_dl, s_beg, s_off, s_scan, kPlainRound};
  const uint32_t b0 = blockIdx.x * (uint32_t)kPlainRound;
  if (b0 >= n) return;
  expand_block(c, rb, first + b0, (int)min((uint32_t)kPlainRound, n - b0));
  flush_counters(c);
}

__global__ void __launch_bounds__(kPlainThreads) plain_reverse_kernel(PlainArgs A, int which,
                                                                      uint32_t first, uint32_t n,
                                                                      float radius) {
  __shared__ uint32_t s_idx[kPlainRound];
  __shared__ int s_vid[kPlainRound], s_beg[kPlainRound], s_off[kPlainRound];
  __shared__ float s_d[kPlainRound], s_dl[kPlainRound];
  __shared__ int s_scan[kScanScratch];
  Ctx c(A.P, *A.st);
  plain_ctx(c, A);
  const RoundBuf rb{s_idx, s_vid, s_d, s_dl, s_beg, s_off, s_scan, kPlainRound};
  const uint32_t b0 = blockIdx.x * (uint32_t)kPlainRound;
  if (b0 >= n) return;
  reverse_expand_block(c, rb, which, first + b0, (int)min((uint32_t)kPlainRound, n - b0), radius,
                       bucket_hi(c.st), true);
}

// Split of the far pile into the open bucket (forward search) or into the
// near ring (reverse passes, which = 0/1); kept items go to far_next.
__global__ void plain_split_kernel(PlainArgs A, uint32_t fn, int which) {
  Ctx c(A.P, *A.st);
  plain_ctx(c, A);
  QueryState &st = *A.st;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < fn) {
    const Label item = A.far_cur[i];
    bool keep;
    float key;
    if (which < 0) {
      keep = offer(c, item.vid, item.d, item.dl, (uint32_t)item.parent, true);
      key = keep ? key_of(c, item.vid, item.d) : 0.0f;
    } else {
      keep = false;
      key = item.d;
      if (item.d <= reverse_dist(c, which, item.vid)) {
        if (item.d < bucket_hi(st)) {
          const uint32_t pos = atomicAdd(&st.near_tail, 1u);
          c.nearq[pos & A.P.near_mask] = (uint32_t)item.vid;
        } else {
          keep = true;
        }
      }
    }
    if (keep) {
      const uint32_t w = warp_agg_inc(&st.far_wpos);
      A.far_next[w] = item;
      atomicMin(&st.far_min_bits, __float_as_uint(key));
    }
  }
  flush_counters(c);
}

// Query setup (one thread): epoch, sink of the reverse passes, source label.
__global__ void plain_setup_kernel(PlainArgs A, int q, int phase) {
  const SearchParams &P = A.P;
  QueryState &st = *A.st;
  Ctx c(P, st);
  plain_ctx(c, A);
  if (phase == 0) {
    const int s = st.src, t = st.dst;
    const float L = st.budget;
    if (s < 0 || s >= P.g.n || t < 0 || t >= P.g.n || isnan(L)) {
      fail_query(st, VINE_ERR_INVALID, kSiteInvalid);
      return;
    }
    if (0.0f > L) {
      st.done = 1;
      return;
    }
    const uint32_t idx = atomicAdd(&st.chunk_fill, 1u);
    if (idx >= st.chunk_end) {
      fail_query(st, VINE_ERR_CAPACITY, kSiteArena);
      return;
    }
    P.pool[idx] = Label{s, 0.0f, 0.0f, -1};
    st.inc_idx = idx;
    if (s == t) {
      st.inc_key = pack_key(0.0f, 0.0f);
      st.done = 1;
      if (P.mode == VINE_MODE_PARETO) {
        c.sinks[0] = idx;
        st.sink_n = 1;
      }
    }
  } else if (phase == 1 || phase == 2) {  // start reverse pass (phase - 1)
    VState *sv = &c.vs[st.dst];
    if (phase == 1) {
      bool claimed = false;
      relax_pair(&sv->e_del, st.epoch, 0.0f, &claimed);
      if (claimed) atomicExch(reinterpret_cast<unsigned int *>(&sv->hlen), kInfBits);
    } else {
      atomicMin(reinterpret_cast<unsigned int *>(&sv->hlen), 0u);
    }
    c.nearq[st.near_tail & P.near_mask] = (uint32_t)st.dst;
    st.near_tail += 1;
  } else {  // phase 3: place the source label into the first bucket
    const VView sv = c.view(st.src);
    const uint32_t idx = st.inc_idx;
    st.inc_idx = 0xffffffffu;
    if (!sv.reach) {
      st.done = 1;
      return;
    }
    st.lo = sv.hlen;
    st.hi_bits = __float_as_uint(sv.hlen + st.width);
    // a chain of one label at the source
    VState *vs = &c.vs[st.src];
    P.next[idx] = kNone;
    vs->bhead = idx;
    *reinterpret_cast<volatile unsigned long long *>(&vs->bep) =
        ((unsigned long long)__float_as_uint(0.0f) << 32) | st.bcur;
    c.near_ring()[st.near_tail & P.near_mask] = make_uint2(idx, (uint32_t)st.src);
    st.near_tail += 1;
    st.b_labels = 1;
  }
}

// Results of one query (one block): Pareto set, answer, statistics.
__global__ void plain_finish_kernel(PlainArgs A, int q) {
  const SearchParams &P = A.P;
  QueryState &st = *A.st;
  const int tid = threadIdx.x, G = blockDim.x;
  __shared__ uint32_t alive;
  if (tid == 0) alive = 0;
  __syncthreads();
  if (P.mode == VINE_MODE_PARETO && !st.abort) {
    const uint32_t k = min(st.sink_n, (uint32_t)P.sink_cap);
    for (uint32_t i = tid; i < k; i += G) {
      const Label a = load_label(&P.pool[P.sinklist[i]]);
      if (a.vid & (int)kDeadBit) continue;
      atomicAdd(&alive, 1u);
      const uint64_t ka = pack_key(a.d, a.dl);
      int rank = 0;
      for (uint32_t j = 0; j < k; ++j) {
        const Label b = load_label(&P.pool[P.sinklist[j]]);
        if (b.vid & (int)kDeadBit) continue;
        if (pack_key(b.d, b.dl) < ka) ++rank;
      }
      if (rank < P.pareto_stride && P.pareto_d) {
        P.pareto_d[(size_t)q * P.pareto_stride + rank] = a.d;
        P.pareto_dl[(size_t)q * P.pareto_stride + rank] = a.dl;
      }
      if (rank == 0) {
        st.inc_key = ka;
        st.inc_idx = P.sinklist[i];
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    copy_out_path(P, st, q, st.abort == 0 && st.inc_key != ~0ull);
    const bool ok = st.abort == 0;
    const bool found = ok && st.inc_key != ~0ull;
    P.status[q] = ok ? VINE_OK : st.abort;
    P.found[q] = found ? 1 : 0;
    P.cost[q] = found ? key_d(st.inc_key) : INFINITY;
    P.odelay[q] = found ? key_dl(st.inc_key) : INFINITY;
    if (P.pareto_n) P.pareto_n[q] = (P.mode == VINE_MODE_PARETO && ok) ? (int32_t)alive : 0;
    if (P.stats) {
      int64_t *s = P.stats + (size_t)q * VINE_STAT_COUNT;
      s[VINE_STAT_EXPANDED] = st.n_expanded;
      s[VINE_STAT_RELAXED] = st.n_relaxed;
      s[VINE_STAT_INSERTED] = st.n_inserted;
      s[VINE_STAT_DOMINATED] = st.n_dominated;
      s[VINE_STAT_BUCKETS] = st.n_buckets;
      s[VINE_STAT_ROUNDS] = st.n_rounds;
      s[VINE_STAT_SPILLS] = st.n_spills;
      s[VINE_STAT_CYCLES] = 0;
      s[VINE_STAT_ABORT_SITE] = st.abort_site;
      s[VINE_STAT_BOUND_ROUNDS] = 0;
      s[VINE_STAT_BOUND_CYCLES] = 0;
      s[VINE_STAT_CHAIN_STEPS] = 0;
      s[VINE_STAT_SPLIT_CYCLES] = 0;
      s[VINE_STAT_SPLIT_ITEMS] = 0;
      s[VINE_STAT_POLICY_CYCLES] = 0;
      s[VINE_STAT_LOAD_CYCLES] = 0;
      s[VINE_STAT_RELAX_CYCLES] = 0;
      s[VINE_STAT_START_NS] = 0;
      s[VINE_STAT_TIME_NS] = 0;
      s[VINE_STAT_REST_ITEMS] = 0;
      s[VINE_STAT_IDLE_CYCLES] = 0;
      s[VINE_STAT_PUBLISH_CYCLES] = 0;
    }
  }
}

// Host side of the bucket policy (fixed width or AR), the same rules as the
// device scheduler step, applied between rounds like the reference's host AR
// step (algorithm/cspp.cuh:254-284).
void host_policy(QueryState &h, int policy, float width0, int table_log2) {
  const double xs = std::log2(1.0 + (double)h.b_labels);
  if (h.hist_n < kHist) {
    h.hist[h.hist_n++] = xs;
  } else {
    for (int i = 1; i < kHist; ++i) h.hist[i - 1] = h.hist[i];
    h.hist[kHist - 1] = xs;
  }
  if (policy != VINE_POLICY_AR) {
    h.width = width0;
    return;
  }
  double pred = xs;
  const bool ar_ok = burg_forecast(h.hist, h.hist_n, 3, &pred);
  float width = h.width;
  const int n = h.hist_n;
  if (n >= 4 && h.hist[n - 1] < h.hist[n - 2] && h.hist[n - 2] < h.hist[n - 3] &&
      h.hist[n - 3] < h.hist[n - 4]) {
    width *= 1.5f;
  } else if (ar_ok) {
    const double est = std::exp2(pred);
    const double target = 0.25 * (double)(1 << table_log2);
    const double ratio = std::min(2.0, std::max(0.5, target / std::max(est, 1.0)));
    width = (float)(width * ratio);
  }
  h.width = std::min(std::max(width, width0 * 0.125f), width0 * 64.0f);
}

float bits_float(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}
uint32_t float_bits(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  return b;
}

}  // namespace

void PlainWorkspace::release() {
  cudaFree(vs);
  cudaFree(nearq);
  cudaFree(far[0]);
  cudaFree(far[1]);
  cudaFree(locks);
  cudaFree(pool);
  cudaFree(next);
  cudaFree(sinklist);
  cudaFree(path_arena);
  cudaFree(path_start);
  cudaFree(path_len);
  cudaFree(path_top);
  cudaFree(st);
  cudaFreeHost(st_host);
  *this = PlainWorkspace();
}

static int ensure_plain_workspace(vine_graph *g, const Resolved &r, int32_t nq) {
  PlainWorkspace &w = g->plain;
  const vine_config &c = r.cfg;
  const int64_t far_cap = std::max<int64_t>(c.far_capacity, int64_t(1) << 24);
  if (w.vs == nullptr || w.far_cap != far_cap || w.pool_cap != c.pool_labels) {
    w.release();
    VINE_CUDA_TRY(cudaMalloc(&w.vs, sizeof(VState) * (size_t)g->n));
    VINE_CUDA_TRY(cudaMemset(w.vs, 0, sizeof(VState) * (size_t)g->n));
    VINE_CUDA_TRY(cudaMalloc(&w.nearq, sizeof(uint2) * (size_t)kPlainNear));
    VINE_CUDA_TRY(cudaMalloc(&w.far[0], sizeof(Label) * (size_t)far_cap));
    VINE_CUDA_TRY(cudaMalloc(&w.far[1], sizeof(Label) * (size_t)far_cap));
    VINE_CUDA_TRY(cudaMalloc(&w.locks, sizeof(int) << kPlainLockLog2));
    VINE_CUDA_TRY(cudaMemset(w.locks, 0, sizeof(int) << kPlainLockLog2));
    VINE_CUDA_TRY(cudaMalloc(&w.pool, sizeof(Label) * (size_t)c.pool_labels));
    VINE_CUDA_TRY(cudaMalloc(&w.next, sizeof(uint32_t) * (size_t)c.pool_labels));
    VINE_CUDA_TRY(cudaMalloc(&w.sinklist, sizeof(uint32_t) * 4096));
    VINE_CUDA_TRY(cudaMalloc(&w.st, sizeof(QueryState)));
    VINE_CUDA_TRY(cudaMallocHost(&w.st_host, sizeof(QueryState)));
    w.n = g->n;
    w.far_cap = far_cap;
    w.pool_cap = c.pool_labels;
    w.bctr = 0;
    w.epoch_next = 1;
  }
  if (w.q_cap < nq) {
    cudaFree(w.path_arena);
    cudaFree(w.path_start);
    cudaFree(w.path_len);
    cudaFree(w.path_top);
    w.path_arena = nullptr;
    w.path_start = nullptr;
    w.path_len = nullptr;
    w.path_top = nullptr;
    w.q_cap = std::max<int64_t>(nq, 1024);
    w.path_cap = w.q_cap * 4096;
    VINE_CUDA_TRY(cudaMalloc(&w.path_arena, sizeof(int32_t) * (size_t)w.path_cap));
    VINE_CUDA_TRY(cudaMalloc(&w.path_start, sizeof(int64_t) * (size_t)w.q_cap));
    VINE_CUDA_TRY(cudaMalloc(&w.path_len, sizeof(int32_t) * (size_t)w.q_cap));
    VINE_CUDA_TRY(cudaMalloc(&w.path_top, sizeof(unsigned long long)));
  }
  return VINE_OK;
}

int plain_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *h_src,
              const int32_t *h_dst, const float *h_budget, const DeviceOutputs &out,
              cudaStream_t stream, PathOut *paths) {
  const vine_config &c = r.cfg;
  if (c.policy == VINE_POLICY_MLP)
    return fail(VINE_ERR_INVALID, "the plain engine runs the fixed or AR policy only");
  VINE_TRY(ensure_plain_workspace(g, r, nq));
  PlainWorkspace &w = g->plain;
  if (w.epoch_next > 0xF0000000u - (uint32_t)nq || w.bctr > 0xF0000000u) {
    VINE_CUDA_TRY(cudaMemsetAsync(w.vs, 0, sizeof(VState) * (size_t)g->n, stream));
    w.epoch_next = 1;
    w.bctr = 0;
  }
  PlainArgs A;
  std::memset(&A, 0, sizeof(A));
  SearchParams &P = A.P;
  P.g = g->dev();
  P.nq = nq;
  P.cost = out.cost;
  P.odelay = out.delay;
  P.found = out.found;
  P.status = out.status;
  P.stats = out.stats;
  P.pareto_d = out.pareto_d;
  P.pareto_dl = out.pareto_delay;
  P.pareto_n = out.pareto_n;
  P.pareto_stride = out.pareto_stride;
  P.path_arena = w.path_arena;
  P.path_cap = w.path_cap;
  P.path_top = w.path_top;
  P.path_start = w.path_start;
  P.path_len = w.path_len;
  P.rest_cap = 0;
  P.vs = w.vs;
  P.nearq = w.nearq;
  P.near_mask = (uint32_t)(kPlainNear - 1);
  P.far_cap = w.far_cap;
  P.sinklist = w.sinklist;
  P.sink_cap = 4096;
  P.pool = w.pool;
  P.next = w.next;
  P.pool_cap = w.pool_cap;
  P.mode = c.mode;
  P.policy = c.policy;
  P.use_bounds = c.use_bounds;
  P.width0 = r.width0;
  P.len_scale = std::max(1.0f, g->mean_len);
  P.round_cap = r.round_cap;
  P.wait_limit = c.wait_limit;
  P.time_limit_ns = 0;  // the host loop below enforces time_limit_ms
  P.table_log2 = c.table_log2;
  P.grid_scope = 1;
  A.st = static_cast<QueryState *>(w.st);
  A.locks = w.locks;
  QueryState &h = *static_cast<QueryState *>(w.st_host);
  const float delta_del = std::max(1.0f, 4.0f * g->mean_delay);
  const float delta_len = std::max(1.0f, 4.0f * g->mean_len);
  const uint32_t split_cap = c.split_threshold > 0 ? (uint32_t)c.split_threshold : 0xffffffffu;
  int cur = 0;
  VINE_CUDA_TRY(cudaMemsetAsync(w.path_top, 0, sizeof(unsigned long long), stream));
  auto push = [&]() -> int {
    VINE_CUDA_TRY(cudaMemcpyAsync(w.st, &h, sizeof(QueryState), cudaMemcpyHostToDevice, stream));
    return VINE_OK;
  };
  auto pull = [&]() -> int {
    VINE_CUDA_TRY(cudaMemcpyAsync(&h, w.st, sizeof(QueryState), cudaMemcpyDeviceToHost, stream));
    VINE_CUDA_TRY(cudaStreamSynchronize(stream));
    return VINE_OK;
  };
  auto args = [&]() {
    A.far_cur = w.far[cur];
    A.far_next = w.far[cur ^ 1];
    return A;
  };
  // splits the far pile (which < 0: forward search, else reverse pass)
  auto split = [&](int which) -> int {
    const uint32_t fn = h.far_n;
    h.far_wpos = 0;
    h.far_min_bits = kInfBits;
    VINE_TRY(push());
    plain_split_kernel<<<(fn + 255) / 256, 256, 0, stream>>>(args(), fn, which);
    VINE_CUDA_TRY(cudaGetLastError());
    VINE_TRY(pull());
    cur ^= 1;
    h.far_n = h.far_wpos;
    if (h.far_n > (uint64_t)w.far_cap && !h.abort) {
      h.abort = VINE_ERR_CAPACITY;
      h.abort_site = kSiteBand;
    }
    return VINE_OK;
  };
  std::chrono::steady_clock::time_point t_query;
  // time_limit_ms on the host clock: checked once per round / bucket
  auto timed_out = [&]() {
    if (c.time_limit_ms <= 0) return false;
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_query).count();
    if (ms <= (double)c.time_limit_ms) return false;
    if (!h.abort) {
      h.abort = VINE_ERR_TIMEOUT;
      h.abort_site = kSiteTime;
    }
    return true;
  };
  for (int32_t q = 0; q < nq; ++q) {
    t_query = std::chrono::steady_clock::now();
    std::memset(&h, 0, sizeof(QueryState));
    h.q = q;
    h.src = h_src[q];
    h.dst = h_dst[q];
    h.budget = h_budget[q];
    h.epoch = w.epoch_next + (uint32_t)q;
    h.bcur = ++w.bctr;
    h.qbase = h.bcur;
    h.inc_key = ~0ull;
    h.inc_idx = 0xffffffffu;
    h.far_min_bits = kInfBits;
    h.chunk_fill = 0;  // each query's answer path is copied out: reuse the arena
    h.chunk_end = (uint32_t)w.pool_cap;
    h.band_hi = INFINITY;  // one far pile (no band / rest split here)
    h.width = r.width0;
    h.split_cap = (int)std::min<uint32_t>(split_cap, 0x7fffffffu);
    VINE_TRY(push());
    plain_setup_kernel<<<1, 1, 0, stream>>>(args(), q, 0);
    VINE_TRY(pull());
    if (!h.done && !h.abort && c.use_bounds) {
      for (int which = 0; which < 2 && !h.abort; ++which) {
        const float delta = which == 0 ? delta_del : delta_len;
        const float radius = which == 0 ? h.budget : INFINITY;
        h.near_head = h.near_tail = 0;
        h.far_n = 0;
        h.far_min_bits = kInfBits;
        h.lo = 0.0f;
        h.hi_bits = float_bits(delta);
        VINE_TRY(push());
        plain_setup_kernel<<<1, 1, 0, stream>>>(args(), q, 1 + which);
        VINE_TRY(pull());
        while (!h.abort && !timed_out()) {
          const uint32_t avail = h.near_tail - h.near_head;
          if (avail == 0) {
            if (h.far_n == 0) break;
            h.lo = std::max(bits_float(h.hi_bits), bits_float(h.far_min_bits));
            h.hi_bits = float_bits(h.lo + delta);
            VINE_TRY(split(which));
            continue;
          }
          const uint32_t first = h.near_head;
          h.near_head += avail;
          h.n_rounds++;
          VINE_TRY(push());
          plain_reverse_kernel<<<(avail + kPlainRound - 1) / kPlainRound, kPlainThreads, 0, stream>>>(
              args(), which, first, avail, radius);
          VINE_CUDA_TRY(cudaGetLastError());
          VINE_TRY(pull());
        }
      }
      h.near_head = h.near_tail = 0;
      h.far_n = 0;
      h.far_min_bits = kInfBits;
    }
    if (!h.done && !h.abort) {
      VINE_TRY(push());
      plain_setup_kernel<<<1, 1, 0, stream>>>(args(), q, 3);
      VINE_TRY(pull());
    }
    while (!h.done && !h.abort && !timed_out()) {
      const uint32_t avail = h.near_tail - h.near_head;
      if (avail == 0) {
        // bucket finished: its chains become settled when bcur advances
        host_policy(h, c.policy, r.width0, c.table_log2);
        h.n_buckets++;
        const float fmin = bits_float(h.far_min_bits);
        const float inc_d = bits_float((uint32_t)(h.inc_key >> 32));
        if (h.far_n == 0 || (c.mode == VINE_MODE_OPTIMAL && h.inc_key != ~0ull && fmin > inc_d)) {
          h.done = 1;
          break;
        }
        h.lo = std::max(bits_float(h.hi_bits), fmin);
        float hi = h.lo + h.width;
        if (!(hi > h.lo)) hi = std::nextafter(h.lo, INFINITY);
        h.hi_bits = float_bits(hi);
        h.bcur = ++w.bctr;
        h.b_labels = h.b_expanded = h.b_rounds = h.b_dominated = 0;
        h.b_candidates = h.b_spilled = h.b_relaxed = 0;
        VINE_TRY(split(-1));
        continue;
      }
      const uint32_t n = std::min<uint32_t>(avail, split_cap);
      const uint32_t first = h.near_head;
      h.near_head += n;
      h.n_rounds++;
      h.b_rounds++;
      if (h.n_rounds > kMaxRounds) {
        h.abort = VINE_ERR_TIMEOUT;
        h.abort_site = kSiteRounds;
        break;
      }
      VINE_TRY(push());
      plain_round_kernel<<<(n + kPlainRound - 1) / kPlainRound, kPlainThreads, 0, stream>>>(args(),
                                                                                        first, n);
      VINE_CUDA_TRY(cudaGetLastError());
      VINE_TRY(pull());
      h.n_expanded += h.r_live;
      h.b_expanded += h.r_live;
      h.r_live = 0;
    }
    VINE_TRY(push());
    plain_finish_kernel<<<1, 256, 0, stream>>>(args(), q);
    VINE_CUDA_TRY(cudaGetLastError());
  }
  w.epoch_next += (uint32_t)nq;
  if (paths) {
    paths->arena = w.path_arena;
    paths->start = w.path_start;
    paths->len = w.path_len;
  }
  return VINE_OK;
}

}  // namespace vine
