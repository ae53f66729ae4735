// Batched exact CSP engine: one persistent kernel, one query per CTA worker.
//
// Replaces the reference's per-query host loop RUN_CSPP
// (algorithm/cspp.cuh:134-296), which launched expand / recheck / Thrust scan
// / fill kernels and copied the frontier size to the host every round.  Here
// each CTA pulls a query from a device work queue, runs the whole bucketed
// label search with block barriers only, writes the result and pulls the next
// query.  Per-query state lives in per-worker HBM regions (lazily reset by an
// epoch tag) and in shared memory:
//
//   * bucket table  -- labels of the open bucket, keyed by vertex, in shared
//                      memory with an HBM spill table; replaces the 96-slot
//                      shared hash + global dominance lists
//                      (algorithm/bucket.cuh:80-119, algorithm/dominance.cuh:15-153)
//   * settled delay -- one float per vertex summarising finished buckets
//   * near queue    -- ring of arena indices still to expand in this bucket
//   * far pile      -- labels beyond the bucket, split into later buckets
//                      (the reference's DOP split / recheck, cspp.cuh:179-216,
//                      algorithm/bucket.cuh:217-245)
//   * arena         -- every accepted label with its parent, for paths
//
// One round: load up to `split` near labels, prefix-sum their out-degrees,
// then every thread relaxes one arc at a time (load-balanced search), which
// keeps all lanes busy for both degree-2 road vertices and power-law hubs.

#include "engine_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

namespace vine {

namespace {

constexpr int kHist = kBurgMaxN;
constexpr uint32_t kInfBits = 0x7f800000u;
constexpr int kScanScratch = 40;
constexpr long long kMaxRounds = 1ll << 26;

struct BatchParams {
  DevGraph g;
  int32_t nq;
  const int32_t *src;
  const int32_t *dst;
  const float *budget;
  const int32_t *order;
  // outputs
  float *cost;
  float *odelay;
  int32_t *found;
  int32_t *status;
  int64_t *stats;
  float *pareto_d;
  float *pareto_dl;
  int32_t *pareto_n;
  int32_t pareto_stride;
  int32_t *best_idx;
  // workspace
  VState *vs;
  uint32_t *nearq;
  uint32_t near_mask;
  Label *far;
  int64_t far_cap;
  TEntry *spill;
  uint32_t *spill_used;
  int spill_log2;
  uint32_t spill_limit;
  uint32_t *sinklist;
  int sink_cap;
  Label *pool;
  unsigned long long *pool_top;
  int64_t pool_cap;
  uint32_t chunk;
  unsigned long long *queue;
  TEntry *rebuild;
  Label *retry;
  uint32_t retry_cap;
  uint32_t epoch_base;
  // configuration
  int mode;
  int policy;
  int use_bounds;
  float width0;
  int round_cap;
  int table_log2;
  int lock_log2;
  int probe;
  const float *mlp;
  float *trace;
  unsigned long long *trace_top;
  int64_t trace_cap;
};

struct __align__(16) CtaState {
  unsigned long long inc_key;
  long long t0;
  long long n_expanded, n_relaxed, n_inserted, n_dominated, n_buckets, n_rounds, n_spills;
  double hist[kHist];
  int q, src, dst;
  float budget;
  uint32_t epoch;
  uint32_t inc_idx;
  int inc_lock;
  float lo, width;
  uint32_t hi_bits;  // bucket upper key (float bits); lowered when the table overflows
  uint32_t far_n, far_wpos, far_min_bits;
  uint32_t near_head, near_tail;
  uint32_t s_count;
  uint32_t chunk_fill, chunk_end;
  int abort;
  int n_round, e_round;
  int done;
  int split_cap;
  int hist_n;
  uint32_t sink_n;
  uint32_t b_labels, b_expanded, b_rounds, b_dominated, b_candidates, b_spilled, b_relaxed;
  uint32_t r_live;
  uint32_t ovf_n;      // deferred candidates in the active retry list
  uint32_t ovf_cur;    // which retry list receives deferrals
  int overflow;        // a table insert failed this round
  uint32_t keep_n;
  int rb_again;
  int rb_count;        // rebalances in the open bucket
  float x_prev[kFeat];
  float x[kFeat];
  float mh[2 * kHid];
  float y[kOut];
};

__device__ __forceinline__ VState load_vs(const VState *p) {
  float4 raw = __ldcg(reinterpret_cast<const float4 *>(p));
  VState s;
  s.epoch = __float_as_uint(raw.x);
  s.sdel = raw.y;
  s.hlen = raw.z;
  s.hdel = raw.w;
  return s;
}

__device__ __forceinline__ Label load_label(const Label *p) {
  int4 raw = __ldcg(reinterpret_cast<const int4 *>(p));
  Label l;
  l.vid = raw.x;
  l.d = __int_as_float(raw.y);
  l.dl = __int_as_float(raw.z);
  l.parent = raw.w;
  return l;
}

__device__ __forceinline__ float bucket_hi(const CtaState &st) {
  return __uint_as_float(*reinterpret_cast<const volatile uint32_t *>(&st.hi_bits));
}

struct Ctx {
  const BatchParams &P;
  CtaState &st;
  BucketTable bt;
  VState *vs;
  uint32_t *nearq;
  Label *far;
  uint32_t *sinks;
  TEntry *rebuild;
  Label *retry;
  uint32_t c_dominated = 0, c_near = 0, c_far = 0, c_spills = 0, c_candidates = 0;
  __device__ Ctx(const BatchParams &p, CtaState &s) : P(p), st(s) {}
};

// Sink label that beats the incumbent (optimal mode): stored in the arena and
// published under a small lock so that key and arena index stay paired.
__device__ void sink_improve(Ctx &c, int32_t v, float nd, float ndl, uint32_t parent,
                             uint64_t key) {
  CtaState &st = c.st;
  const uint32_t idx = atomicAdd(&st.chunk_fill, 1u);
  if (idx >= st.chunk_end) {
    st.abort = VINE_ERR_CAPACITY;
    return;
  }
  c.P.pool[idx] = Label{v, nd, ndl, (int32_t)parent};
  const bool ok = with_lock(&st.inc_lock, [&]() {
    volatile unsigned long long *ik = &st.inc_key;
    if (key < *ik) {
      *ik = key;
      st.inc_idx = idx;
    }
  });
  if (!ok) st.abort = VINE_ERR_TIMEOUT;
}

// Offers one label (v, nd, ndl) to the search.  from_far = true when it comes
// from the far pile (budget already checked); returns true when a far label
// must stay in the far pile.
__device__ bool offer(Ctx &c, int32_t v, float nd, float ndl, uint32_t parent, bool from_far) {
  const BatchParams &P = c.P;
  CtaState &st = c.st;
  const VState s = load_vs(&c.vs[v]);
  const bool fresh = (s.epoch == st.epoch);
  float hl = 0.0f, hd = 0.0f;
  if (P.use_bounds) {
    if (!fresh) return false;  // not within the bounds of any feasible path
    hl = s.hlen;
    hd = s.hdel;
  }
  const float lb_dl = ndl + hd;
  if (!from_far) {
    c.c_candidates++;
    if (lb_dl > st.budget) return false;  // include/constraint.hpp:99-101
  }
  if (fresh && ndl >= s.sdel) {  // dominated by a label of a finished bucket
    c.c_dominated++;
    return false;
  }
  const float f = nd + hl;
  if (P.mode == VINE_MODE_OPTIMAL) {
    const uint64_t key = pack_key(f, lb_dl);
    if (key >= *reinterpret_cast<volatile unsigned long long *>(&st.inc_key)) return false;
    if (v == st.dst) {
      sink_improve(c, v, nd, ndl, parent, key);
      return false;
    }
  }
  if (f < bucket_hi(st)) {
    uint32_t idx = 0;
    bool spilled = false;
    Label *pool = P.pool;
    uint32_t *fill = &st.chunk_fill;
    const uint32_t end = st.chunk_end;
    auto alloc = [pool, fill, end, v, nd, ndl, parent]() -> uint32_t {
      const uint32_t i = atomicAdd(fill, 1u);
      if (i >= end) return kBadIdx;
      pool[i] = Label{v, nd, ndl, (int32_t)parent};
      return i;
    };
    const InsertResult r = table_insert(c.bt, P.pool, v, nd, ndl, alloc, &idx, &spilled);
    if (r == kDominated) {
      c.c_dominated++;
      return false;
    }
    if (r == kLockTimeout) {
      st.abort = VINE_ERR_TIMEOUT;
      return false;
    }
    if (r == kFull) {
      // Bucket split: the open bucket holds more labels than the tables do.
      // Its upper key drops to this label's key, so this label goes to the
      // far pile; table labels at or above the new bound follow at the next
      // rebalance (between rounds), which frees their slots.  A label at the
      // bucket's lowest key cannot be split off: it waits in a retry list
      // and is offered again after the rebalance.
      st.overflow = 1;
      c.c_spills++;
      if (f > st.lo) {
        atomicMin(&st.hi_bits, __float_as_uint(f));
        goto to_far;
      }
      const uint32_t k = atomicAdd(&st.ovf_n, 1u);
      if (k >= P.retry_cap) {
        st.abort = VINE_ERR_CAPACITY;
        return false;
      }
      c.retry[st.ovf_cur * P.retry_cap + k] = Label{v, nd, ndl, (int32_t)parent};
      return false;
    }
    c.c_near++;
    if (spilled) c.c_spills++;
    const uint32_t pos = atomicAdd(&st.near_tail, 1u);
    c.nearq[pos & P.near_mask] = idx;
    if (P.mode == VINE_MODE_PARETO && v == st.dst) {
      const uint32_t k = atomicAdd(&st.sink_n, 1u);
      if (k < (uint32_t)P.sink_cap) c.sinks[k] = idx;
      else st.abort = VINE_ERR_CAPACITY;
    }
    return false;
  }
to_far:
  if (from_far) return true;
  const uint32_t pos = warp_agg_inc(&st.far_n);
  if (pos >= (uint64_t)P.far_cap) {
    st.abort = VINE_ERR_CAPACITY;
    return false;
  }
  c.far[pos] = Label{v, nd, ndl, (int32_t)parent};
  atomicMin(&st.far_min_bits, __float_as_uint(f));
  c.c_far++;
  return false;
}

// Closes one bucket-table entry at the end of its bucket: a live label with
// key below the (possibly lowered) upper bound is settled; one at or above it
// was split off and returns to the far pile (its arena copy is retired).
__device__ void fold_entry(Ctx &c, const TEntry &e, float hi) {
  if (e.idx & kDeadBit) return;
  const BatchParams &P = c.P;
  CtaState &st = c.st;
  float hl = 0.0f;
  if (P.use_bounds) hl = load_vs(&c.vs[e.vid]).hlen;
  const float f = e.d + hl;
  if (f < hi) {
    settle(&c.vs[e.vid], st.epoch, e.dl);
    return;
  }
  const Label lab = load_label(&P.pool[e.idx]);
  atomicOr(reinterpret_cast<unsigned int *>(&P.pool[e.idx].vid), kDeadBit);
  const uint32_t pos = warp_agg_inc(&st.far_n);
  if (pos >= (uint64_t)P.far_cap) {
    st.abort = VINE_ERR_CAPACITY;
    return;
  }
  c.far[pos] = Label{e.vid, e.d, e.dl, lab.parent};
  atomicMin(&st.far_min_bits, __float_as_uint(f));
}

// Makes sure the current arena chunk has room for `need` more labels
// (thread 0 only, between barriers).
__device__ void pool_reserve(const BatchParams &P, CtaState &st, uint32_t need) {
  if ((uint64_t)st.chunk_fill + need <= (uint64_t)st.chunk_end) return;
  const uint64_t size = need > P.chunk ? need : P.chunk;
  const unsigned long long base = atomicAdd(P.pool_top, (unsigned long long)size);
  if (base + size > (unsigned long long)P.pool_cap) {
    st.abort = VINE_ERR_CAPACITY;
    st.chunk_fill = st.chunk_end = 0;
    return;
  }
  st.chunk_fill = (uint32_t)base;
  st.chunk_end = (uint32_t)(base + size);
}

// Scheduler step at a bucket boundary, run by warp 0.  Chooses the width and
// split threshold of the next bucket; records a trace row for the finished
// bucket when tracing is on.
__device__ void policy_step(const BatchParams &P, CtaState &st) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    const double xs = log2(1.0 + (double)st.b_labels);
    if (st.hist_n < kHist) {
      st.hist[st.hist_n++] = xs;
    } else {
      for (int i = 1; i < kHist; ++i) st.hist[i - 1] = st.hist[i];
      st.hist[kHist - 1] = xs;
    }
    if (P.trace) {
      const unsigned long long r = atomicAdd(P.trace_top, 1ull);
      if ((long long)r < P.trace_cap) {
        float *row = P.trace + r * 20;
        for (int i = 0; i < kFeat; ++i) row[i] = st.x_prev[i];
        row[16] = (float)st.q;
        row[17] = st.width;
        row[18] = (float)st.b_expanded;
        row[19] = (float)st.b_rounds;
      }
    }
    double pred = xs;
    const bool ar_ok = burg_forecast(st.hist, st.hist_n, 3, &pred);
    BucketStats b;
    b.far_n = (float)st.far_n;
    b.bucket_labels = (float)st.b_labels;
    b.expanded = (float)st.b_expanded;
    b.rounds = (float)st.b_rounds;
    b.total_expanded = (float)st.n_expanded;
    b.buckets = (float)st.n_buckets;
    b.width_rel = log2f(st.width / P.width0);
    b.dominated_frac = st.b_candidates ? (float)st.b_dominated / (float)st.b_candidates : 0.0f;
    const bool have_inc = st.inc_key != ~0ull;
    b.inc_found = have_inc ? 1.0f : 0.0f;
    b.inc_gap = have_inc ? log2f(1.0f + fmaxf(0.0f, key_d(st.inc_key) - bucket_hi(st)) / P.width0) : -1.0f;
    const float far_min = __uint_as_float(st.far_min_bits);
    b.far_gap = st.far_n ? log2f(1.0f + fmaxf(0.0f, far_min - bucket_hi(st)) / P.width0) : -1.0f;
    b.table_fill = (float)st.b_labels / (float)(1 << P.table_log2);
    b.spilled = st.b_spilled ? 1.0f : 0.0f;
    b.mean_degree = st.b_expanded ? (float)st.b_relaxed / (float)st.b_expanded : 0.0f;
    b.ar_delta = ar_ok ? (float)(pred - xs) : 0.0f;
    b.budget_rel = log2f(1.0f + st.budget / P.width0);
    make_features(b, st.x);
    // default (fixed) decision
    float width = P.width0;
    int split = P.round_cap;
    if (P.policy == VINE_POLICY_AR || P.policy == VINE_POLICY_MLP) {
      // AR rule, after algorithm/cspp.cuh:254-284: widen by 1.5x while the
      // bucket sizes have fallen three times in a row ("ending part");
      // otherwise steer the forecast size towards a quarter of the table.
      width = st.width;
      const int n = st.hist_n;
      if (n >= 4 && st.hist[n - 1] < st.hist[n - 2] && st.hist[n - 2] < st.hist[n - 3] &&
          st.hist[n - 3] < st.hist[n - 4]) {
        width *= 1.5f;
      } else if (ar_ok) {
        const double est = exp2(pred);
        const double target = 0.25 * (double)(1 << P.table_log2);
        double ratio = target / fmax(est, 1.0);
        ratio = fmin(2.0, fmax(0.5, ratio));
        width = (float)(width * ratio);
      }
      width = fminf(fmaxf(width, P.width0 * 0.125f), P.width0 * 64.0f);
    }
    st.width = width;
    st.split_cap = split;
  }
  __syncwarp();
  if (P.policy == VINE_POLICY_MLP && P.mlp != nullptr) {
    mlp_forward_warp(P.mlp, st.x, st.mh, st.y);
    if (lane == 0) {
      const float y0 = st.y[0], y1 = st.y[1];
      if (isfinite(y0) && isfinite(y1)) {
        // the network only reorders work: its outputs are clamped and any
        // width > 0 keeps the search exact
        st.width = P.width0 * exp2f(fminf(fmaxf(y0, -3.0f), 6.0f));
        const float lc = fminf(fmaxf(y1, 5.0f), log2f((float)P.round_cap));
        st.split_cap = max(32, min(P.round_cap, (int)exp2f(lc)));
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    for (int i = 0; i < kFeat; ++i) st.x_prev[i] = st.x[i];
  }
  __syncwarp();
}


__device__ __forceinline__ float key_of(const Ctx &c, int32_t vid, float d) {
  return c.P.use_bounds ? d + load_vs(&c.vs[vid]).hlen : d;
}

// Stores a label of the open bucket into the tables without dominance checks
// (used to rebuild the tables; the labels are mutually non-dominated).
__device__ bool insert_unchecked(const BucketTable &bt, const TEntry &x) {
  const uint32_t hmask = (1u << bt.log2h) - 1u;
  const uint32_t h0 = hash_vid(x.vid, bt.log2h);
  for (int p = 0; p < bt.probe; ++p) {
    TEntry *e = &bt.t[(h0 + p) & hmask];
    if (atomicCAS(&e->vid, kEmpty, x.vid) == kEmpty) {
      e->d = x.d;
      e->dl = x.dl;
      e->idx = x.idx;
      return true;
    }
  }
  const uint32_t cnt = atomicAdd(bt.s_count, 1u);
  if (cnt >= bt.s_limit) return false;
  const uint32_t smask = (1u << bt.log2s) - 1u;
  const uint32_t g0 = hash_vid(x.vid, bt.log2s);
  for (uint32_t q = 0; q <= smask; ++q) {
    const uint32_t pos = (g0 + q) & smask;
    TEntry *e = &bt.s[pos];
    if (atomicCAS(&e->vid, kEmpty, x.vid) == kEmpty) {
      bt.s_used[cnt] = pos;
      e->d = x.d;
      e->dl = x.dl;
      e->idx = x.idx;
      return true;
    }
  }
  return false;
}

// Rebalance after a bucket-table overflow (all threads, between rounds).
// 1. If the labels below the bucket's upper key still fill more than half of
//    the tables, lower the key further using a 32-bin histogram of the keys.
// 2. Move every live table label at or above the key back to the far pile
//    (retiring its arena copy) and rebuild the tables from the rest.
// 3. Drop retired / split-off entries from the near queue.
// 4. Offer the deferred lowest-key candidates again.
// Exactness does not depend on any of the choices made here: labels only move
// between this bucket and later ones.
__device__ void rebalance(Ctx &c, TEntry *table, int H, int *hist) {
  const BatchParams &P = c.P;
  CtaState &st = c.st;
  const int tid = threadIdx.x, G = blockDim.x;
  const uint32_t cap = (uint32_t)H + P.spill_limit;
  if (tid == 0) {
    if (++st.rb_count > 32) st.abort = VINE_ERR_CAPACITY;
  }
  __syncthreads();
  if (st.abort) return;
  for (int iter = 0; iter < 8; ++iter) {
    if (tid < 32) hist[tid] = 0;
    __syncthreads();
    const float lo = st.lo, hi = bucket_hi(st);
    const float scale = 32.0f / (hi - lo);
    const uint32_t sc = st.s_count;
    for (uint32_t i = tid; i < (uint32_t)H + sc; i += G) {
      const TEntry e = i < (uint32_t)H ? table[i] : c.bt.s[c.bt.s_used[i - H]];
      if (e.vid == kEmpty || (e.idx & kDeadBit)) continue;
      const float f = key_of(c, e.vid, e.d);
      if (f >= hi) continue;
      const int b = min(31, max(0, (int)((f - lo) * scale)));
      atomicAdd(&hist[b], 1);
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t total = 0;
      for (int b = 0; b < 32; ++b) total += (uint32_t)hist[b];
      st.rb_again = 0;
      if (total > cap / 2) {
        uint32_t run = 0;
        int k = 0;
        while (k < 32 && run + (uint32_t)hist[k] <= cap / 2) run += (uint32_t)hist[k++];
        if (k == 0) {
          k = 1;
          st.rb_again = 1;  // one bin alone is too crowded: subdivide it
        }
        float nh = lo + (hi - lo) * ((float)k / 32.0f);
        if (!(nh > lo)) {
          nh = nextafterf(lo, INFINITY);
          st.rb_again = 0;
        }
        if (nh < hi) st.hi_bits = __float_as_uint(nh);
        else st.rb_again = 0;
      }
    }
    __syncthreads();
    if (!st.rb_again) break;
  }
  // evict and collect the labels that stay
  if (tid == 0) st.keep_n = 0;
  __syncthreads();
  {
    const float hi = bucket_hi(st);
    const uint32_t sc = st.s_count;
    for (uint32_t i = tid; i < (uint32_t)H + sc; i += G) {
      const TEntry e = i < (uint32_t)H ? table[i] : c.bt.s[c.bt.s_used[i - H]];
      if (e.vid == kEmpty || (e.idx & kDeadBit)) continue;
      const float f = key_of(c, e.vid, e.d);
      if (f < hi) {
        const uint32_t k = warp_agg_inc(&st.keep_n);
        c.rebuild[k] = e;
      } else {
        const Label lab = load_label(&P.pool[e.idx]);
        atomicOr(reinterpret_cast<unsigned int *>(&P.pool[e.idx].vid), kDeadBit);
        const uint32_t pos = warp_agg_inc(&st.far_n);
        if (pos >= (uint64_t)P.far_cap) {
          st.abort = VINE_ERR_CAPACITY;
        } else {
          c.far[pos] = Label{e.vid, e.d, e.dl, lab.parent};
          atomicMin(&st.far_min_bits, __float_as_uint(f));
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < H; i += G) table[i].vid = kEmpty;
    for (uint32_t i = tid; i < sc; i += G) c.bt.s[c.bt.s_used[i]].vid = kEmpty;
    __syncthreads();
    if (tid == 0) st.s_count = 0;
    __syncthreads();
    const uint32_t kn = st.keep_n;
    for (uint32_t i = tid; i < kn; i += G)
      if (!insert_unchecked(c.bt, c.rebuild[i])) st.abort = VINE_ERR_CAPACITY;
    __syncthreads();
  }
  // compact the near queue in place (each tile is read before it is written)
  {
    const float hi = bucket_hi(st);
    const uint32_t head = st.near_head, tail = st.near_tail;
    if (tid == 0) st.keep_n = 0;
    __syncthreads();
    for (uint32_t base = head; base < tail; base += (uint32_t)G) {
      const uint32_t i = base + tid;
      const bool valid = i < tail;
      uint32_t idx = 0;
      if (valid) idx = c.nearq[i & P.near_mask];
      __syncthreads();
      if (valid) {
        const Label lab = load_label(&P.pool[idx]);
        if (!(lab.vid & (int)kDeadBit) && key_of(c, lab.vid, lab.d) < hi) {
          const uint32_t w = warp_agg_inc(&st.keep_n);
          c.nearq[(head + w) & P.near_mask] = idx;
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      st.near_tail = head + st.keep_n;
      st.overflow = 0;
    }
    __syncthreads();
  }
  // offer the deferred candidates again (new deferrals go to the other list)
  const uint32_t cur = st.ovf_cur, n = st.ovf_n;
  __syncthreads();
  if (tid == 0) {
    st.ovf_cur = cur ^ 1u;
    st.ovf_n = 0;
  }
  __syncthreads();
  for (uint32_t base = 0; base < n; base += (uint32_t)G) {
    if (tid == 0) pool_reserve(P, st, (uint32_t)G);
    __syncthreads();
    if (st.abort) break;
    const uint32_t i = base + tid;
    if (i < n) {
      const Label lab = c.retry[cur * P.retry_cap + i];
      if (offer(c, lab.vid, lab.d, lab.dl, (uint32_t)lab.parent, true)) {
        const uint32_t pos = warp_agg_inc(&st.far_n);
        if (pos >= (uint64_t)P.far_cap) {
          st.abort = VINE_ERR_CAPACITY;
        } else {
          c.far[pos] = lab;
          atomicMin(&st.far_min_bits, __float_as_uint(key_of(c, lab.vid, lab.d)));
        }
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(1024) batch_kernel(BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int H = 1 << P.table_log2;
  const int NL = 1 << P.lock_log2;
  const int RC = P.round_cap;
  TEntry *table = reinterpret_cast<TEntry *>(smem);
  int *locks = reinterpret_cast<int *>(table + H);
  uint32_t *r_idx = reinterpret_cast<uint32_t *>(locks + NL);
  int *r_vid = reinterpret_cast<int *>(r_idx + RC);
  float *r_d = reinterpret_cast<float *>(r_vid + RC);
  float *r_dl = r_d + RC;
  int *r_beg = reinterpret_cast<int *>(r_dl + RC);
  int *r_off = r_beg + RC;
  int *scan = r_off + RC;
  CtaState &st = *reinterpret_cast<CtaState *>(
      (reinterpret_cast<uintptr_t>(scan + kScanScratch) + 15) & ~(uintptr_t)15);

  const int tid = threadIdx.x, G = blockDim.x;
  const int slot = blockIdx.x;
  Ctx c(P, st);
  c.vs = P.vs + (size_t)slot * P.g.n;
  c.nearq = P.nearq + (size_t)slot * (P.near_mask + 1u);
  c.far = P.far + (size_t)slot * P.far_cap;
  c.sinks = P.sinklist + (size_t)slot * P.sink_cap;
  c.rebuild = P.rebuild + ((size_t)slot << P.table_log2) + (size_t)slot * P.spill_limit;
  c.retry = P.retry + (size_t)slot * 2 * P.retry_cap;
  c.bt.t = table;
  c.bt.log2h = P.table_log2;
  c.bt.probe = P.probe;
  c.bt.locks = locks;
  c.bt.lock_mask = NL - 1;
  c.bt.s = P.spill + ((size_t)slot << P.spill_log2);
  c.bt.log2s = P.spill_log2;
  c.bt.s_used = P.spill_used + (size_t)slot * P.spill_limit;
  c.bt.s_count = &st.s_count;
  c.bt.s_limit = P.spill_limit;

  for (int i = tid; i < H; i += G) table[i].vid = kEmpty;
  for (int i = tid; i < NL; i += G) locks[i] = 0;
  if (tid == 0) {
    st.chunk_fill = 0;
    st.chunk_end = 0;
    st.s_count = 0;
  }
  __syncthreads();

  for (;;) {
    if (tid == 0) {
      const unsigned long long k = atomicAdd(P.queue, 1ull);
      st.q = (k < (unsigned long long)P.nq) ? (P.order ? P.order[k] : (int)k) : -1;
    }
    __syncthreads();
    const int q = st.q;
    if (q < 0) break;

    // ------------------------------------------------------------- setup
    if (tid == 0) {
      st.t0 = clock64();
      st.src = P.src[q];
      st.dst = P.dst[q];
      st.budget = P.budget[q];
      st.epoch = P.epoch_base + (uint32_t)q;
      st.inc_key = ~0ull;
      st.inc_idx = 0xffffffffu;
      st.inc_lock = 0;
      st.far_n = 0;
      st.far_wpos = 0;
      st.far_min_bits = kInfBits;
      st.near_head = st.near_tail = 0;
      st.s_count = 0;
      st.abort = 0;
      st.done = 0;
      st.n_expanded = st.n_relaxed = st.n_inserted = st.n_dominated = 0;
      st.n_buckets = st.n_rounds = st.n_spills = 0;
      st.hist_n = 0;
      st.sink_n = 0;
      st.b_labels = st.b_expanded = st.b_rounds = st.b_dominated = 0;
      st.b_candidates = st.b_spilled = st.b_relaxed = 0;
      st.r_live = 0;
      st.ovf_n = 0;
      st.ovf_cur = 0;
      st.overflow = 0;
      st.rb_count = 0;
      st.width = P.width0;
      st.split_cap = P.round_cap;
      for (int i = 0; i < kFeat; ++i) st.x_prev[i] = 0.0f;
      const int s = st.src, t = st.dst;
      const float L = st.budget;
      if (s < 0 || s >= P.g.n || t < 0 || t >= P.g.n || isnan(L)) {
        st.abort = VINE_ERR_INVALID;
      } else if (0.0f > L) {
        st.done = 1;  // even the source label violates the budget
      } else {
        pool_reserve(P, st, 1);
        if (!st.abort) {
          const uint32_t idx = st.chunk_fill++;
          P.pool[idx] = Label{s, 0.0f, 0.0f, -1};
          if (s == t) {
            // the source label is the unique Pareto-optimal sink label
            st.inc_key = pack_key(0.0f, 0.0f);
            st.inc_idx = idx;
            st.done = 1;
            if (P.mode == VINE_MODE_PARETO) {
              c.sinks[0] = idx;
              st.sink_n = 1;
            }
          } else {
            st.lo = 0.0f;
            st.hi_bits = __float_as_uint(P.width0);
            table[hash_vid(s, P.table_log2) & (H - 1)] = TEntry{s, 0.0f, 0.0f, idx};
            c.nearq[0] = idx;
            st.near_tail = 1;
            st.b_labels = 1;
          }
        }
      }
    }
    __syncthreads();

    // --------------------------------------------------- bucket / round loop
    while (!st.done && !st.abort) {
      if (st.overflow) {
        rebalance(c, table, H, scan);
        continue;
      }
      const uint32_t avail = st.near_tail - st.near_head;
      if (avail == 0) {
        // ---- bucket finished: settle its labels, pick the next bucket
        atomicAdd(&st.b_dominated, c.c_dominated);
        atomicAdd(&st.b_candidates, c.c_candidates);
        atomicAdd(&st.b_spilled, c.c_spills);
        atomicAdd(&st.b_labels, c.c_near);
        atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
        atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
        atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
        c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
        {
          const float hi = bucket_hi(st);
          for (int i = tid; i < H; i += G) {
            const TEntry e = table[i];
            if (e.vid != kEmpty) {
              fold_entry(c, e, hi);
              table[i].vid = kEmpty;
            }
          }
          const uint32_t sc = st.s_count;
          for (uint32_t i = tid; i < sc; i += G) {
            const uint32_t pos = c.bt.s_used[i];
            const TEntry e = c.bt.s[pos];
            fold_entry(c, e, hi);
            c.bt.s[pos].vid = kEmpty;
          }
        }
        __syncthreads();
        if (tid < 32) policy_step(P, st);
        if (tid == 0) {
          st.n_buckets++;
          st.s_count = 0;
          const float fmin = __uint_as_float(st.far_min_bits);
          if (st.far_n == 0) {
            st.done = 1;
          } else if (P.mode == VINE_MODE_OPTIMAL && st.inc_key != ~0ull && fmin > key_d(st.inc_key)) {
            st.done = 1;
          } else {
            st.lo = fmaxf(bucket_hi(st), fmin);
            float hi = st.lo + st.width;
            if (!(hi > st.lo)) hi = nextafterf(st.lo, INFINITY);
            st.hi_bits = __float_as_uint(hi);
          }
          st.far_min_bits = kInfBits;
          st.far_wpos = 0;
          st.rb_count = 0;
          st.b_labels = st.b_expanded = st.b_rounds = st.b_dominated = 0;
          st.b_candidates = st.b_spilled = st.b_relaxed = 0;
        }
        __syncthreads();
        if (st.done) break;
        // ---- split the far pile: labels below hi enter the bucket
        const uint32_t fn = st.far_n;
        for (uint32_t base = 0; base < fn; base += (uint32_t)G) {
          if (tid == 0) pool_reserve(P, st, (uint32_t)G);
          __syncthreads();
          if (st.abort) break;
          const uint32_t i = base + tid;
          Label item;
          const bool valid = i < fn;
          if (valid) item = c.far[i];
          __syncthreads();  // the whole tile is read before it is overwritten
          if (valid) {
            const bool keep = offer(c, item.vid, item.d, item.dl, (uint32_t)item.parent, true);
            if (keep) {
              const uint32_t w = warp_agg_inc(&st.far_wpos);
              c.far[w] = item;
              float hl = 0.0f;
              if (P.use_bounds) hl = load_vs(&c.vs[item.vid]).hlen;
              atomicMin(&st.far_min_bits, __float_as_uint(item.d + hl));
            }
          }
        }
        __syncthreads();
        if (tid == 0) st.far_n = st.far_wpos;
        __syncthreads();
        continue;
      }

      // ---- one expansion round over up to split_cap near labels
      const int n_round = (int)min((uint32_t)min(RC, st.split_cap), avail);
      for (int i = tid; i < n_round; i += G) {
        const uint32_t idx = c.nearq[(st.near_head + (uint32_t)i) & P.near_mask];
        const Label lab = load_label(&P.pool[idx]);
        int deg = 0;
        const int v = lab.vid & 0x7fffffff;
        bool live = !(lab.vid & (int)kDeadBit);
        if (live) {
          float hl = 0.0f, hd = 0.0f;
          if (P.use_bounds) {
            const VState s = load_vs(&c.vs[v]);
            hl = s.hlen;
            hd = s.hdel;
          }
          // split off by a bucket split: it returns to the far pile at the fold
          if (lab.d + hl >= bucket_hi(st)) live = false;
          if (P.mode == VINE_MODE_OPTIMAL) {
            const uint64_t key = pack_key(lab.d + hl, lab.dl + hd);
            if (key >= *reinterpret_cast<volatile unsigned long long *>(&st.inc_key)) live = false;
          }
        }
        int beg = 0;
        if (live) {
          beg = __ldg(&P.g.row[v]);
          deg = __ldg(&P.g.row[v + 1]) - beg;
          if (deg > 0) warp_agg_inc(&st.r_live);
        }
        r_idx[i] = idx;
        r_vid[i] = v;
        r_d[i] = lab.d;
        r_dl[i] = lab.dl;
        r_beg[i] = beg;
        r_off[i] = deg;
      }
      __syncthreads();
      const int total = block_exclusive_scan(r_off, n_round, scan);
      if (tid == 0) {
        st.near_head += (uint32_t)n_round;
        st.n_rounds++;
        st.b_rounds++;
        if (st.n_rounds > kMaxRounds) st.abort = VINE_ERR_TIMEOUT;  // hard progress bound
        st.n_expanded += st.r_live;
        st.b_expanded += st.r_live;
        st.r_live = 0;
        st.n_relaxed += total;
        st.b_relaxed += (uint32_t)total;
        pool_reserve(P, st, (uint32_t)total);
      }
      __syncthreads();
      if (st.abort) break;
      for (int e = tid; e < total; e += G) {
        const int k = upper_index(r_off, n_round, e);
        const int j = r_beg[k] + (e - r_off[k]);
        const int v = __ldg(&P.g.col[j]);
        const float2 w = __ldg(&P.g.w[j]);
        offer(c, v, r_d[k] + w.x, r_dl[k] + w.y, r_idx[k], false);
      }
      __syncthreads();
    }
    __syncthreads();

    // ------------------------------------------------------------- finish
    // fold thread-local counters and clear what the query left in the table
    atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
    atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
    atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
    c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
    for (int i = tid; i < H; i += G) table[i].vid = kEmpty;
    {
      const uint32_t sc = st.s_count;
      for (uint32_t i = tid; i < sc; i += G) c.bt.s[c.bt.s_used[i]].vid = kEmpty;
    }
    if (P.mode == VINE_MODE_PARETO && !st.abort) {
      // alive sink labels are exactly the sink's Pareto set; rank-sort them
      const uint32_t k = min(st.sink_n, (uint32_t)P.sink_cap);
      __syncthreads();
      uint32_t alive_local = 0;
      for (uint32_t i = tid; i < k; i += G) {
        const Label a = load_label(&P.pool[c.sinks[i]]);
        if (a.vid & (int)kDeadBit) continue;
        ++alive_local;
        const uint64_t ka = pack_key(a.d, a.dl);
        int rank = 0;
        for (uint32_t j = 0; j < k; ++j) {
          const Label b = load_label(&P.pool[c.sinks[j]]);
          if (b.vid & (int)kDeadBit) continue;
          if (pack_key(b.d, b.dl) < ka) ++rank;
        }
        if (rank < P.pareto_stride && P.pareto_d) {
          P.pareto_d[(size_t)q * P.pareto_stride + rank] = a.d;
          P.pareto_dl[(size_t)q * P.pareto_stride + rank] = a.dl;
        }
        if (rank == 0) {
          st.inc_key = ka;
          st.inc_idx = c.sinks[i];
        }
      }
      __syncthreads();
      if (tid == 0) st.sink_n = 0;
      __syncthreads();
      atomicAdd(&st.sink_n, alive_local);
    }
    __syncthreads();
    if (tid == 0) {
      const bool ok = st.abort == 0;
      const bool found = ok && st.inc_key != ~0ull;
      P.status[q] = ok ? VINE_OK : st.abort;
      P.found[q] = found ? 1 : 0;
      P.cost[q] = found ? key_d(st.inc_key) : INFINITY;
      P.odelay[q] = found ? key_dl(st.inc_key) : INFINITY;
      P.best_idx[q] = found ? (int32_t)st.inc_idx : -1;
      if (P.pareto_n) P.pareto_n[q] = (P.mode == VINE_MODE_PARETO && ok) ? (int32_t)st.sink_n : 0;
      if (P.stats) {
        int64_t *s = P.stats + (size_t)q * VINE_STAT_COUNT;
        s[VINE_STAT_EXPANDED] = st.n_expanded;
        s[VINE_STAT_RELAXED] = st.n_relaxed;
        s[VINE_STAT_INSERTED] = st.n_inserted;
        s[VINE_STAT_DOMINATED] = st.n_dominated;
        s[VINE_STAT_BUCKETS] = st.n_buckets;
        s[VINE_STAT_ROUNDS] = st.n_rounds;
        s[VINE_STAT_SPILLS] = st.n_spills;
        s[VINE_STAT_CYCLES] = clock64() - st.t0;
      }
      st.s_count = 0;
    }
    __syncthreads();
  }
}

// Orders queries by decreasing budget class (floor(log2(budget + 1))), a
// cheap proxy for query difficulty: the longest queries start first.
__global__ void order_kernel(int32_t nq, const float *budget, int32_t *order) {
  __shared__ int hist[64];
  __shared__ int base[64];
  for (int i = threadIdx.x; i < 64; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < nq; i += blockDim.x) {
    const float b = budget[i];
    int cls = (b > 0.0f && isfinite(b)) ? min(63, (int)log2f(b + 1.0f)) : 0;
    atomicAdd(&hist[63 - cls], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int i = 0; i < 64; ++i) {
      base[i] = run;
      run += hist[i];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nq; i += blockDim.x) {
    const float b = budget[i];
    int cls = (b > 0.0f && isfinite(b)) ? min(63, (int)log2f(b + 1.0f)) : 0;
    order[atomicAdd(&base[63 - cls], 1)] = i;
  }
}

__global__ void path_len_kernel(const Label *pool, int32_t nq, const int32_t *best,
                                int64_t *len) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  int64_t n = 0;
  for (int32_t k = best[q]; k >= 0; k = __ldcg(&pool[k].parent)) ++n;
  len[q] = n;
}

// In-place exclusive scan of n int64 values by one block (n may be large).
__global__ void scan_i64_kernel(int64_t *a, int32_t n) {
  __shared__ int64_t warp_tot[32];
  __shared__ int64_t carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, G = blockDim.x;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int32_t base = 0; base < n; base += G) {
    const int32_t i = base + tid;
    const int64_t x = i < n ? a[i] : 0;
    int64_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int64_t v = lane < (G >> 5) ? warp_tot[lane] : 0;
      int64_t vi = v;
      for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, vi, o);
        if (lane >= o) vi += y;
      }
      if (lane < (G >> 5)) warp_tot[lane] = vi - v;
    }
    __syncthreads();
    const int64_t excl = carry + warp_tot[warp] + incl - x;
    if (i < n) a[i] = excl;
    __syncthreads();
    if (tid == G - 1) carry = excl + x;
    __syncthreads();
  }
  if (tid == 0) a[n] = carry;
}

__global__ void path_write_kernel(const Label *pool, int32_t nq, const int32_t *best,
                                  const int64_t *off, int32_t *path) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  int64_t pos = off[q + 1] - 1;
  for (int32_t k = best[q]; k >= 0; k = __ldcg(&pool[k].parent)) {
    path[pos--] = __ldcg(&pool[k].vid) & 0x7fffffff;
  }
}

size_t batch_smem_bytes(int table_log2, int lock_log2, int round_cap) {
  size_t b = (sizeof(TEntry) << table_log2) + (sizeof(int) << lock_log2) +
             (size_t)round_cap * 24 + kScanScratch * sizeof(int);
  b = (b + 15) & ~(size_t)15;
  return b + sizeof(CtaState) + 16;
}

}  // namespace

void BatchWorkspace::release() {
  cudaFree(vs);
  cudaFree(nearq);
  cudaFree(far);
  cudaFree(spill);
  cudaFree(spill_used);
  cudaFree(rebuild);
  cudaFree(retry);
  cudaFree(sinklist);
  cudaFree(pool);
  cudaFree(counters);
  cudaFree(best_idx);
  cudaFree(order);
  cudaFree(trace);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  *this = BatchWorkspace();
}

static int lock_log2_for(int table_log2) { return std::max(5, table_log2 - 1); }

static int ensure_batch_workspace(vine_graph *g, const Resolved &r, int32_t nq) {
  BatchWorkspace &w = g->batch;
  const vine_config &c = r.cfg;
  const int64_t spill_n = int64_t(1) << c.spill_log2;
  const uint32_t spill_limit = (uint32_t)(spill_n * 3 / 4);
  int64_t near_need = (int64_t(1) << c.table_log2) + spill_limit + 1;
  int64_t near_cap = 1;
  while (near_cap < near_need) near_cap <<= 1;
  const int sink_cap = 4096;
  const bool same = w.slots == r.slots && w.block_threads == c.block_threads &&
                    w.table_log2 == c.table_log2 && w.spill_log2 == c.spill_log2 &&
                    w.far_cap == c.far_capacity && w.near_cap == near_cap &&
                    w.pool_cap == c.pool_labels;
  if (!same) {
    w.release();
    const size_t n = (size_t)g->n;
    VINE_CUDA_TRY(cudaMalloc(&w.vs, sizeof(VState) * n * r.slots));
    VINE_CUDA_TRY(cudaMemset(w.vs, 0, sizeof(VState) * n * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.nearq, sizeof(uint32_t) * (size_t)near_cap * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.far, sizeof(Label) * (size_t)c.far_capacity * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.spill, sizeof(TEntry) * (size_t)spill_n * r.slots));
    VINE_CUDA_TRY(cudaMemset(w.spill, 0xff, sizeof(TEntry) * (size_t)spill_n * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.spill_used, sizeof(uint32_t) * (size_t)spill_limit * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.rebuild, sizeof(TEntry) * (((size_t)1 << c.table_log2) + spill_limit) * r.slots));
    w.retry_cap = 1 << 16;
    VINE_CUDA_TRY(cudaMalloc(&w.retry, sizeof(Label) * 2 * (size_t)w.retry_cap * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.sinklist, sizeof(uint32_t) * (size_t)sink_cap * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.pool, sizeof(Label) * (size_t)c.pool_labels));
    VINE_CUDA_TRY(cudaMalloc(&w.counters, sizeof(unsigned long long) * 8));
    w.slots = r.slots;
    w.block_threads = c.block_threads;
    w.table_log2 = c.table_log2;
    w.spill_log2 = c.spill_log2;
    w.far_cap = c.far_capacity;
    w.near_cap = near_cap;
    w.sink_cap = sink_cap;
    w.pool_cap = c.pool_labels;
    w.epoch_next = 1;
  }
  if (w.q_cap < nq) {
    cudaFree(w.best_idx);
    cudaFree(w.order);
    w.best_idx = nullptr;
    w.order = nullptr;
    const int64_t cap = std::max<int64_t>(nq, 1024);
    VINE_CUDA_TRY(cudaMalloc(&w.best_idx, sizeof(int32_t) * (size_t)cap));
    VINE_CUDA_TRY(cudaMalloc(&w.order, sizeof(int32_t) * (size_t)cap));
    w.q_cap = cap;
  }
  if (c.trace && w.trace == nullptr) {
    w.trace_cap = 1 << 20;
    VINE_CUDA_TRY(cudaMalloc(&w.trace, sizeof(float) * 20 * (size_t)w.trace_cap));
  }
  return VINE_OK;
}

int batch_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
              const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
              cudaStream_t stream, Label **pool_out) {
  const vine_config &c = r.cfg;
  VINE_TRY(ensure_batch_workspace(g, r, nq));
  BatchWorkspace &w = g->batch;
  if (w.epoch_next > 0xF0000000u - (uint32_t)nq) {
    VINE_CUDA_TRY(cudaMemsetAsync(w.vs, 0, sizeof(VState) * (size_t)g->n * w.slots, stream));
    w.epoch_next = 1;
  }
  BatchParams P;
  std::memset(&P, 0, sizeof(P));
  P.g = g->dev();
  P.nq = nq;
  P.src = d_src;
  P.dst = d_dst;
  P.budget = d_budget;
  P.order = c.order_queries ? w.order : nullptr;
  P.cost = out.cost;
  P.odelay = out.delay;
  P.found = out.found;
  P.status = out.status;
  P.stats = out.stats;
  P.pareto_d = out.pareto_d;
  P.pareto_dl = out.pareto_delay;
  P.pareto_n = out.pareto_n;
  P.pareto_stride = out.pareto_stride;
  P.best_idx = out.best_idx ? out.best_idx : w.best_idx;
  P.vs = w.vs;
  P.nearq = w.nearq;
  P.near_mask = (uint32_t)(w.near_cap - 1);
  P.far = w.far;
  P.far_cap = w.far_cap;
  P.spill = w.spill;
  P.spill_used = w.spill_used;
  P.spill_log2 = c.spill_log2;
  P.spill_limit = (uint32_t)(((int64_t)1 << c.spill_log2) * 3 / 4);
  P.sinklist = w.sinklist;
  P.rebuild = w.rebuild;
  P.retry = w.retry;
  P.retry_cap = (uint32_t)w.retry_cap;
  P.sink_cap = w.sink_cap;
  P.pool = w.pool;
  P.pool_top = w.counters + 0;
  P.pool_cap = w.pool_cap;
  P.chunk = 1u << 14;
  P.queue = w.counters + 1;
  P.epoch_base = w.epoch_next;
  P.mode = c.mode;
  P.policy = c.policy;
  P.use_bounds = c.use_bounds;
  P.width0 = r.width0;
  P.round_cap = r.round_cap;
  P.table_log2 = c.table_log2;
  P.lock_log2 = lock_log2_for(c.table_log2);
  P.probe = 16;
  P.mlp = (c.policy == VINE_POLICY_MLP && c.mlp) ? c.mlp->params : nullptr;
  P.trace = c.trace ? w.trace : nullptr;
  P.trace_top = w.counters + 3;
  P.trace_cap = w.trace_cap;
  w.epoch_next += (uint32_t)nq;

  const size_t smem = batch_smem_bytes(c.table_log2, P.lock_log2, r.round_cap);
  VINE_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  VINE_CUDA_TRY(cudaMemsetAsync(w.counters, 0, sizeof(unsigned long long) * 8, stream));
  if (c.order_queries && nq > 0) order_kernel<<<1, 1024, 0, stream>>>(nq, d_budget, w.order);
  batch_kernel<<<r.slots, c.block_threads, smem, stream>>>(P);
  VINE_CUDA_TRY(cudaGetLastError());
  if (pool_out) *pool_out = w.pool;
  return VINE_OK;
}

int batch_slots(const vine_graph *g, const vine_config &c, int round_cap, int *slots) {
  const size_t smem = batch_smem_bytes(c.table_log2, lock_log2_for(c.table_log2), round_cap);
  VINE_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  int per_sm = 0;
  VINE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel,
                                                              c.block_threads, smem));
  if (per_sm < 1) return fail(VINE_ERR_INVALID, "batch kernel does not fit on an SM with this configuration");
  if (c.ctas_per_sm > 0) per_sm = std::min(per_sm, c.ctas_per_sm);
  *slots = per_sm * g->sm_count;
  return VINE_OK;
}

int path_lengths(const Label *pool, int32_t nq, const int32_t *d_best_idx, int64_t *d_offsets,
                 cudaStream_t stream) {
  if (nq <= 0) {
    VINE_CUDA_TRY(cudaMemsetAsync(d_offsets, 0, sizeof(int64_t), stream));
    return VINE_OK;
  }
  path_len_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(pool, nq, d_best_idx, d_offsets);
  scan_i64_kernel<<<1, 1024, 0, stream>>>(d_offsets, nq);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

int path_write(const Label *pool, int32_t nq, const int32_t *d_best_idx,
               const int64_t *d_offsets, int32_t *d_path, cudaStream_t stream) {
  if (nq <= 0) return VINE_OK;
  path_write_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(pool, nq, d_best_idx, d_offsets,
                                                          d_path);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

}  // namespace vine
