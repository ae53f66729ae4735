// Device search logic shared by the batch engine (one query per CTA, state
// in shared memory) and the plain engine (one query on the whole GPU, state
// in global memory).  All functions take the query state by reference; the
// caller decides where it lives.
//
// Per query:  bounds passes (optional) -> bucket loop { expansion until the
// open bucket is empty (block-synchronous rounds, or warps pulling labels
// from the bucket's ring in the batch engine) -> fold -> scheduler -> open
// the next bucket from the far band / rest pile }.
// Exactness argument: see engine.cuh.  The reference's round structure this
// replaces is RUN_CSPP (algorithm/cspp.cuh:173-296) with
// ck_expand_bucket_with_filter (algorithm/bucket.cuh:15-195),
// second_level_pruning (algorithm/dominance.cuh:15-153), ck_recheck_bucket
// (algorithm/bucket.cuh:217-245) and ck_fill_buckets (bucket.cuh:197-215).
#pragma once

#include "engine.cuh"
#include "../../include/vine.h"

namespace vine {

constexpr int kHist = kBurgMaxN;
constexpr uint32_t kInfBits = 0x7f800000u;
constexpr int kScanScratch = 40;
constexpr long long kMaxRounds = 1ll << 26;  // hard progress bound per query
constexpr int kBins = 64;                    // key bins of the band (binned mode)
constexpr long long kMaxBuckets = 1ll << 22; // hard bound on buckets per query

struct SearchParams {
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
  // workspace (per worker regions are strided by the worker index)
  VState *vs;
  uint32_t *nearq;
  uint32_t near_mask;
  Label *far;        // band pile: keys in [bucket hi, band_hi)
  int64_t far_cap;
  Label *rest;       // keys >= band_hi
  int64_t rest_cap;
  float *far_key;    // key f = d + h(v) of every band / rest pile entry (the
  float *rest_key;   // key is fixed for a query, so rescans need no h lookup)
  int band_mult;     // band width in bucket widths
  uint2 *chunks;     // per worker: arena chunks (base, size) kept across queries
  int max_chunks;
  int32_t *path_arena;  // answer paths copied out at query end
  int64_t path_cap;
  unsigned long long *path_top;
  int64_t *path_start;  // per query
  int32_t *path_len;    // per query
  uint32_t *sinklist;
  int sink_cap;
  uint32_t *bctr;  // per worker: last bucket id used (persists across calls)
  Label *pool;
  uint32_t *next;  // arena-parallel overflow-chain links
  unsigned long long *pool_top;
  int64_t pool_cap;
  uint32_t chunk;
  unsigned long long *queue;
  const unsigned long long *epoch_ptr;  // epoch base of this call (device)
  // configuration
  int mode;
  int policy;
  int use_bounds;
  float width0;
  float ar_scale;   // multiplier on the AR rule's width (AR and MLP policies)
  float len_scale;  // mean arc length: feature normalisation
  float delta_del;
  float delta_len;
  int round_cap;
  int table_log2;
  int lock_log2;
  int probe;
  int grid_scope;  // 1: one query spread over the whole grid (plain engine)
  int sync_rounds; // batch engine: 1 = block-synchronous rounds, 0 = warps pull work
  int binned;      // forward band kept in kBins key bins (batch engine)
  int64_t bin_cap; // labels per bin (far_cap / kBins)
  int split_staging;                 // bucket opening reads tiles through bulk copies
  long long wait_limit;              // polls / lock attempts of a bounded wait
  unsigned long long time_limit_ns;  // per query, 0 = none
  const float *mlp;
  float *trace;
  unsigned long long *trace_top;
  int64_t trace_cap;
};

// State of one query in flight.
struct __align__(16) QueryState {
  unsigned long long inc_key;  // lexicographic (cost, delay) of the incumbent
  long long t0;
  unsigned long long g0;  // global timer at the start of the query (ns)
  long long n_expanded, n_relaxed, n_inserted, n_dominated, n_buckets, n_rounds, n_spills;
  unsigned long long n_chain_steps;
  long long n_bound_rounds, bound_cycles;
  long long split_cycles, split_items, policy_cycles, load_cycles, relax_cycles, rest_items;
  unsigned long long idle_cycles, publish_cycles;
  // arena chunk cursor: fill (low word) and end (high word) of the current
  // chunk, also updated as one 64-bit word when warps reserve concurrently
  uint32_t chunk_fill, chunk_end;
  double hist[kHist];
  int q, src, dst;
  float budget;
  uint32_t epoch;
  uint32_t inc_idx;
  int inc_lock;
  float lo, width;
  float ar_width;  // the AR rule's own width state (before scaling)
  uint32_t hi_bits;  // bucket upper key (float bits)
  uint32_t qbase, bcur;
  uint32_t far_n, far_wpos, far_min_bits;
  uint32_t rest_n, rest_wpos, rest_min_bits;
  float band_hi;
  uint32_t n_chunks, cur_chunk;
  int abort_site;
  int rb_band;
  uint32_t near_head, near_tail;
  uint32_t near_commit;  // ring entries below this are published (async mode)
  uint32_t pending;      // labels of the open bucket not yet fully expanded
  int chunk_lock;
  uint32_t slab_fill[32], slab_end[32];  // per-warp arena slabs (async mode)
  // band bins (binned mode): bin j holds band labels with key in
  // [band_lo + j / bin_inv, band_lo + (j + 1) / bin_inv)
  uint32_t bin_n[kBins], bin_min[kBins], bin_wpos[kBins], bin_pre[kBins + 1];
  float band_lo, bin_inv;
  int bin_last;  // last bin scanned when the open bucket started

  int abort;
  int done;
  int tile_broken;  // a staged tile's copy never landed: the worker stops
  int split_cap;
  int hist_n;
  uint32_t sink_n;
  uint32_t b_labels, b_expanded, b_rounds, b_dominated, b_candidates, b_spilled, b_relaxed;
  uint32_t r_live;
  float x_prev[kFeat];
  float x[kFeat];
  float mh[2 * kHid];
  float y[kOut];
};

__device__ __forceinline__ float bucket_hi(const QueryState &st) {
  return __uint_as_float(*reinterpret_cast<const volatile uint32_t *>(&st.hi_bits));
}

__device__ __forceinline__ Label load_label(const Label *p) {
  const int4 raw = __ldcg(reinterpret_cast<const int4 *>(p));
  Label l;
  l.vid = raw.x;
  l.d = __int_as_float(raw.y);
  l.dl = __int_as_float(raw.z);
  l.parent = raw.w;
  return l;
}

// Shared-memory (batch) or global (plain) arrays of one expansion round.
struct RoundBuf {
  uint32_t *idx;
  int *vid;
  float *d;
  float *dl;
  int *beg;
  int *off;
  int *scan;
  int cap;
};

struct Ctx {
  const SearchParams &P;
  QueryState &st;
  BucketTable bt;
  VState *vs;
  uint32_t *nearq;
  Label *far;
  Label *rest;
  float *far_key = nullptr;   // keys beside the band bins (batch engine)
  float *rest_key = nullptr;  // keys beside the rest pile (batch engine)
  uint32_t *sinks;
  uint32_t c_dominated = 0, c_near = 0, c_far = 0, c_spills = 0, c_candidates = 0;
  unsigned long long c_idle = 0, c_publish = 0;  // warps-pull waits (lane 0 of each warp)
  // async mode: arena slots come from this warp's slab (slab_fill points at
  // its fill counter; the slab always has room for the 32 arcs in flight)
  uint32_t *slab_fill = nullptr;
  __device__ Ctx(const SearchParams &p, QueryState &s) : P(p), st(s) {}
  // One arena slot (kBadIdx when the arena is exhausted).
  __device__ __forceinline__ uint32_t alloc_one();
  __device__ VView view(int v) const {
    return view_vs(&vs[v], st.epoch, st.qbase, st.bcur, P.use_bounds != 0);
  }
  // Forward-search ring entries: (arena index, vertex).  The reverse bound
  // searches use the same memory as a ring of vertex ids.
  __device__ __forceinline__ uint2 *near_ring() const { return reinterpret_cast<uint2 *>(nearq); }
};

__device__ __forceinline__ float key_of(const Ctx &c, int32_t vid, float d) {
  return c.P.use_bounds ? d + c.view(vid).hlen : d;
}

// Records the first failure of the query (status + where it happened).
__device__ __forceinline__ void fail_query(QueryState &st, int status, int site) {
  if (atomicCAS(&st.abort, 0, status) == 0) st.abort_site = site;
}

enum AbortSite {
  kSiteArena = 1, kSiteArenaAlloc = 2, kSiteNear = 3, kSiteBand = 4, kSiteRest = 5,
  kSiteSink = 6, kSiteLock = 7, kSiteRounds = 8, kSitePath = 9, kSiteChunks = 10,
  kSiteInvalid = 11, kSiteAsync = 12, kSiteTime = 13, kSiteRing = 14, kSiteTile = 15
};  // the values of enum vine_abort_site (vine.h)

// Device global timer in nanoseconds.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// True (and the query failed with VINE_ERR_TIMEOUT) once the query has run
// longer than its time limit.
__device__ __forceinline__ bool over_time(const SearchParams &P, QueryState &st) {
  if (P.time_limit_ns == 0) return false;
  if (global_ns() - st.g0 <= P.time_limit_ns) return false;
  fail_query(st, VINE_ERR_TIMEOUT, kSiteTime);
  return true;
}

// Next arena chunk with room for `need` labels: a kept chunk of the worker
// (reused across its queries) or a new one from the global arena.  Caller has
// exclusive use of the chunk list (one thread between barriers, or the
// chunk lock).  Returns false (query failed) when the arena is exhausted.
__device__ inline bool next_chunk(const SearchParams &P, QueryState &st, uint32_t need,
                                  uint32_t *base, uint32_t *size) {
  uint2 *list = P.chunks + (size_t)blockIdx.x * P.max_chunks;
  while (st.cur_chunk + 1 < st.n_chunks) {  // a kept chunk that is large enough
    const uint2 ch = list[++st.cur_chunk];
    if (ch.y >= need) {
      *base = ch.x;
      *size = ch.y;
      return true;
    }
  }
  if ((int)st.n_chunks >= P.max_chunks) {
    fail_query(st, VINE_ERR_CAPACITY, kSiteChunks);
    return false;
  }
  const uint64_t sz = need > P.chunk ? need : P.chunk;
  const unsigned long long b = atomicAdd(P.pool_top, (unsigned long long)sz);
  if (b + sz > (unsigned long long)P.pool_cap) {
    fail_query(st, VINE_ERR_CAPACITY, kSiteArena);
    return false;
  }
  list[st.n_chunks] = make_uint2((uint32_t)b, (uint32_t)sz);
  st.cur_chunk = st.n_chunks++;
  *base = (uint32_t)b;
  *size = (uint32_t)sz;
  return true;
}

// Makes sure the current arena chunk has room for `need` more labels (one
// thread, between barriers).  A batch worker keeps the chunks it was given in
// a list and reuses them for its next queries (its answer paths are copied
// out at the end of each query), so the arena holds one query per worker.
__device__ inline void pool_reserve(const SearchParams &P, QueryState &st, uint32_t need) {
  if ((uint64_t)st.chunk_fill + need <= (uint64_t)st.chunk_end) return;
  uint32_t base = 0, size = 0;
  if (!next_chunk(P, st, need, &base, &size)) {
    st.chunk_fill = st.chunk_end = 0;
    return;
  }
  st.chunk_fill = base;
  st.chunk_end = base + size;
}

// Reserves `need` consecutive arena slots while other warps of the block do
// the same (async mode): a compare-and-swap on the (fill, end) word of the
// current chunk; the one warp that finds the chunk exhausted moves the worker
// to its next chunk under the chunk lock.  Returns the first slot, or kBadIdx
// when the query failed.
__device__ inline uint32_t arena_take(const SearchParams &P, QueryState &st, uint32_t need) {
  unsigned long long *pk = reinterpret_cast<unsigned long long *>(&st.chunk_fill);
  for (long long it = 0; it < P.wait_limit; ++it) {
    if (*reinterpret_cast<volatile int *>(&st.abort)) return kBadIdx;
    const unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(pk);
    const uint32_t fill = (uint32_t)old, end = (uint32_t)(old >> 32);
    if ((uint64_t)fill + need <= (uint64_t)end) {
      if (atomicCAS(pk, old, old + need) == old) return fill;
      continue;
    }
    uint32_t got = kBadIdx;
    bool retry = false;
    const bool locked = with_lock(&st.chunk_lock, [&]() {
      const unsigned long long cur = *reinterpret_cast<volatile unsigned long long *>(pk);
      if ((uint64_t)(uint32_t)cur + need <= (uint64_t)(uint32_t)(cur >> 32)) {
        retry = true;  // another warp switched chunks meanwhile
        return;
      }
      uint32_t base = 0, size = 0;
      if (!next_chunk(P, st, need, &base, &size)) return;
      atomicExch(pk, ((unsigned long long)(base + size) << 32) | (unsigned long long)(base + need));
      got = base;
    }, false, P.wait_limit);
    if (!locked) {
      fail_query(st, VINE_ERR_TIMEOUT, kSiteLock);
      return kBadIdx;
    }
    if (!retry) return got;
  }
  fail_query(st, VINE_ERR_TIMEOUT, kSiteArena);
  return kBadIdx;
}

__device__ __forceinline__ uint32_t Ctx::alloc_one() {
  if (slab_fill) return atomicAdd(slab_fill, 1u);
  const uint32_t i = atomicAdd(&st.chunk_fill, 1u);
  return i < *reinterpret_cast<volatile uint32_t *>(&st.chunk_end) ? i : kBadIdx;
}

// Rewinds the worker's arena to its first kept chunk (start of a query).
__device__ inline void pool_rewind(const SearchParams &P, QueryState &st) {
  if (st.n_chunks == 0) {
    st.chunk_fill = st.chunk_end = 0;
    st.cur_chunk = 0;
    return;
  }
  const uint2 ch = P.chunks[(size_t)blockIdx.x * P.max_chunks];
  st.cur_chunk = 0;
  st.chunk_fill = ch.x;
  st.chunk_end = ch.x + ch.y;
}

// Copies the answer's path (source .. sink) out of the arena into the path
// arena (one thread).  Two walks of the parent chain: count, then write.
__device__ inline void copy_out_path(const SearchParams &P, QueryState &st, int q, bool found) {
  P.path_len[q] = 0;
  P.path_start[q] = 0;
  if (!found || P.path_arena == nullptr) return;
  int32_t n = 0;
  for (int32_t k = (int32_t)st.inc_idx; k >= 0; k = __ldcg(&P.pool[k].parent)) ++n;
  const unsigned long long base = atomicAdd(P.path_top, (unsigned long long)n);
  if (base + n > (unsigned long long)P.path_cap) {
    fail_query(st, VINE_ERR_CAPACITY, kSitePath);
    return;
  }
  int64_t pos = (int64_t)base + n - 1;
  for (int32_t k = (int32_t)st.inc_idx; k >= 0; k = __ldcg(&P.pool[k].parent))
    P.path_arena[pos--] = __ldcg(&P.pool[k].vid) & 0x7fffffff;
  P.path_start[q] = (int64_t)base;
  P.path_len[q] = n;
}

// Sink label that beats the incumbent (optimal mode): stored in the arena and
// published under a small lock so that key and arena index stay paired.
__device__ __forceinline__ void sink_improve(Ctx &c, int32_t v, float nd, float ndl, uint32_t parent,
                             uint64_t key) {
  QueryState &st = c.st;
  const uint32_t idx = c.alloc_one();
  if (idx == kBadIdx) {
    fail_query(st, VINE_ERR_CAPACITY, kSiteArenaAlloc);
    return;
  }
  c.P.pool[idx] = Label{v, nd, ndl, (int32_t)parent};
  const bool ok = with_lock(&st.inc_lock, [&]() {
    volatile unsigned long long *ik = &st.inc_key;
    if (key < *ik) {
      *ik = key;
      st.inc_idx = idx;
    }
  }, c.P.grid_scope != 0, c.P.wait_limit);
  if (!ok) fail_query(st, VINE_ERR_TIMEOUT, kSiteLock);
}


// Files a label beyond the open bucket: into the band pile when its key is
// below band_hi, else into the rest pile.
// Bin of key f in the band (monotone in f, clamped to [0, kBins)).
__device__ __forceinline__ int band_bin(const QueryState &st, float f) {
  const float x = (f - st.band_lo) * st.bin_inv;
  return x > 0.0f ? min(kBins - 1, (int)x) : 0;
}

// Files a band label (f < band_hi) into its bin; false when the bin is full.
__device__ __forceinline__ bool push_bin(Ctx &c, const Label &l, float f) {
  namespace cg = cooperative_groups;
  QueryState &st = c.st;
  const int j = band_bin(st, f);
  cg::coalesced_group act = cg::coalesced_threads();
  cg::coalesced_group grp = cg::labeled_partition(act, j);
  uint32_t base = 0;
  if (grp.thread_rank() == 0) base = atomicAdd(&st.bin_n[j], grp.size());
  const uint32_t pos = grp.shfl(base, 0) + grp.thread_rank();
  if (pos >= (uint64_t)c.P.bin_cap) return false;
  const size_t at = (size_t)j * (size_t)c.P.bin_cap + pos;
  c.far[at] = l;
  c.far_key[at] = f;
  atomicMin(&st.bin_min[j], __float_as_uint(f));
  return true;
}

__device__ __forceinline__ void push_far(Ctx &c, const Label &l, float f) {
  QueryState &st = c.st;
  // binned band: a full bin sends the label to the rest pile, which is
  // rescanned when a bucket opens while its minimum lies below band_hi
  if (c.P.binned && f < st.band_hi && push_bin(c, l, f)) return;
  if (!c.P.binned && f < st.band_hi) {
    const uint32_t pos = warp_agg_inc(&st.far_n);
    if (pos >= (uint64_t)c.P.far_cap) {
      fail_query(st, VINE_ERR_CAPACITY, kSiteBand);
      return;
    }
    c.far[pos] = l;
    atomicMin(&st.far_min_bits, __float_as_uint(f));
  } else {
    const uint32_t pos = warp_agg_inc(&st.rest_n);
    if (pos >= (uint64_t)c.P.rest_cap) {
      fail_query(st, VINE_ERR_CAPACITY, kSiteRest);
      return;
    }
    c.rest[pos] = l;
    if (c.rest_key) c.rest_key[pos] = f;
    atomicMin(&st.rest_min_bits, __float_as_uint(f));
  }
}

// Offers one label (v, nd, ndl) to the search, given v's state view s.
// from_far = true when it comes from the far pile (budget already checked);
// returns true when a far label must stay in the far pile.  A label accepted
// into the open bucket is queued on the near ring, or, when near_out is given,
// its arena index is returned there for the caller to queue.
__device__ __forceinline__ bool offer_with(Ctx &c, int32_t v, float nd, float ndl, uint32_t parent,
                                  bool from_far, const VView &s, uint32_t *near_out = nullptr) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  if (!s.reach) return false;  // no feasible completion from v (bounds mode)
  const float lb_dl = ndl + s.hdel;
  if (!from_far) {
    c.c_candidates++;
    if (lb_dl > st.budget) return false;  // include/constraint.hpp:99-101
  }
  if (ndl >= s.sdel) {  // dominated by a label of a finished bucket
    c.c_dominated++;
    return false;
  }
  const float f = nd + s.hlen;
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
    auto alloc = [&c, pool, v, nd, ndl, parent]() -> uint32_t {
      const uint32_t i = c.alloc_one();
      if (i != kBadIdx) pool[i] = Label{v, nd, ndl, (int32_t)parent};
      return i;
    };
    const InsertResult r =
        table_insert(c.bt, P.pool, v, nd, ndl, alloc, &idx, &spilled, P.grid_scope != 0);
    if (r == kDominated) {
      c.c_dominated++;
      return false;
    }
    if (r != kInserted) {
      if (r == kLockTimeout) fail_query(st, VINE_ERR_TIMEOUT, kSiteLock);
      else fail_query(st, VINE_ERR_CAPACITY, kSiteArenaAlloc);
      return false;
    }
    c.c_near++;
    if (spilled) c.c_spills++;
    if (near_out) {
      *near_out = idx;
    } else {
      const uint32_t pos = warp_agg_inc(&st.near_tail);
      if (pos - *reinterpret_cast<volatile uint32_t *>(&st.near_head) > P.near_mask) {
        fail_query(st, VINE_ERR_CAPACITY, kSiteNear);  // the open bucket outgrew the ring
        return false;
      }
      c.near_ring()[pos & P.near_mask] = make_uint2(idx, (uint32_t)v);
    }
    if (P.mode == VINE_MODE_PARETO && v == st.dst) {
      const uint32_t k = atomicAdd(&st.sink_n, 1u);
      if (k < (uint32_t)P.sink_cap) c.sinks[k] = idx;
      else fail_query(st, VINE_ERR_CAPACITY, kSiteSink);
    }
    return false;
  }
  if (from_far) return true;
  push_far(c, Label{v, nd, ndl, (int32_t)parent}, f);
  c.c_far++;
  return false;
}

__device__ __forceinline__ bool offer(Ctx &c, int32_t v, float nd, float ndl, uint32_t parent, bool from_far) {
  return offer_with(c, v, nd, ndl, parent, from_far, c.view(v));
}

// Items per thread whose independent global loads are issued together before
// any of them is used (hides HBM latency on the sparse gathers of a round).
constexpr int kBatch = 4;

// Expands near-queue items [first, first + n) with the calling block
// (n <= rb.cap): loads the labels, prefix-sums their out-degrees, then every
// thread relaxes one arc at a time (load-balanced search over the round),
// keeping all lanes busy for degree-2 road vertices and power-law hubs alike.
__device__ __forceinline__ void expand_block(Ctx &c, const RoundBuf &rb, uint32_t first, int n) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const int tid = threadIdx.x, G = blockDim.x;
  const int sid = spread_index(tid, G);
  const float hi = bucket_hi(st);
  const long long t_load = clock64();
  for (int i0 = sid; i0 < n; i0 += G * kBatch) {
    uint32_t idx[kBatch];
    Label lab[kBatch];
    VView s[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int i = i0 + b * G;
      idx[b] = i < n ? c.near_ring()[(first + (uint32_t)i) & P.near_mask].x : 0u;
      if ((uint64_t)idx[b] >= (uint64_t)P.pool_cap) {  // protocol slip: fail, do not follow
        fail_query(st, VINE_ERR_INTERNAL, kSiteRing);
        idx[b] = 0u;
      }
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (i0 + b * G < n) lab[b] = load_label(&P.pool[idx[b]]);
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (i0 + b * G < n && (uint32_t)(lab[b].vid & 0x7fffffff) >= (uint32_t)P.g.n) {
        fail_query(st, VINE_ERR_INTERNAL, kSiteRing);
        lab[b].vid = (int)kDeadBit;  // vertex 0, dead: expands nothing
      }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      s[b] = VView{0.0f, true, 0.0f, 0.0f, 0u};
      if (P.use_bounds && i0 + b * G < n) s[b] = c.view(lab[b].vid & 0x7fffffff);
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int i = i0 + b * G;
      if (i >= n) break;
      const int v = lab[b].vid & 0x7fffffff;
      bool live = !(lab[b].vid & (int)kDeadBit);
      int beg = 0, deg = 0;
      if (live) {
        const float f = lab[b].d + s[b].hlen;
        if (!(f < hi)) live = false;
        if (live && P.mode == VINE_MODE_OPTIMAL) {
          const uint64_t key = pack_key(f, lab[b].dl + s[b].hdel);
          if (key >= *reinterpret_cast<volatile unsigned long long *>(&st.inc_key)) live = false;
        }
      }
      if (live) {
        beg = __ldg(&P.g.row[v]);
        deg = __ldg(&P.g.row[v + 1]) - beg;
        if (deg > 0) warp_agg_inc(&st.r_live);
      }
      rb.idx[i] = idx[b];
      rb.vid[i] = v;
      rb.d[i] = lab[b].d;
      rb.dl[i] = lab[b].dl;
      rb.beg[i] = beg;
      rb.off[i] = deg;
    }
  }
  __syncthreads();
  const int total = block_exclusive_scan(rb.off, n, rb.scan);
  if (tid == 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_relaxed), (unsigned long long)total);
    atomicAdd(&st.b_relaxed, (uint32_t)total);
    // one arena slot per arc at most (batch engine: one arena chunk per CTA)
    if (!P.grid_scope) pool_reserve(P, st, (uint32_t)total);
  }
  if (!P.grid_scope) {
    __syncthreads();
    if (st.abort) return;
  }
  const long long t_relax = clock64();
  if (tid == 0 && !P.grid_scope) st.load_cycles += t_relax - t_load;
  for (int e0 = sid; e0 < total; e0 += G * kBatch) {
    int vv[kBatch];
    float nd[kBatch], nl[kBatch];
    uint32_t par[kBatch];
    VView s[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int e = e0 + b * G;
      vv[b] = -1;
      if (e < total) {
        const int k = upper_index(rb.off, n, e);
        const int j = rb.beg[k] + (e - rb.off[k]);
        vv[b] = __ldg(&P.g.col[j]);
        const float2 w = __ldg(&P.g.w[j]);
        nd[b] = rb.d[k] + w.x;
        nl[b] = rb.dl[k] + w.y;
        par[b] = rb.idx[k];
      }
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (vv[b] >= 0) s[b] = c.view(vv[b]);
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (vv[b] >= 0) offer_with(c, vv[b], nd[b], nl[b], par[b], false, s[b]);
  }
  __syncthreads();
  if (tid == 0 && !P.grid_scope) st.relax_cycles += clock64() - t_relax;
}

// Reverse (sink-rooted) bounded single-criterion search, one round over
// near items [first, first + n) with the calling block.  which = 0: delay
// distance up to `radius` (the budget); which = 1: length distance over the
// vertices the delay pass reached.  Distances live in VState; improved
// vertices go to the near ring (key < hi and ring_ok) or the far pile.
__device__ inline void reverse_expand_block(Ctx &c, const RoundBuf &rb, int which, uint32_t first, int n,
                                     float radius, float hi, bool ring_ok) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const int tid = threadIdx.x, G = blockDim.x;
  const int sid = spread_index(tid, G);
  for (int i = sid; i < n; i += G) {
    const int v = (int)c.nearq[(first + (uint32_t)i) & P.near_mask];
    const int beg = __ldg(&P.g.rrow[v]);
    const VView s = view_vs(&c.vs[v], st.epoch, st.qbase, st.bcur, true);
    rb.vid[i] = v;
    rb.d[i] = which == 0 ? s.hdel : s.hlen;
    rb.beg[i] = beg;
    rb.off[i] = __ldg(&P.g.rrow[v + 1]) - beg;
  }
  __syncthreads();
  const int total = block_exclusive_scan(rb.off, n, rb.scan);
  if (tid == 0)
    atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_relaxed), (unsigned long long)total);
  // every arc may push one entry: use the ring only if it can take them all
  const bool use_ring = ring_ok && (*reinterpret_cast<volatile uint32_t *>(&st.near_tail) -
                                    *reinterpret_cast<volatile uint32_t *>(&st.near_head)) +
                                           (uint32_t)total < P.near_mask;
  for (int e = sid; e < total; e += G) {
    const int k = upper_index(rb.off, n, e);
    const int j = rb.beg[k] + (e - rb.off[k]);
    const int u = __ldg(&P.g.rcol[j]);
    const float2 w = __ldg(&P.g.rw[j]);
    const float nd = rb.d[k] + (which == 0 ? w.y : w.x);
    if (nd > radius) continue;
    VState *su = &c.vs[u];
    bool improved;
    if (which == 0) {
      bool claimed = false;
      improved = relax_pair(&su->e_del, st.epoch, nd, &claimed);
      // first touch in this query: the length bound starts unknown
      if (claimed) atomicExch(reinterpret_cast<unsigned int *>(&su->hlen), kInfBits);
    } else {
      if (__ldcg(&su->e_del) != st.epoch) continue;  // u has no feasible completion
      const unsigned old = atomicMin(reinterpret_cast<unsigned int *>(&su->hlen), __float_as_uint(nd));
      improved = __float_as_uint(nd) < old;
    }
    if (!improved) continue;
    if (nd < hi && use_ring) {
      const uint32_t pos = warp_agg_inc(&st.near_tail);
      c.nearq[pos & P.near_mask] = (uint32_t)u;
    } else {
      const uint32_t pos = warp_agg_inc(&st.far_n);
      if (pos >= (uint64_t)P.far_cap) {
        fail_query(st, VINE_ERR_CAPACITY, kSiteBand);
      } else {
        c.far[pos] = Label{u, nd, 0.0f, -1};
        atomicMin(&st.far_min_bits, __float_as_uint(nd));
      }
    }
  }
  __syncthreads();
}

// Current reverse distance of v in pass `which` (+inf when unset).
__device__ __forceinline__ float reverse_dist(const Ctx &c, int which, int v) {
  const VView s = view_vs(&c.vs[v], c.st.epoch, c.st.qbase, c.st.bcur, true);
  if (which == 0) return __ldcg(&c.vs[v].e_del) == c.st.epoch ? s.hdel : INFINITY;
  return __ldcg(&c.vs[v].e_del) == c.st.epoch ? s.hlen : INFINITY;
}


// Scheduler step at a bucket boundary, run by one warp.  Chooses the width
// of the next bucket; records a trace row (the features seen when the
// finished bucket was opened, its width and its outcome) when tracing is on.
// Policies: fixed width; AR(3) forecast of the bucket size (after
// algorithm/cspp.cuh:254-284); the learned MLP, which scales the AR rule's
// width when its gate output says that pays (clamped: any positive width
// keeps the search exact), with the AR rule as fallback.
__device__ inline void policy_step(const SearchParams &P, QueryState &st) {
  const int lane = threadIdx.x & 31;
  float prev_width = 0.0f;  // the width the finished bucket was opened with (lane 0)
  if (lane == 0) {
    prev_width = st.width;
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
        float *row = P.trace + r * VINE_TRACE_COLS;
        for (int i = 0; i < kFeat; ++i) row[i] = st.x_prev[i];
        row[16] = (float)st.q;
        row[17] = st.width;
        row[18] = (float)st.b_expanded;
        row[19] = (float)st.b_rounds;
      }
    }
    double pred = xs;
    const bool ar_ok = burg_forecast(st.hist, st.hist_n, 3, &pred);
    const float hi = bucket_hi(st);
    BucketStats b;
    b.far_n = (float)st.far_n;
    b.bucket_labels = (float)st.b_labels;
    b.expanded = (float)st.b_expanded;
    b.rounds = (float)st.b_rounds;
    b.total_expanded = (float)st.n_expanded;
    b.buckets = (float)st.n_buckets;
    b.width_rel = log2f(st.width / P.len_scale);
    b.dominated_frac = st.b_candidates ? (float)st.b_dominated / (float)st.b_candidates : 0.0f;
    const bool have_inc = st.inc_key != ~0ull;
    b.inc_found = have_inc ? 1.0f : 0.0f;
    b.inc_gap = have_inc ? log2f(1.0f + fmaxf(0.0f, key_d(st.inc_key) - hi) / P.len_scale) : -1.0f;
    const float far_min = __uint_as_float(st.far_min_bits);
    b.far_gap = st.far_n ? log2f(1.0f + fmaxf(0.0f, far_min - hi) / P.len_scale) : -1.0f;
    b.table_fill = (float)st.b_labels / (float)(1 << P.table_log2);
    b.spilled = st.b_spilled ? 1.0f : 0.0f;
    b.mean_degree = st.b_expanded ? (float)st.b_relaxed / (float)st.b_expanded : 0.0f;
    b.ar_delta = ar_ok ? (float)(pred - xs) : 0.0f;
    b.budget_rel = log2f(1.0f + st.budget / P.len_scale);
    make_features(b, st.x);
    float width = P.width0;
    const int split = P.round_cap;
    if (P.policy == VINE_POLICY_AR || P.policy == VINE_POLICY_MLP) {
      // widen by 1.5x while bucket sizes fell three times in a row ("ending
      // part"), otherwise steer the forecast size towards a quarter of the
      // shared-memory table
      width = st.ar_width;
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
      st.ar_width = width;
      width *= P.ar_scale;
    }
    st.width = width;
    st.split_cap = split;
  }
  __syncwarp();
  if (P.policy == VINE_POLICY_MLP && P.mlp != nullptr) {
    mlp_forward_warp(P.mlp, st.x, st.mh, st.y);
    if (lane == 0) {
      const float y0 = st.y[0], y1 = st.y[1];
      // y1 is a gate: the network's estimate that leaving the AR rule's
      // width pays for this query.  Only then does y0 scale that width for
      // this bucket, within the range of multipliers it was trained on
      // (2^-1.5 .. 2^1.5); otherwise, and for non-finite outputs, the AR
      // rule's width stands.
      if (isfinite(y0) && isfinite(y1) && y1 > 0.5f)
        st.width = st.ar_width * exp2f(fminf(fmaxf(y0, -1.5f), 1.5f));
      // While the network narrows the buckets, their sizes fall and the AR
      // rule's own width widens (its "ending" step); when the gate then
      // closes, that width would open one bucket many times the table's
      // size, whose spills cost more than the network ever saves.  So the
      // width grows by at most 2x a bucket, the AR rule's own largest step.
      st.width = fminf(st.width, 2.0f * prev_width);
    }
    __syncwarp();
  }
  if (lane == 0) {
    for (int i = 0; i < kFeat; ++i) st.x_prev[i] = st.x[i];
  }
  __syncwarp();
}

}  // namespace vine
