// Device-side building blocks of the exact CSP engine (sm_100a).
//
// Search order.  Labels are processed in buckets of a key f = d + h(v), where
// h is a consistent lower bound on the remaining cost (0 without bounds).
// A bucket is the key range [lo, hi); it is expanded in synchronous rounds
// until no label with key in range remains.  Children of a label never have a
// smaller key (consistency), so once a bucket is finished every later label
// at vertex v has a larger d than every label of the bucket at v.  Hence the
// labels of finished buckets at v can be summarised by one number, the
// smallest delay among them ("settled delay", VState::sdel): a candidate is
// dominated by a settled label iff its delay is >= sdel.  Inside the open
// bucket, labels are compared exactly against each other in a per-vertex
// bucket table (shared-memory hash table, spill to HBM).  The reference's
// dominance (include/label.hpp:234-236) and constraint
// (include/constraint.hpp:99-101) are applied unchanged; only the order of
// work differs, so the surviving sink labels are the same.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

namespace vine {

constexpr int32_t kEmpty = -1;
constexpr uint32_t kDeadBit = 0x80000000u;
constexpr long long kDefaultWaitLimit = 1ll << 26;  // bounded waits before giving up

// One accepted label in the arena.  vid's top bit marks a label killed by a
// dominating label of the same bucket.  parent is the arena index of the label
// it was expanded from (-1 for the source).
struct Label {
  int32_t vid;
  float d;
  float dl;
  int32_t parent;
};

// Per (worker, vertex) state, lazily reset by tags: a value is only valid
// for the query / bucket whose tag sits beside it.  32 bytes = one sector.
//   (epoch, sdel)  smallest delay of labels at v in finished buckets whose
//                  table entries were folded (8-byte CAS pair)
//   (e_del, hdel)  reverse delay distance to the sink (bounds mode, CAS pair)
//   (bep, bmin)    bucket id and smallest delay of v's overflow chain; a
//                  chain of an earlier bucket of the same query counts as
//                  settled (8-byte pair, written under v's stripe lock)
//   hlen           reverse length distance (bounds mode; valid with e_del)
//   bhead          arena index of the newest label of v's overflow chain
struct __align__(32) VState {
  uint32_t epoch;
  float sdel;
  uint32_t e_del;
  float hdel;
  uint32_t bep;
  float bmin;
  float hlen;
  uint32_t bhead;
};
// view_vs reads a state with one 256-bit load, which needs exactly this
// size and alignment (arrays of VState then keep every element aligned).
static_assert(sizeof(VState) == 32 && alignof(VState) == 32, "VState must be one aligned 32-byte sector");

// What one query sees of a vertex.
struct VView {
  float sdel;   // effective settled delay (+inf when none)
  bool reach;   // bounds valid: v can lie on a feasible path
  float hdel, hlen;
  uint32_t bep; // chain tag
};

// qbase / bcur: first bucket id of the query and id of the open bucket.
__device__ __forceinline__ VView view_vs(const VState *p, uint32_t epoch, uint32_t qbase,
                                         uint32_t bcur, bool bounds) {
  // the whole 32-byte state in one 256-bit load (L2, like __ldcg); VState
  // is 32-byte aligned
  uint4 a, b;
  asm volatile("ld.global.cg.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z),
                 "=r"(b.w)
               : "l"(p)
               : "memory");
  VView v;
  float sd = a.x == epoch ? __uint_as_float(a.y) : INFINITY;
  if (b.x >= qbase && b.x < bcur) sd = fminf(sd, __uint_as_float(b.y));
  v.sdel = sd;
  v.bep = b.x;
  if (bounds) {
    v.reach = a.z == epoch && __uint_as_float(b.z) < INFINITY;
    v.hdel = __uint_as_float(a.w);
    v.hlen = __uint_as_float(b.z);
  } else {
    v.reach = true;
    v.hdel = 0.0f;
    v.hlen = 0.0f;
  }
  return v;
}

// Lowers the epoch-tagged distance pair at `pair` to nd; true when improved.
// *claimed is set when this call was the first write of the epoch.
__device__ __forceinline__ bool relax_pair(uint32_t *pair, uint32_t epoch, float nd,
                                           bool *claimed) {
  unsigned long long *w = reinterpret_cast<unsigned long long *>(pair);
  unsigned long long old = __ldcg(w);
  for (;;) {
    const uint32_t e = (uint32_t)old;
    const float cur = e == epoch ? __uint_as_float((uint32_t)(old >> 32)) : INFINITY;
    if (!(nd < cur)) return false;
    const unsigned long long nw = ((unsigned long long)__float_as_uint(nd) << 32) | epoch;
    const unsigned long long prev = atomicCAS(w, old, nw);
    if (prev == old) {
      *claimed = (e != epoch);
      return true;
    }
    old = prev;
  }
}

// Bucket-table slots in shared memory, structure of arrays: tv[s] vertex id
// (kEmpty = free), tw[s] = (d, delay), ti[s] arena index (top bit = killed).
// Slots form aligned groups of kGroup; a vertex hashes to one group and its
// labels only ever occupy slots of that group, so a probe is four 16-byte
// loads of vertex ids and a compare in registers.
constexpr int kGroup = 16;

struct DevGraph {
  int32_t n;
  int64_t m;
  const int32_t *row;  // [n+1]
  const int32_t *col;  // [m]
  const float2 *w;     // [m] {len, delay}
  const int32_t *rrow; // reverse CSR (in-arcs)
  const int32_t *rcol;
  const float2 *rw;
};

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ uint64_t pack_key(float d, float dl) {
  // For non-negative floats the IEEE bit patterns are ordered like the
  // values, so this 64-bit key orders labels lexicographically by (d, dl).
  return ((uint64_t)__float_as_uint(d) << 32) | (uint64_t)__float_as_uint(dl);
}
__device__ __forceinline__ float key_d(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ float key_dl(uint64_t k) { return __uint_as_float((uint32_t)k); }

__device__ __forceinline__ bool dominates(float ad, float al, float bd, float bl) {
  return ad <= bd && al <= bl;  // include/label.hpp:234-236
}

__device__ __forceinline__ uint32_t hash_vid(int32_t v, int log2n) {
  return ((uint32_t)v * 2654435769u) >> (32 - log2n);
}

// First slot of v's group in a table of 1 << log2h slots (log2h >= 6).
__device__ __forceinline__ uint32_t group_base(int32_t v, int log2h) {
  return hash_vid(v, log2h - 4) << 4;
}

// Warp-aggregated increment: one atomic per group of converged lanes.
__device__ __forceinline__ uint32_t warp_agg_inc(uint32_t *ctr) {
  namespace cg = cooperative_groups;
  cg::coalesced_group grp = cg::coalesced_threads();
  uint32_t base = 0;
  if (grp.thread_rank() == 0) base = atomicAdd(ctr, (uint32_t)grp.size());
  base = grp.shfl(base, 0);
  return base + (uint32_t)grp.thread_rank();
}

// Thread -> work-item order that deals consecutive items to different warps
// (item j goes to lane j / nwarps of warp j % nwarps): a round with fewer
// items than threads then keeps every warp busy with a few lanes instead of
// packing the items into a few warps whose divergent lanes run one path at a
// time.  A permutation of [0, G) for G a multiple of 32.
__device__ __forceinline__ int spread_index(int tid, int G) {
  return (tid & 31) * (G >> 5) + (tid >> 5);
}

__device__ __forceinline__ void atomic_min_float_nonneg(float *addr, float v) {
  // non-negative floats order like their bit patterns
  atomicMin(reinterpret_cast<unsigned int *>(addr), __float_as_uint(v));
}

// Runs `body` while holding spin lock *l and returns true, or returns false
// after `limit` failed attempts.  The critical section and the release
// sit inside the spin loop: a lane that took the lock finishes and releases
// it before it can reach any reconvergence point where it might wait for a
// lane of its own warp that is still spinning on the same lock.
// gpu_scope: the lock and the data it guards are shared by several CTAs (the
// plain engine's global-memory locks); the fences must then order memory for
// the whole device, not just the block.
template <typename Body>
__device__ __forceinline__ bool with_lock(int *l, Body body, bool gpu_scope, long long limit) {
  for (long long it = 0; it < limit; ++it) {
    if (atomicCAS(l, 0, 1) == 0) {
      if (gpu_scope) __threadfence();
      else __threadfence_block();
      body();
      if (gpu_scope) __threadfence();
      else __threadfence_block();
      atomicExch(l, 0);
      return true;
    }
    if (it > 64) __nanosleep(32);
  }
  return false;
}

// Folds one label of a finished bucket into the settled delay of v.
__device__ __forceinline__ void settle(VState *vs, uint32_t epoch, float dl) {
  unsigned long long *w = reinterpret_cast<unsigned long long *>(vs);
  unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(w);
  for (;;) {
    const uint32_t e = (uint32_t)old;
    const float s = __uint_as_float((uint32_t)(old >> 32));
    if (e == epoch && s <= dl) return;
    const unsigned long long nw = ((unsigned long long)__float_as_uint(dl) << 32) | epoch;
    const unsigned long long prev = atomicCAS(w, old, nw);
    if (prev == old) return;
    old = prev;
  }
}

// ------------------------------------------------------------ block scan

// Exclusive prefix sum of a[0..n) in place (shared memory), returns the total.
// `scratch` holds >= 33 ints of shared memory.  All threads must call.
__device__ inline int block_exclusive_scan(int *a, int n, int *scratch) {
  const int G = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = (G + 31) >> 5;
  const int per = (n + G - 1) / G;
  const int beg = min(n, tid * per), end = min(n, beg + per);
  int local = 0;
  for (int i = beg; i < end; ++i) local += a[i];
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int v = lane < nwarps ? scratch[lane] : 0;
    int vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, vi, o);
      if (lane >= o) vi += y;
    }
    if (lane < nwarps) scratch[lane] = vi - v;  // exclusive warp offsets
    if (lane == nwarps - 1) scratch[32] = vi;   // total
  }
  __syncthreads();
  int run = scratch[warp] + incl - local;
  for (int i = beg; i < end; ++i) {
    int x = a[i];
    a[i] = run;
    run += x;
  }
  const int total = scratch[32];
  __syncthreads();
  return total;
}

// Largest i in [0, n) with off[i] <= e (off non-decreasing, off[0] = 0 <= e).
__device__ __forceinline__ int upper_index(const int *off, int n, int e) {
  int lo = 0, hi = n;  // invariant: off[lo] <= e, answer in [lo, hi)
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (off[mid] <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------ bucket table

// Outcome of inserting a candidate into the bucket store.
enum InsertResult { kInserted = 0, kDominated = 1, kFull = 2, kLockTimeout = 3 };

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kBadIdx = 0xffffffffu;  // allocator out of arena space

// Store of the labels of the open bucket.  First level: a shared-memory hash
// table keyed by vertex (one aligned group of kGroup slots per vertex).  When
// v's group is full, further labels of v go to v's overflow chain in HBM: a
// linked list through the arena (next[] parallel to it) whose head and
// minimum delay live in v's VState, tagged with the bucket id, so chains need
// no clearing and have no capacity limit other than the arena.
struct BucketTable {
  int32_t *tv;         // shared-memory slots: vertex ids
  float2 *tw;          //   (d, delay)
  uint32_t *ti;        //   arena index | dead bit
  int log2h;           // slots = 1 << log2h
  int probe;           // 0: no shared level (every label goes to a chain)
  int *locks;          // striped locks (shared memory)
  int lock_mask;
  VState *vs;          // per-vertex state of this worker
  uint32_t *next;      // arena-parallel chain links
  uint32_t epoch;      // query epoch
  uint32_t qbase;      // first bucket id of the query
  uint32_t bcur;       // id of the open bucket
  unsigned long long *chain_steps;  // statistics: chain labels read
  long long spin_limit;  // lock attempts before an insert gives up
};

// Dominance test of candidate (d, dl) against one stored label; kills the
// stored label when the candidate dominates it.  Returns true when the
// candidate is dominated.  Caller holds v's stripe lock.
__device__ __forceinline__ bool check_one(float ed, float el, float d, float dl, bool *kill) {
  *kill = false;
  if (dominates(ed, el, d, dl)) return true;
  if (dominates(d, dl, ed, el)) *kill = true;
  return false;
}

// Body of table_insert; the caller holds v's stripe lock (whose acquire
// fence orders the plain shared-memory loads below).
template <typename Alloc>
__device__ __forceinline__ InsertResult table_insert_locked(const BucketTable &bt, Label *pool,
                                                            int32_t v, float d, float dl,
                                                            Alloc &idx_alloc, uint32_t *out_idx,
                                                            bool *spilled) {
  uint32_t match = 0, empty = 0, base = 0;
  if (bt.probe) {
    base = group_base(v, bt.log2h);
    const int4 *g4 = reinterpret_cast<const int4 *>(bt.tv + base);
#pragma unroll
    for (int k = 0; k < kGroup / 4; ++k) {
      const int4 q = g4[k];
      const int sh = 4 * k;
      match |= (uint32_t)(q.x == v) << sh | (uint32_t)(q.y == v) << (sh + 1) |
               (uint32_t)(q.z == v) << (sh + 2) | (uint32_t)(q.w == v) << (sh + 3);
      empty |= (uint32_t)(q.x == kEmpty) << sh | (uint32_t)(q.y == kEmpty) << (sh + 1) |
               (uint32_t)(q.z == kEmpty) << (sh + 2) | (uint32_t)(q.w == kEmpty) << (sh + 3);
    }
    for (uint32_t m = match; m; m &= m - 1) {
      const uint32_t sl = base + (uint32_t)(__ffs(m) - 1);
      const uint32_t eidx = bt.ti[sl];
      if (eidx & kDeadBit) continue;
      const float2 w = bt.tw[sl];
      bool kill;
      if (check_one(w.x, w.y, d, dl, &kill)) return kDominated;
      if (kill) {
        bt.ti[sl] = eidx | kDeadBit;
        atomicOr(reinterpret_cast<unsigned int *>(&pool[eidx].vid), kDeadBit);
      }
    }
  }
  // Labels of v beyond its group live in v's overflow chain.  Slots are never
  // freed during a bucket, so a group that still had a free slot means v has
  // no chain in this bucket.
  const bool had_free = empty != 0;
  volatile VState *vs = &bt.vs[v];
  uint32_t bep = 0;
  if (!had_free) {
    bep = vs->bep;
    if (bep == bt.bcur) {
      // Dead labels are unlinked as the walk meets them (only the holder of
      // v's stripe lock walks or changes v's chain), so a vertex that takes
      // many labels in one wide bucket keeps a chain of its live labels, not
      // of every label it ever held.  bmin keeps the dead labels' delays:
      // each was dominated by a label of the same bucket with a delay no
      // larger, so the settled delay of v is unchanged.
      uint32_t steps = 0, prev = kNone;
      for (uint32_t k = vs->bhead; k != kNone;) {
        ++steps;
        const uint32_t nk = __ldcg(&bt.next[k]);
        const int4 raw = __ldcg(reinterpret_cast<const int4 *>(&pool[k]));
        bool dead = (raw.x & (int)kDeadBit) != 0;
        if (!dead) {
          bool kill;
          if (check_one(__int_as_float(raw.y), __int_as_float(raw.z), d, dl, &kill)) {
            if (bt.chain_steps) atomicAdd(bt.chain_steps, (unsigned long long)steps);
            return kDominated;
          }
          if (kill) {
            atomicOr(reinterpret_cast<unsigned int *>(&pool[k].vid), kDeadBit);
            dead = true;
          }
        }
        if (dead) {
          if (prev == kNone) vs->bhead = nk;
          else __stcg(&bt.next[prev], nk);
        } else {
          prev = k;
        }
        k = nk;
      }
      if (bt.chain_steps) atomicAdd(bt.chain_steps, (unsigned long long)steps);
    }
  }
  // not dominated: claim a free slot of the group (other vertices may race)
  for (uint32_t m = empty; m; m &= m - 1) {
    const uint32_t sl = base + (uint32_t)(__ffs(m) - 1);
    if (atomicCAS(&bt.tv[sl], kEmpty, v) == kEmpty) {
      const uint32_t idx = idx_alloc();
      if (idx == kBadIdx) {
        bt.ti[sl] = kDeadBit;  // never expanded, never settled
        return kFull;
      }
      bt.tw[sl] = make_float2(d, dl);
      bt.ti[sl] = idx;
      *out_idx = idx;
      *spilled = false;
      return kInserted;
    }
  }
  // group full: push onto v's overflow chain in HBM
  if (had_free) bep = vs->bep;  // the group filled up while we probed it
  const uint32_t idx = idx_alloc();
  if (idx == kBadIdx) return kFull;
  float bmin = dl;
  uint32_t head = kNone;
  if (bep == bt.bcur) {
    head = vs->bhead;
    bmin = fminf(bmin, vs->bmin);
  } else if (bep >= bt.qbase && bep < bt.bcur) {
    settle(const_cast<VState *>(vs), bt.epoch, vs->bmin);
  }
  bt.next[idx] = head;
  vs->bhead = idx;
  __threadfence_block();
  // publish (bep, bmin) together for lock-free readers
  *reinterpret_cast<volatile unsigned long long *>(&vs->bep) =
      ((unsigned long long)__float_as_uint(bmin) << 32) | bt.bcur;
  *out_idx = idx;
  *spilled = true;
  return kInserted;
}

// Checks candidate (v, d, dl) against the labels of the open bucket at v,
// kills the ones it dominates (marking their arena labels dead) and, when it
// is not dominated, stores it with arena index `idx_alloc()` (which also
// writes the arena label, so a kill can never be overwritten).  Exact: all
// operations on one vertex are serialised by that vertex's stripe lock, and
// a candidate is only dropped when a stored label dominates it.  gpu_scope:
// the stripe locks live in global memory and are shared by all CTAs.
template <typename Alloc>
__device__ __forceinline__ InsertResult table_insert(const BucketTable &bt, Label *pool, int32_t v, float d,
                                     float dl, Alloc idx_alloc, uint32_t *out_idx,
                                     bool *spilled, bool gpu_scope) {
  int *lk = &bt.locks[(uint32_t)v & (uint32_t)bt.lock_mask];
  InsertResult r = kLockTimeout;
  with_lock(lk, [&]() { r = table_insert_locked(bt, pool, v, d, dl, idx_alloc, out_idx, spilled); },
            gpu_scope, bt.spin_limit);
  return r;
}

// ------------------------------------------------ scheduler (AR and MLP)

constexpr int kFeat = 16;
constexpr int kHid = 64;
constexpr int kOut = 2;
constexpr int kMlpParams = kHid * kFeat + kHid + kHid * kHid + kHid + kOut * kHid + kOut;

// Burg's maximum-entropy AR(p) fit (J. P. Burg, 1967; the recursion as given
// in standard spectral-estimation texts) of the mean-removed series x[0..n),
// then a one-step forecast x_hat[n].  Plays the role of the reference's
// AR::AutoRegression / ARMaxEntropy (include/AR.cpp:6-147) as used by
// RUN_CSPP (algorithm/cspp.cuh:263-284).  Returns false when the fit is
// degenerate (constant series or too few points).
constexpr int kBurgMaxN = 32;
__host__ __device__ inline bool burg_forecast(const double *x, int n, int p, double *out) {
  if (n <= p || p < 1 || p > 8 || n > kBurgMaxN) return false;
  double mean = 0.0;
  for (int i = 0; i < n; ++i) mean += x[i];
  mean /= n;
  double f[kBurgMaxN], b[kBurgMaxN], a[9], an[9];
  for (int i = 0; i < n; ++i) f[i] = b[i] = x[i] - mean;
  for (int i = 0; i <= p; ++i) a[i] = 0.0;
  a[0] = 1.0;
  for (int m = 1; m <= p; ++m) {
    double num = 0.0, den = 0.0;
    for (int k = m; k < n; ++k) {
      num += f[k] * b[k - 1];
      den += f[k] * f[k] + b[k - 1] * b[k - 1];
    }
    if (!(den > 0.0)) return false;
    const double km = -2.0 * num / den;
    for (int i = 0; i <= m; ++i) an[i] = a[i] + km * (m - i >= 0 ? a[m - i] : 0.0);
    for (int i = 0; i <= m; ++i) a[i] = an[i];
    // update prediction errors, from the end so b[k-1] is still the old value
    for (int k = n - 1; k >= m; --k) {
      const double fk = f[k], bk = b[k - 1];
      f[k] = fk + km * bk;
      b[k] = bk + km * fk;
    }
  }
  double pred = 0.0;
  for (int i = 1; i <= p; ++i) pred -= a[i] * (x[n - i] - mean);
  *out = mean + pred;
  return true;
}

// Scheduler features of one bucket boundary (the 16 MLP inputs).
struct BucketStats {
  float far_n, bucket_labels, expanded, rounds, total_expanded, buckets, width_rel,
      dominated_frac, inc_found, inc_gap, far_gap, table_fill, spilled, mean_degree, ar_delta,
      budget_rel;
};

__host__ __device__ inline void make_features(const BucketStats &s, float *x) {
  x[0] = log2f(1.0f + s.far_n);
  x[1] = log2f(1.0f + s.bucket_labels);
  x[2] = log2f(1.0f + s.expanded);
  x[3] = log2f(1.0f + s.rounds);
  x[4] = log2f(1.0f + s.total_expanded);
  x[5] = log2f(1.0f + s.buckets);
  x[6] = s.width_rel;
  x[7] = s.dominated_frac;
  x[8] = s.inc_found;
  x[9] = s.inc_gap;
  x[10] = s.far_gap;
  x[11] = s.table_fill;
  x[12] = s.spilled;
  x[13] = s.mean_degree;
  x[14] = s.ar_delta;
  x[15] = s.budget_rel;
}

// Forward pass of the 16-64-64-2 ReLU MLP by one warp (lanes split the 64
// hidden units two each).  params layout: W1[64][16] b1[64] W2[64][64] b2[64]
// W3[2][64] b3[2].  `h` is 128 floats of scratch visible to the warp.
__device__ inline void mlp_forward_warp(const float *__restrict__ params, const float *x,
                                        float *h, float *y) {
  const int lane = threadIdx.x & 31;
  const float *W1 = params, *b1 = W1 + kHid * kFeat, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid,
              *W3 = b2 + kHid, *b3 = W3 + kOut * kHid;
  for (int j = lane; j < kHid; j += 32) {
    float acc = b1[j];
    for (int i = 0; i < kFeat; ++i) acc += W1[j * kFeat + i] * x[i];
    h[j] = fmaxf(acc, 0.0f);
  }
  __syncwarp();
  float h2[2];
  for (int r = 0; r < 2; ++r) {
    const int j = lane + 32 * r;
    float acc = b2[j];
    for (int i = 0; i < kHid; ++i) acc += W2[j * kHid + i] * h[i];
    h2[r] = fmaxf(acc, 0.0f);
  }
  __syncwarp();
  h[kHid + lane] = h2[0];
  h[kHid + lane + 32] = h2[1];
  __syncwarp();
  if (lane < kOut) {
    float acc = b3[lane];
    for (int i = 0; i < kHid; ++i) acc += W3[lane * kHid + i] * h[kHid + i];
    y[lane] = acc;
  }
  __syncwarp();
}

}  // namespace vine
