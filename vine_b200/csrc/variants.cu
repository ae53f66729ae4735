// Label variants on the GPU: the reference's other label types through one
// templated engine (include/label.hpp:46-465, include/constraint.hpp:21-187).
//
//   VINE_LABEL_CSP      (d, delay)                     CSP=1 and CSP=4 (2-OSP)
//   VINE_LABEL_HOP      (d, delay, hop)                CSP=2, hop-constrained
//   VINE_LABEL_MAXCOST  (d, delay, hop, maxcost)       CSP=3, max arc length
//   VINE_LABEL_QOS      (d, bandwidth = min arc delay) network QoS
//
// Each kind supplies the reference's expand, dominate and constraint (Ops<K>
// below); the search is generic.  Unlike the CSP engine (batch.cu), whose
// settled-delay summary is only valid for two criteria, a label here is
// compared against every live label stored at its vertex: per-vertex chains
// in HBM, serialised by striped locks in shared memory, dominated labels
// marked dead and unlinked.  Labels are expanded in buckets of cost d
// (label correcting inside a bucket, block-synchronous rounds with a
// load-balanced arc list), one query per CTA worker of a persistent kernel.
// Every generated label is a real path and dominance never discards a label
// that an equal-or-better label does not cover, so the best feasible sink
// label -- lexicographically smallest (d, delay, hop, maxcost), for QoS the
// smallest d and then the largest bandwidth -- is exact.  Costs only grow
// along a path (weights >= 0), so a label whose d exceeds the incumbent's is
// dropped.

#include "engine_host.h"
#include "search.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace vine {
namespace {

struct __align__(16) VLabel {
  int32_t vid;  // top bit: dead (dominated by a label stored later)
  float d;
  float r0, r1, r2;
  int32_t parent;  // arena index, -1 for the source
  uint32_t next;   // next label of the same vertex's chain (kNone = end)
  uint32_t pad;
};

constexpr float kQosStart = 21474836.0f;  // the reference's initial bandwidth (include/label.hpp:396-399)

template <int K>
struct Ops;

template <>
struct Ops<VINE_LABEL_CSP> {
  static constexpr int kKey = 2;
  __device__ static void source(VLabel &l) { l.r0 = l.r1 = l.r2 = 0.0f; }
  __device__ static void expand(const VLabel &a, float len, float dly, VLabel &c) {
    c.d = a.d + len;
    c.r0 = a.r0 + dly;  // include/label.hpp:214-222
    c.r1 = c.r2 = 0.0f;
  }
  __device__ static bool dominates(const VLabel &a, const VLabel &b) {
    return a.d <= b.d && a.r0 <= b.r0;  // include/label.hpp:234-236
  }
  __device__ static bool feasible(const VLabel &l, float L, float, float) {
    return !(l.r0 > L);  // include/constraint.hpp:99-101
  }
  __device__ static void key(const VLabel &l, float *k) {
    k[0] = l.d;
    k[1] = l.r0;
  }
};

template <>
struct Ops<VINE_LABEL_HOP> {
  static constexpr int kKey = 3;
  __device__ static void source(VLabel &l) { l.r0 = l.r1 = l.r2 = 0.0f; }
  __device__ static void expand(const VLabel &a, float len, float dly, VLabel &c) {
    c.d = a.d + len;  // include/label.hpp:88-97
    c.r0 = a.r0 + dly;
    c.r1 = a.r1 + 1.0f;
    c.r2 = 0.0f;
  }
  __device__ static bool dominates(const VLabel &a, const VLabel &b) {
    return a.d <= b.d && a.r0 <= b.r0 && a.r1 <= b.r1;  // include/label.hpp:99-104
  }
  __device__ static bool feasible(const VLabel &l, float L, float H, float) {
    return !(l.r0 > L || l.r1 > H);  // include/constraint.hpp:42-48
  }
  __device__ static void key(const VLabel &l, float *k) {
    k[0] = l.d;
    k[1] = l.r0;
    k[2] = l.r1;
  }
};

template <>
struct Ops<VINE_LABEL_MAXCOST> {
  static constexpr int kKey = 4;
  __device__ static void source(VLabel &l) { l.r0 = l.r1 = l.r2 = 0.0f; }
  __device__ static void expand(const VLabel &a, float len, float dly, VLabel &c) {
    c.d = a.d + len;  // include/label.hpp:151-160
    c.r0 = a.r0 + dly;
    c.r1 = a.r1 + 1.0f;
    c.r2 = fmaxf(a.r2, len);
  }
  __device__ static bool dominates(const VLabel &a, const VLabel &b) {
    return a.d <= b.d && a.r0 <= b.r0 && a.r1 <= b.r1 && a.r2 <= b.r2;  // :161-166
  }
  __device__ static bool feasible(const VLabel &l, float L, float H, float M) {
    return !(l.r0 > L || l.r1 > H || l.r2 > M);  // include/constraint.hpp:73-79
  }
  __device__ static void key(const VLabel &l, float *k) {
    k[0] = l.d;
    k[1] = l.r0;
    k[2] = l.r1;
    k[3] = l.r2;
  }
};

template <>
struct Ops<VINE_LABEL_QOS> {
  static constexpr int kKey = 2;
  __device__ static void source(VLabel &l) {
    l.r0 = kQosStart;
    l.r1 = l.r2 = 0.0f;
  }
  __device__ static void expand(const VLabel &a, float len, float dly, VLabel &c) {
    c.d = a.d + len;  // include/label.hpp:424-431
    c.r0 = fminf(a.r0, dly);
    c.r1 = c.r2 = 0.0f;
  }
  __device__ static bool dominates(const VLabel &a, const VLabel &b) {
    return a.d <= b.d && a.r0 >= b.r0;  // include/label.hpp:445-450
  }
  __device__ static bool feasible(const VLabel &l, float L, float, float) {
    return !(l.r0 < L);  // include/constraint.hpp:180-182
  }
  __device__ static void key(const VLabel &l, float *k) {
    k[0] = l.d;
    k[1] = -l.r0;  // larger bandwidth first
  }
};

template <int N>
__device__ __forceinline__ bool key_less(const float *a, const float *b) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    if (a[i] < b[i]) return true;
    if (a[i] > b[i]) return false;
  }
  return false;
}

struct VParams {
  DevGraph g;
  int32_t nq;
  const int32_t *src, *dst;
  const float *lim_delay, *lim_hop, *lim_max;
  float *cost, *delay, *extra;  // extra: [nq * 2] (hop, maxcost)
  int32_t *found, *status;
  int64_t *stats;
  uint64_t *head;    // per worker x vertex: (epoch << 32) | newest chain label
  uint32_t *near;    // per worker ring of arena indices
  uint32_t near_mask;
  uint32_t *far;     // per worker far pile
  int64_t far_cap;
  VLabel *pool;      // per worker slice of pool_per_worker labels
  int64_t pool_per_worker;
  int32_t *path_arena;
  int64_t path_cap;
  unsigned long long *path_top;
  int64_t *path_start;
  int32_t *path_len;
  unsigned long long *queue;
  uint32_t epoch_base;
  float width;
  int lock_log2;
  long long wait_limit;
  unsigned long long time_limit_ns;
};

struct VState {
  unsigned long long g0;
  long long t0;
  int q, src, dst;
  float L, H, M;
  uint32_t epoch;
  uint32_t pool_fill;
  uint32_t near_head, near_tail;
  uint32_t far_n, far_wpos, far_min_bits;
  float lo, hi;
  float inc_key[4];
  uint32_t inc_idx;
  int inc_lock;
  int abort, abort_site, done;
  unsigned long long n_expanded, n_relaxed, n_inserted, n_dominated, n_buckets, n_rounds;
};

constexpr int kVBatch = 2;  // labels per thread per round

__device__ __forceinline__ void vfail(VState &st, int status, int site) {
  if (atomicCAS(&st.abort, 0, status) == 0) st.abort_site = site;
}

__device__ __forceinline__ uint32_t valloc(VState &st, const VParams &P) {
  const uint32_t i = atomicAdd(&st.pool_fill, 1u);
  if ((int64_t)i >= P.pool_per_worker) {
    vfail(st, VINE_ERR_CAPACITY, kSiteArenaAlloc);
    return kBadIdx;
  }
  return i;
}

// Offers a feasible label at the sink to the incumbent (stored in the arena
// so that its path can be rebuilt).
template <int K>
__device__ void vsink(const VParams &P, VState &st, VLabel *pool, const VLabel &c, int *ilock) {
  float k[4] = {0, 0, 0, 0};
  Ops<K>::key(c, k);
  float cur[4];
  // unlocked pre-check against the published incumbent
  for (int i = 0; i < 4; ++i) cur[i] = *reinterpret_cast<volatile float *>(&st.inc_key[i]);
  if (st.inc_idx != kNone && !key_less<Ops<K>::kKey>(k, cur)) return;
  const uint32_t idx = valloc(st, P);
  if (idx == kBadIdx) return;
  pool[idx] = c;
  pool[idx].next = kNone;
  const bool ok = with_lock(ilock, [&]() {
    volatile float *ik = st.inc_key;
    float now[4] = {ik[0], ik[1], ik[2], ik[3]};
    if (*reinterpret_cast<volatile uint32_t *>(&st.inc_idx) == kNone || key_less<Ops<K>::kKey>(k, now)) {
      for (int i = 0; i < 4; ++i) ik[i] = k[i];
      *reinterpret_cast<volatile uint32_t *>(&st.inc_idx) = idx;
    }
  }, false, P.wait_limit);
  if (!ok) vfail(st, VINE_ERR_TIMEOUT, kSiteLock);
}

// Dominance against v's chain and insertion (caller queues the label).
// Returns the arena index, or kBadIdx when dominated / failed.
template <int K>
__device__ uint32_t vinsert(const VParams &P, VState &st, VLabel *pool, uint64_t *head,
                            int *locks, int lock_mask, const VLabel &c, unsigned long long *dom) {
  const int v = c.vid;
  uint32_t res = kBadIdx;
  const bool ok = with_lock(&locks[v & lock_mask], [&]() {
    volatile uint64_t *hp = reinterpret_cast<volatile uint64_t *>(&head[v]);
    const uint64_t h = *hp;
    uint32_t first = (uint32_t)(h >> 32) == st.epoch ? (uint32_t)h : kNone;
    uint32_t prev = kNone;
    for (uint32_t k = first; k != kNone;) {
      VLabel &s = pool[k];
      const uint32_t nxt = *reinterpret_cast<volatile uint32_t *>(&s.next);
      const int32_t sv = *reinterpret_cast<volatile int32_t *>(&s.vid);
      bool unlink = (sv & (int)kDeadBit) != 0;
      if (!unlink) {
        const VLabel sl{sv, *reinterpret_cast<volatile float *>(&s.d),
                        *reinterpret_cast<volatile float *>(&s.r0),
                        *reinterpret_cast<volatile float *>(&s.r1),
                        *reinterpret_cast<volatile float *>(&s.r2), 0, 0, 0};
        if (Ops<K>::dominates(sl, c)) {
          (*dom)++;
          return;  // the candidate is dominated
        }
        if (Ops<K>::dominates(c, sl)) {
          atomicOr(reinterpret_cast<unsigned int *>(&s.vid), kDeadBit);
          unlink = true;
        }
      }
      if (unlink) {  // drop k from the chain (only lock holders touch it)
        if (prev == kNone) first = nxt;
        else *reinterpret_cast<volatile uint32_t *>(&pool[prev].next) = nxt;
      } else {
        prev = k;
      }
      k = nxt;
    }
    const uint32_t idx = valloc(st, P);
    if (idx == kBadIdx) return;
    VLabel n = c;
    n.next = first;
    pool[idx] = n;
    __threadfence_block();
    *hp = ((uint64_t)st.epoch << 32) | idx;
    res = idx;
  }, false, P.wait_limit);
  if (!ok) vfail(st, VINE_ERR_TIMEOUT, kSiteLock);
  return res;
}

template <int K>
__global__ void __launch_bounds__(512, 1) variant_kernel(VParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int G = blockDim.x, tid = threadIdx.x, slot = blockIdx.x;
  const int NL = 1 << P.lock_log2;
  const int RC = G * kVBatch;
  int *locks = reinterpret_cast<int *>(smem);
  uint32_t *r_idx = reinterpret_cast<uint32_t *>(locks + NL);
  int *r_beg = reinterpret_cast<int *>(r_idx + RC);
  int *r_off = r_beg + RC;
  int *scan = r_off + RC;
  VState &st = *reinterpret_cast<VState *>(
      (reinterpret_cast<uintptr_t>(scan + kScanScratch) + 15) & ~(uintptr_t)15);

  uint64_t *head = P.head + (size_t)slot * P.g.n;
  uint32_t *near = P.near + (size_t)slot * (P.near_mask + 1u);
  uint32_t *far = P.far + (size_t)slot * P.far_cap;
  VLabel *pool = P.pool + (size_t)slot * P.pool_per_worker;
  for (int i = tid; i < NL; i += G) locks[i] = 0;
  __syncthreads();

  for (;;) {
    if (tid == 0) {
      const unsigned long long k = atomicAdd(P.queue, 1ull);
      st.q = k < (unsigned long long)P.nq ? (int)k : -1;
    }
    __syncthreads();
    const int q = st.q;
    if (q < 0) break;
    if (tid == 0) {
      st.t0 = clock64();
      st.g0 = global_ns();
      st.src = P.src[q];
      st.dst = P.dst[q];
      st.L = P.lim_delay[q];
      st.H = P.lim_hop ? P.lim_hop[q] : 100.0f;
      st.M = P.lim_max ? P.lim_max[q] : 10000.0f;
      st.epoch = P.epoch_base + (uint32_t)q;
      st.pool_fill = 0;
      st.near_head = st.near_tail = 0;
      st.far_n = st.far_wpos = 0;
      st.far_min_bits = kInfBits;
      st.inc_idx = kNone;
      st.inc_lock = 0;
      for (int i = 0; i < 4; ++i) st.inc_key[i] = INFINITY;
      st.abort = st.abort_site = st.done = 0;
      st.n_expanded = st.n_relaxed = st.n_inserted = st.n_dominated = 0;
      st.n_buckets = st.n_rounds = 0;
      st.lo = 0.0f;
      st.hi = P.width;
      const int s = st.src, t = st.dst;
      if (s < 0 || s >= P.g.n || t < 0 || t >= P.g.n || isnan(st.L)) {
        vfail(st, VINE_ERR_INVALID, kSiteInvalid);
      } else {
        VLabel src{s, 0.0f, 0, 0, 0, -1, kNone, 0};
        Ops<K>::source(src);
        if (!Ops<K>::feasible(src, st.L, st.H, st.M)) {
          st.done = 1;  // even the source label violates the constraint
        } else {
          const uint32_t idx = valloc(st, P);
          pool[idx] = src;
          head[s] = ((uint64_t)st.epoch << 32) | idx;
          if (s == t) {
            Ops<K>::key(src, st.inc_key);
            st.inc_idx = idx;
            st.done = 1;
          } else {
            near[0] = idx;
            st.near_tail = 1;
          }
        }
      }
    }
    __syncthreads();
    unsigned long long dom = 0;
    while (!st.done && !st.abort) {
      const uint32_t avail = st.near_tail - st.near_head;
      if (avail == 0) {
        // ---- next bucket: its key range starts at the far pile's minimum
        if (st.far_n == 0) break;
        if (tid == 0) {
          st.n_buckets++;
          if (P.time_limit_ns && global_ns() - st.g0 > P.time_limit_ns)
            vfail(st, VINE_ERR_TIMEOUT, kSiteTime);
          st.lo = fmaxf(st.hi, __uint_as_float(st.far_min_bits));
          st.hi = st.lo + P.width;
          if (!(st.hi > st.lo)) st.hi = nextafterf(st.lo, INFINITY);
          st.far_min_bits = kInfBits;
          st.far_wpos = 0;
        }
        __syncthreads();
        const uint32_t fn = st.far_n;
        const float hi = st.hi;
        const float inc_d = st.inc_key[0];
        for (uint32_t base = 0; base < fn; base += (uint32_t)G) {
          const uint32_t i = base + tid;
          uint32_t idx = kNone;
          VLabel l;
          if (i < fn) {
            idx = far[i];
            l = pool[idx];
          }
          __syncthreads();  // the tile is read before it is overwritten
          if (idx != kNone && !(l.vid & (int)kDeadBit) && !(l.d > inc_d)) {
            if (l.d < hi) {
              const uint32_t pos = atomicAdd(&st.near_tail, 1u);
              if (pos - st.near_head > P.near_mask) vfail(st, VINE_ERR_CAPACITY, kSiteNear);
              else near[pos & P.near_mask] = idx;
            } else {
              const uint32_t w = atomicAdd(&st.far_wpos, 1u);
              far[w] = idx;
              atomicMin(&st.far_min_bits, __float_as_uint(l.d));
            }
          }
          __syncthreads();
        }
        if (tid == 0) st.far_n = st.far_wpos;
        __syncthreads();
        continue;
      }
      // ---- one round over up to RC labels of the open bucket
      const int n = (int)min((uint32_t)RC, avail);
      const uint32_t first = st.near_head;
      __syncthreads();
      if (tid == 0) {
        st.near_head += (uint32_t)n;
        st.n_rounds++;
      }
      const float inc_d0 = *reinterpret_cast<volatile float *>(&st.inc_key[0]);
      for (int i = tid; i < n; i += G) {
        const uint32_t idx = near[(first + (uint32_t)i) & P.near_mask];
        const VLabel l = pool[idx];
        int deg = 0, beg = 0;
        if (!(l.vid & (int)kDeadBit) && !(l.d > inc_d0)) {
          beg = __ldg(&P.g.row[l.vid]);
          deg = __ldg(&P.g.row[l.vid + 1]) - beg;
          if (deg > 0) atomicAdd(&st.n_expanded, 1ull);
        }
        r_idx[i] = idx;
        r_beg[i] = beg;
        r_off[i] = deg;
      }
      __syncthreads();
      const int total = block_exclusive_scan(r_off, n, scan);
      if (tid == 0) st.n_relaxed += (unsigned long long)total;
      const float hi = st.hi;
      for (int e = tid; e < total; e += G) {
        const int k = upper_index(r_off, n, e);
        const int j = r_beg[k] + (e - r_off[k]);
        const uint32_t pidx = r_idx[k];
        const VLabel a = pool[pidx];
        VLabel c;
        c.vid = __ldg(&P.g.col[j]);
        const float2 w = __ldg(&P.g.w[j]);
        Ops<K>::expand(a, w.x, w.y, c);
        c.parent = (int32_t)pidx;
        c.next = kNone;
        c.pad = 0;
        if (!Ops<K>::feasible(c, st.L, st.H, st.M)) continue;
        if (c.d > *reinterpret_cast<volatile float *>(&st.inc_key[0])) continue;
        if (c.vid == st.dst) {
          vsink<K>(P, st, pool, c, &st.inc_lock);
          continue;
        }
        const uint32_t idx = vinsert<K>(P, st, pool, head, locks, NL - 1, c, &dom);
        if (idx == kBadIdx) continue;
        atomicAdd(&st.n_inserted, 1ull);
        if (c.d < hi) {
          const uint32_t pos = atomicAdd(&st.near_tail, 1u);
          if (pos - st.near_head > P.near_mask) vfail(st, VINE_ERR_CAPACITY, kSiteNear);
          else near[pos & P.near_mask] = idx;
        } else {
          const uint32_t pos = atomicAdd(&st.far_n, 1u);
          if ((int64_t)pos >= P.far_cap) vfail(st, VINE_ERR_CAPACITY, kSiteBand);
          else {
            far[pos] = idx;
            atomicMin(&st.far_min_bits, __float_as_uint(c.d));
          }
        }
      }
      __syncthreads();
    }
    if (dom) atomicAdd(&st.n_dominated, dom);
    __syncthreads();
    if (tid == 0) {
      const bool ok = st.abort == 0;
      const bool found = ok && st.inc_idx != kNone;
      P.status[q] = ok ? VINE_OK : st.abort;
      P.found[q] = found ? 1 : 0;
      if (found) {
        const VLabel b = pool[st.inc_idx];
        P.cost[q] = b.d;
        P.delay[q] = b.r0;
        if (P.extra) {
          P.extra[2 * (size_t)q] = b.r1;
          P.extra[2 * (size_t)q + 1] = b.r2;
        }
      } else {
        P.cost[q] = INFINITY;
        P.delay[q] = INFINITY;
        if (P.extra) P.extra[2 * (size_t)q] = P.extra[2 * (size_t)q + 1] = 0.0f;
      }
      // answer path (source .. sink) into the path arena
      P.path_len[q] = 0;
      P.path_start[q] = 0;
      if (found) {
        int32_t len = 0;
        for (int32_t k = (int32_t)st.inc_idx; k >= 0; k = pool[k].parent) ++len;
        const unsigned long long b0 = atomicAdd(P.path_top, (unsigned long long)len);
        if (b0 + len > (unsigned long long)P.path_cap) {
          P.status[q] = VINE_ERR_CAPACITY;
        } else {
          int64_t pos = (int64_t)b0 + len - 1;
          for (int32_t k = (int32_t)st.inc_idx; k >= 0; k = pool[k].parent)
            P.path_arena[pos--] = pool[k].vid & 0x7fffffff;
          P.path_start[q] = (int64_t)b0;
          P.path_len[q] = len;
        }
      }
      if (P.stats) {
        int64_t *s = P.stats + (size_t)q * VINE_STAT_COUNT;
        for (int i = 0; i < VINE_STAT_COUNT; ++i) s[i] = 0;
        s[VINE_STAT_EXPANDED] = (int64_t)st.n_expanded;
        s[VINE_STAT_RELAXED] = (int64_t)st.n_relaxed;
        s[VINE_STAT_INSERTED] = (int64_t)st.n_inserted;
        s[VINE_STAT_DOMINATED] = (int64_t)st.n_dominated;
        s[VINE_STAT_BUCKETS] = (int64_t)st.n_buckets;
        s[VINE_STAT_ROUNDS] = (int64_t)st.n_rounds;
        s[VINE_STAT_CYCLES] = clock64() - st.t0;
        s[VINE_STAT_ABORT_SITE] = st.abort_site;
        s[VINE_STAT_START_NS] = (int64_t)st.g0;
        s[VINE_STAT_TIME_NS] = (int64_t)(global_ns() - st.g0);
      }
    }
    __syncthreads();
  }
}

size_t variant_smem(int block_threads, int lock_log2) {
  size_t b = ((size_t)4 << lock_log2) + (size_t)block_threads * kVBatch * 12 +
             kScanScratch * sizeof(int);
  b = (b + 15) & ~(size_t)15;
  return b + sizeof(VState) + 16;
}

template <int K>
int launch_variant(const VParams &P, int slots, int threads, size_t smem, cudaStream_t s) {
  VINE_CUDA_TRY(cudaFuncSetAttribute(variant_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  variant_kernel<K><<<slots, threads, smem, s>>>(P);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

// Device buffers of one variant call (allocated per call: variants are not
// the hot path).
struct VBuffers {
  std::vector<void *> ptrs;
  template <typename T>
  int alloc(T **p, size_t count) {
    *p = nullptr;
    if (cudaMalloc(p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess)
      return fail(VINE_ERR_CUDA, "variant engine: allocation failed");
    ptrs.push_back(*p);
    return VINE_OK;
  }
  ~VBuffers() {
    for (void *p : ptrs) cudaFree(p);
  }
};

}  // namespace
}  // namespace vine

using namespace vine;

extern "C" {

int vine_solve_labels(vine_graph *g, int32_t kind, int32_t nq, const int32_t *src,
                      const int32_t *dst, const float *delay_limit, const float *hop_limit,
                      const float *maxcost_limit, const vine_config *cfg, vine_results *out,
                      float *extra) {
  if (!g || !out || nq < 0) return fail(VINE_ERR_INVALID, "bad arguments");
  if (kind != VINE_LABEL_CSP && kind != VINE_LABEL_HOP && kind != VINE_LABEL_MAXCOST &&
      kind != VINE_LABEL_QOS)
    return fail(VINE_ERR_INVALID, "unknown label kind");
  if (nq == 0) {
    if (out->path_offsets) out->path_offsets[0] = 0;
    return VINE_OK;
  }
  if (!src || !dst || !delay_limit || !out->cost || !out->delay || !out->found)
    return fail(VINE_ERR_INVALID, "missing input/output buffers");
  std::lock_guard<std::mutex> lk(g->mu);
  VINE_CUDA_TRY(cudaSetDevice(g->device));
  vine_config c;
  if (cfg) c = *cfg;
  else vine_config_default(&c);
  const int threads = c.block_threads > 0 ? c.block_threads : 256;
  if (threads < 64 || threads > 512 || threads % 32)
    return fail(VINE_ERR_INVALID, "block_threads must be a multiple of 32 in [64, 512]");
  const int lock_log2 = 11;
  const size_t smem = variant_smem(threads, lock_log2);
  int slots = g->sm_count;
  if (c.max_workers > 0) slots = std::min(slots, (int)c.max_workers);
  slots = std::min<int>(slots, nq);
  const int64_t far_cap = c.far_capacity > 0 ? c.far_capacity : (int64_t(1) << 20);
  const uint32_t near_cap = 1u << 20;
  int64_t pool_total = c.pool_labels;
  if (pool_total <= 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t fixed = (size_t)slots * ((size_t)g->n * 8 + (size_t)near_cap * 4 + (size_t)far_cap * 4);
    pool_total = free_b > fixed ? (int64_t)((free_b - fixed) / 3 / sizeof(VLabel)) : 0;
  }
  const int64_t per_worker = std::min<int64_t>(pool_total / std::max(slots, 1), int64_t(1) << 31);
  if (per_worker < 1024) return fail(VINE_ERR_CAPACITY, "variant engine: label arena too small");

  VBuffers B;
  VParams P;
  std::memset(&P, 0, sizeof(P));
  P.g = g->dev();
  P.nq = nq;
  int32_t *d_src, *d_dst, *d_found, *d_status, *d_plen;
  float *d_L, *d_H = nullptr, *d_M = nullptr, *d_cost, *d_delay, *d_extra;
  int64_t *d_stats = nullptr, *d_pstart;
  unsigned long long *d_ctr;
  VINE_TRY(B.alloc(&d_src, nq));
  VINE_TRY(B.alloc(&d_dst, nq));
  VINE_TRY(B.alloc(&d_L, nq));
  if (hop_limit) VINE_TRY(B.alloc(&d_H, nq));
  if (maxcost_limit) VINE_TRY(B.alloc(&d_M, nq));
  VINE_TRY(B.alloc(&d_cost, nq));
  VINE_TRY(B.alloc(&d_delay, nq));
  VINE_TRY(B.alloc(&d_extra, (size_t)nq * 2));
  VINE_TRY(B.alloc(&d_found, nq));
  VINE_TRY(B.alloc(&d_status, nq));
  VINE_TRY(B.alloc(&d_plen, nq));
  VINE_TRY(B.alloc(&d_pstart, nq));
  if (out->stats) VINE_TRY(B.alloc(&d_stats, (size_t)nq * VINE_STAT_COUNT));
  VINE_TRY(B.alloc(&d_ctr, 2));
  VINE_TRY(B.alloc(&P.head, (size_t)slots * g->n));
  VINE_TRY(B.alloc(&P.near, (size_t)slots * near_cap));
  VINE_TRY(B.alloc(&P.far, (size_t)slots * far_cap));
  VINE_TRY(B.alloc(&P.pool, (size_t)slots * per_worker));
  const int64_t path_cap = std::max<int64_t>((int64_t)nq * 4096, 1 << 20);
  VINE_TRY(B.alloc(&P.path_arena, path_cap));
  cudaStream_t s = g->stream;
  VINE_CUDA_TRY(cudaMemcpyAsync(d_src, src, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
  VINE_CUDA_TRY(cudaMemcpyAsync(d_dst, dst, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s));
  VINE_CUDA_TRY(cudaMemcpyAsync(d_L, delay_limit, sizeof(float) * nq, cudaMemcpyHostToDevice, s));
  if (hop_limit)
    VINE_CUDA_TRY(cudaMemcpyAsync(d_H, hop_limit, sizeof(float) * nq, cudaMemcpyHostToDevice, s));
  if (maxcost_limit)
    VINE_CUDA_TRY(cudaMemcpyAsync(d_M, maxcost_limit, sizeof(float) * nq, cudaMemcpyHostToDevice, s));
  VINE_CUDA_TRY(cudaMemsetAsync(P.head, 0, sizeof(uint64_t) * (size_t)slots * g->n, s));
  VINE_CUDA_TRY(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * 2, s));
  P.src = d_src;
  P.dst = d_dst;
  P.lim_delay = d_L;
  P.lim_hop = d_H;
  P.lim_max = d_M;
  P.cost = d_cost;
  P.delay = d_delay;
  P.extra = d_extra;
  P.found = d_found;
  P.status = d_status;
  P.stats = d_stats;
  P.near_mask = near_cap - 1;
  P.far_cap = far_cap;
  P.pool_per_worker = per_worker;
  P.path_cap = path_cap;
  P.path_top = d_ctr + 1;
  P.path_start = d_pstart;
  P.path_len = d_plen;
  P.queue = d_ctr;
  P.epoch_base = 1;  // head[] is cleared per call: epochs 1 .. nq
  P.width = c.bucket_width > 0.0f ? c.bucket_width : std::max(1.0f, g->mean_len);
  P.lock_log2 = lock_log2;
  P.wait_limit = c.wait_limit > 0 ? c.wait_limit : (1ll << 26);
  P.time_limit_ns = c.time_limit_ms > 0   ? (unsigned long long)c.time_limit_ms * 1000000ull
                    : c.time_limit_ms == 0 ? 600000ull * 1000000ull
                                           : 0ull;
  int rc;
  switch (kind) {
    case VINE_LABEL_HOP: rc = launch_variant<VINE_LABEL_HOP>(P, slots, threads, smem, s); break;
    case VINE_LABEL_MAXCOST: rc = launch_variant<VINE_LABEL_MAXCOST>(P, slots, threads, smem, s); break;
    case VINE_LABEL_QOS: rc = launch_variant<VINE_LABEL_QOS>(P, slots, threads, smem, s); break;
    default: rc = launch_variant<VINE_LABEL_CSP>(P, slots, threads, smem, s); break;
  }
  if (rc != VINE_OK) {
    cudaStreamSynchronize(s);
    return rc;
  }
  std::vector<int32_t> st((size_t)nq), plen((size_t)nq);
  std::vector<int64_t> pstart((size_t)nq);
  std::vector<float> ex((size_t)nq * 2);
  if (cudaMemcpyAsync(out->cost, d_cost, sizeof(float) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(out->delay, d_delay, sizeof(float) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(out->found, d_found, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(st.data(), d_status, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(plen.data(), d_plen, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(pstart.data(), d_pstart, sizeof(int64_t) * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(ex.data(), d_extra, sizeof(float) * 2 * nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      (out->stats && cudaMemcpyAsync(out->stats, d_stats, sizeof(int64_t) * VINE_STAT_COUNT * nq,
                                     cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaStreamSynchronize(s);
    return fail(VINE_ERR_CUDA, std::string("variant engine failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  if (extra) std::memcpy(extra, ex.data(), sizeof(float) * 2 * nq);
  int result = VINE_OK, n_failed = 0;
  for (int32_t q = 0; q < nq; ++q) {
    if (out->status) out->status[q] = st[q];
    if (st[q] != VINE_OK) {
      ++n_failed;
      if (result == VINE_OK) result = st[q];
    }
  }
  if (result != VINE_OK)
    set_error(std::to_string(n_failed) + " of " + std::to_string(nq) +
              " queries failed; first status " + std::to_string(result));
  if (out->path_offsets) {
    int64_t run = 0;
    for (int32_t q = 0; q < nq; ++q) {
      out->path_offsets[q] = run;
      run += plen[q];
    }
    out->path_offsets[nq] = run;
    if (run > out->path_capacity || !out->path) {
      if (result == VINE_OK) result = fail(VINE_ERR_CAPACITY, "path buffer too small (need " + std::to_string(run) + ")");
    } else {
      for (int32_t q = 0; q < nq; ++q)
        if (plen[q] > 0 &&
            cudaMemcpy(out->path + out->path_offsets[q], P.path_arena + pstart[q],
                       sizeof(int32_t) * plen[q], cudaMemcpyDeviceToHost) != cudaSuccess)
          return fail(VINE_ERR_CUDA, "path download failed");
    }
  }
  return result;
}

}  // extern "C"
