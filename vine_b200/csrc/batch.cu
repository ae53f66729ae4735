// Batched exact CSP engine: one persistent kernel, one query per CTA worker.
//
// Replaces the reference's per-query host loop RUN_CSPP
// (algorithm/cspp.cuh:134-296), which launched expand / recheck / Thrust scan
// / fill kernels and copied the frontier size to the host every round.  Here
// each CTA pulls a query from a device work queue (largest budget first), runs
// the whole search on the device, writes the result and pulls the next query.
// Inside a bucket its warps pull labels from the bucket's queue on their own
// (no block barrier per hop); bucket changes are block-synchronous.  Per-query
// state lives in per-worker HBM regions (reset lazily by tags) and in shared
// memory:
//
//   * bucket table  -- labels of the open bucket keyed by vertex: shared
//                      memory first, per-vertex overflow chains in HBM;
//                      replaces the 96-slot shared hash + global dominance
//                      lists (algorithm/bucket.cuh:80-119,
//                      algorithm/dominance.cuh:15-153)
//   * settled delay -- one float per vertex summarising finished buckets
//   * near queue    -- ring of (arena index, vertex) still to expand in this
//                      bucket, published to the warps in reservation order
//   * far band/rest -- labels beyond the bucket: a band of 64 key bins, so that
//                      opening a bucket scans only the bins below its key, and
//                      a rest pile behind it (the reference's DOP split /
//                      recheck, algorithm/cspp.cuh:179-216,
//                      algorithm/bucket.cuh:217-245)
//   * arena         -- every accepted label with its parent, for paths

#include "engine_host.h"
#include "search.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

namespace vine {

namespace {

__device__ void reverse_bucket_async(Ctx &c, int which, float radius);

// One reverse bound pass (which = 0 delay, 1 length) for the query in `c`,
// run by the whole CTA: bucketed label correcting from the sink.
__device__ void cta_reverse_search(Ctx &c, const RoundBuf &rb, int which, float radius,
                                   float delta) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const int tid = threadIdx.x, G = blockDim.x;
  const uint32_t cap = P.near_mask + 1u;
  if (tid == 0) {
    st.near_head = st.near_tail = 0;
    st.far_n = 0;
    st.far_min_bits = kInfBits;
    VState *sv = &c.vs[st.dst];
    if (which == 0) {
      bool claimed = false;
      relax_pair(&sv->e_del, st.epoch, 0.0f, &claimed);
      if (claimed) atomicExch(reinterpret_cast<unsigned int *>(&sv->hlen), kInfBits);
    } else {
      atomicMin(reinterpret_cast<unsigned int *>(&sv->hlen), 0u);
    }
    c.nearq[0] = (uint32_t)st.dst;
    st.near_tail = 1;
    st.lo = 0.0f;
    st.hi_bits = __float_as_uint(delta);
  }
  __syncthreads();
  for (;;) {
    if (st.abort) break;
    const uint32_t avail = st.near_tail - st.near_head;
    if (avail == 0) {
      if (st.far_n == 0) break;
      if (tid == 0) {
        over_time(P, st);
        st.lo = fmaxf(bucket_hi(st), __uint_as_float(st.far_min_bits));
        st.hi_bits = __float_as_uint(st.lo + delta);
        st.far_min_bits = kInfBits;
        st.far_wpos = 0;
      }
      __syncthreads();
      const uint32_t fn = st.far_n;
      const float hi = bucket_hi(st);
      for (uint32_t base = 0; base < fn; base += (uint32_t)G) {
        const uint32_t i = base + tid;
        const bool valid = i < fn;
        Label item;
        if (valid) item = c.far[i];
        __syncthreads();  // the tile is read before it is overwritten
        if (valid && item.d <= reverse_dist(c, which, item.vid)) {  // not superseded
          if (item.d < hi && st.near_tail - st.near_head < cap - 2u * (uint32_t)G) {
            const uint32_t pos = atomicAdd(&st.near_tail, 1u);
            c.nearq[pos & P.near_mask] = (uint32_t)item.vid;
          } else {
            const uint32_t w = warp_agg_inc(&st.far_wpos);
            c.far[w] = item;
            atomicMin(&st.far_min_bits, __float_as_uint(item.d));
          }
        }
        __syncthreads();
      }
      if (tid == 0) st.far_n = st.far_wpos;
      __syncthreads();
      continue;
    }
    if (!P.sync_rounds) {
      // the whole bucket, warps pulling vertices from the ring
      if (tid == 0) {
        st.near_commit = st.near_tail;
        st.pending = st.near_tail - st.near_head;
      }
      __syncthreads();
      reverse_bucket_async(c, which, radius);
      __syncthreads();
      continue;
    }
    const int n_round = (int)min((uint32_t)rb.cap, avail);
    const uint32_t first = st.near_head;
    __syncthreads();
    if (tid == 0) {
      st.near_head += (uint32_t)n_round;
      st.n_rounds++;
      if (st.n_rounds > kMaxRounds) fail_query(st, VINE_ERR_TIMEOUT, kSiteRounds);
      over_time(P, st);
    }
    __syncthreads();
    reverse_expand_block(c, rb, which, first, n_round, radius, bucket_hi(st), true);
  }
  __syncthreads();
  if (tid == 0) {
    st.near_head = st.near_tail = 0;
    st.far_n = 0;
    st.far_min_bits = kInfBits;
  }
  __syncthreads();
}

// ----------------------------------------------------------------------------
// Asynchronous expansion of the open bucket.  Instead of block-wide rounds,
// every warp repeatedly takes a few entries from the near ring, expands their
// labels (one lane per label, then the warp's arcs 32 at a time with a shuffle
// search for each arc's label), and queues the children that stay in the
// bucket.  Chains of labels inside a bucket (long with exact A* keys, whose
// reduced arc costs are near zero along good paths) then advance at the
// latency of one expansion instead of one block-wide round.
//
// Ring protocol: producers reserve entries with atomicAdd(near_tail), write
// them, and publish them in reservation order by advancing near_commit;
// consumers take entries below near_commit with a CAS on near_head.
// `pending` counts queued labels whose expansion is not finished: children
// are counted before their parent is uncounted, so pending == 0 with nothing
// left to take means the bucket is finished.  Every wait is bounded.
constexpr uint32_t kSlab = 1024;  // arena slots a warp takes at a time

// Publishes ring entries [base, base + k) once every earlier reservation is
// published (lane 0 of the producing warp).  The wait is bounded by
// wait_limit and ends early when the query has failed; a producer that gives
// up publishes nothing (the query is failed, and its consumers stop at the
// abort flag before taking entries).
__device__ __forceinline__ void publish_entries(const SearchParams &P, QueryState &st,
                                                uint32_t base, uint32_t k,
                                                unsigned long long *waited) {
  __threadfence_block();
  volatile uint32_t *cm = &st.near_commit;
  if (*cm != base) {
    const long long t0 = clock64();
    long long polls = 0;
    while (*cm != base) {
      if (*reinterpret_cast<volatile int *>(&st.abort) || ++polls > P.wait_limit) {
        if (!*reinterpret_cast<volatile int *>(&st.abort)) fail_query(st, VINE_ERR_TIMEOUT, kSiteAsync);
        *waited += (unsigned long long)(clock64() - t0);
        return;
      }
    }
    *waited += (unsigned long long)(clock64() - t0);
  }
  *cm = base + k;
}

__device__ __forceinline__ void async_push(Ctx &c, bool is_near, uint32_t idx, int32_t v) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const int lane = threadIdx.x & 31;
  const unsigned nm = __ballot_sync(0xffffffffu, is_near);
  if (nm == 0) return;
  const uint32_t k = (uint32_t)__popc(nm);
  uint32_t base = 0;
  if (lane == 0) {
    base = atomicAdd(&st.near_tail, k);
    atomicAdd(&st.pending, k);
    if (base + k - *reinterpret_cast<volatile uint32_t *>(&st.near_head) > P.near_mask + 1u)
      fail_query(st, VINE_ERR_CAPACITY, kSiteNear);  // entries still written: in bounds
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  if (is_near) {
    const uint32_t rank = (uint32_t)__popc(nm & ((1u << lane) - 1u));
    c.near_ring()[(base + rank) & P.near_mask] = make_uint2(idx, (uint32_t)v);
  }
  __syncwarp();
  if (lane == 0) publish_entries(P, st, base, k, &c.c_publish);
  __syncwarp();
}

__device__ __forceinline__ void bucket_async(Ctx &c) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float hi = bucket_hi(st);
  const uint2 *ring = c.near_ring();
  // polls without any change of (near_commit, pending): only a stuck bucket
  // reaches the limit, however long the other warps' expansions take
  long long idle = 0;
  uint32_t seen_commit = 0xffffffffu, seen_pending = 0xffffffffu;
  uint32_t w_expanded = 0, w_relaxed = 0, w_rounds = 0;
  for (;;) {
    // ---- take up to 32 entries (fewer when the ring is short, so that the
    // ---- idle warps share the work)
    uint32_t h = 0, take = 0;
    int stop = 0;
    if (lane == 0) {
      long long t_idle = 0;
      for (;;) {
        if (*reinterpret_cast<volatile int *>(&st.abort)) {
          stop = 1;
          break;
        }
        // head first, then the commit mark: the mark only grows, so the
        // difference cannot go negative even while other warps move the head
        // (read the other way round, a stale mark below a newer head would
        // wrap and hand out unpublished entries)
        h = *reinterpret_cast<volatile uint32_t *>(&st.near_head);
        __threadfence_block();
        const uint32_t cm = *reinterpret_cast<volatile uint32_t *>(&st.near_commit);
        if ((int32_t)(cm - h) > 0) {
          const uint32_t avail = cm - h;
          take = min(32u, max(1u, (avail + (uint32_t)nw - 1u) / (uint32_t)nw));
          if (atomicCAS(&st.near_head, h, h + take) == h) break;
          continue;
        }
        const uint32_t pend = *reinterpret_cast<volatile uint32_t *>(&st.pending);
        if (pend == 0) {
          stop = 1;
          break;
        }
        if (t_idle == 0) t_idle = clock64();
        if (cm != seen_commit || pend != seen_pending) {
          seen_commit = cm;
          seen_pending = pend;
          idle = 0;
        }
        if (++idle > P.wait_limit) {
          fail_query(st, VINE_ERR_TIMEOUT, kSiteAsync);
          stop = 1;
          break;
        }
        if ((idle & 1023) == 0 && over_time(P, st)) {
          stop = 1;
          break;
        }
        __nanosleep(32);
      }
      if (t_idle) c.c_idle += (unsigned long long)(clock64() - t_idle);
    }
    if (__shfl_sync(FULL, stop, 0)) break;
    h = __shfl_sync(FULL, h, 0);
    take = __shfl_sync(FULL, take, 0);
    __threadfence_block();  // entries below near_commit are visible

    // ---- the taken labels, one per lane
    uint32_t idx = 0;
    float d = 0.0f, dl = 0.0f;
    int beg = 0, deg = 0;
    uint2 e = make_uint2(0u, 0u);
    bool entry_ok = false;
    if ((uint32_t)lane < take) {
      e = __ldcg(&ring[(h + (uint32_t)lane) & P.near_mask]);
      // an entry outside the arena or the vertex range would mean a protocol
      // slip: fail the query instead of following it
      entry_ok = (uint64_t)e.x < (uint64_t)P.pool_cap && e.y < (uint32_t)P.g.n;
      if (!entry_ok) fail_query(st, VINE_ERR_INTERNAL, kSiteRing);
    }
    if (entry_ok) {
      idx = e.x;
      const int v = (int)e.y;
      const Label lab = load_label(&P.pool[idx]);  // issued together with the loads below
      const VView s = P.use_bounds ? c.view(v) : VView{0.0f, true, 0.0f, 0.0f, 0u};
      const int r0 = __ldg(&P.g.row[v]);
      const int r1 = __ldg(&P.g.row[v + 1]);
      d = lab.d;
      dl = lab.dl;
      bool live = !(lab.vid & (int)kDeadBit);
      if (live) {
        const float f = d + s.hlen;
        if (!(f < hi)) live = false;
        if (live && P.mode == VINE_MODE_OPTIMAL) {
          const uint64_t key = pack_key(f, dl + s.hdel);
          if (key >= *reinterpret_cast<volatile unsigned long long *>(&st.inc_key)) live = false;
        }
      }
      if (live) {
        beg = r0;
        deg = r1 - r0;
      }
    }
    int incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const int excl = incl - deg;
    // this bucket's counters, kept per warp and folded in once at the end
    w_expanded += (uint32_t)__popc(__ballot_sync(FULL, deg > 0));
    w_relaxed += (uint32_t)total;
    w_rounds += 1u;

    // ---- the arcs, 32 at a time
    if (total > 0) {
      bool failed = false;
      for (int e0 = 0; e0 < total; e0 += 32) {
        // every arc allocates at most one arena slot: keep 32 free in the slab
        int bad = 0;
        if (lane == 0 && st.slab_end[warp] - st.slab_fill[warp] < 32u) {
          const uint32_t b = arena_take(P, st, kSlab);
          if (b == kBadIdx) {
            bad = 1;
          } else {
            st.slab_fill[warp] = b;
            st.slab_end[warp] = b + kSlab;
          }
        }
        if (__shfl_sync(FULL, bad, 0)) {
          failed = true;
          break;
        }
        __syncwarp();
        c.slab_fill = &st.slab_fill[warp];
        const int e = e0 + lane;
        // owner label of arc e: the last lane k with excl_k <= e
        int k = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const int ex = __shfl_sync(FULL, excl, (k + step) & 31);
          if (k + step < 32 && ex <= e) k += step;
        }
        const int obeg = __shfl_sync(FULL, beg, k);
        const int oex = __shfl_sync(FULL, excl, k);
        const float od = __shfl_sync(FULL, d, k);
        const float odl = __shfl_sync(FULL, dl, k);
        const uint32_t oidx = __shfl_sync(FULL, idx, k);
        uint32_t nidx = kNone;
        int u = 0;
        if (e < total) {
          const int j = obeg + (e - oex);
          u = __ldg(&P.g.col[j]);
          const float2 w = __ldg(&P.g.w[j]);
          const VView s = c.view(u);
          offer_with(c, u, od + w.x, odl + w.y, oidx, false, s, &nidx);
        }
        async_push(c, nidx != kNone, nidx, u);
      }
      c.slab_fill = nullptr;
      if (failed) break;  // query failed (abort set)
    }
    __syncwarp();
    if (lane == 0) atomicSub(&st.pending, take);
  }
  // fold the per-warp and per-thread counters into the bucket statistics
  if (lane == 0) {
    atomicAdd(&st.idle_cycles, c.c_idle);
    atomicAdd(&st.publish_cycles, c.c_publish);
    c.c_idle = c.c_publish = 0;
    atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_expanded), (unsigned long long)w_expanded);
    atomicAdd(&st.b_expanded, w_expanded);
    atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_relaxed), (unsigned long long)w_relaxed);
    atomicAdd(&st.b_relaxed, w_relaxed);
    atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_rounds), (unsigned long long)w_rounds);
    atomicAdd(&st.b_rounds, w_rounds);
  }
  atomicAdd(&st.b_dominated, c.c_dominated);
  atomicAdd(&st.b_candidates, c.c_candidates);
  atomicAdd(&st.b_spilled, c.c_spills);
  atomicAdd(&st.b_labels, c.c_near);
  atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
  atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
  atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
  c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
}

// Queues the vertices whose reverse distance improved below the bucket's
// upper key (one per flagged lane) with the ordered publication of async_push;
// entries are vertex ids in the ring's 32-bit view.
__device__ __forceinline__ void async_push_vertex(Ctx &c, bool is_push, int32_t u) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const int lane = threadIdx.x & 31;
  const unsigned nm = __ballot_sync(0xffffffffu, is_push);
  if (nm == 0) return;
  const uint32_t k = (uint32_t)__popc(nm);
  uint32_t base = 0;
  if (lane == 0) {
    base = atomicAdd(&st.near_tail, k);
    atomicAdd(&st.pending, k);
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  if (is_push) {
    const uint32_t rank = (uint32_t)__popc(nm & ((1u << lane) - 1u));
    c.nearq[(base + rank) & P.near_mask] = (uint32_t)u;
  }
  __syncwarp();
  if (lane == 0) publish_entries(P, st, base, k, &c.c_publish);
  __syncwarp();
}

// One bucket [lo, hi) of a reverse bound pass (which = 0 delay, 1 length) with
// warps pulling vertices from the ring, as bucket_async does for labels: each
// vertex's in-arcs are relaxed with its current distance; a vertex improved
// below hi is queued again (while the ring has room), otherwise it goes to the
// far pile.  Distances are exact whatever the order (label correcting).
__device__ void reverse_bucket_async(Ctx &c, int which, float radius) {
  const SearchParams &P = c.P;
  QueryState &st = c.st;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const float hi = bucket_hi(st);
  const uint32_t cap = P.near_mask + 1u;
  long long idle = 0;
  uint32_t seen_commit = 0xffffffffu, seen_pending = 0xffffffffu;
  for (;;) {
    uint32_t h = 0, take = 0;
    int stop = 0;
    if (lane == 0) {
      for (;;) {
        if (*reinterpret_cast<volatile int *>(&st.abort)) {
          stop = 1;
          break;
        }
        // head first, then the commit mark: the mark only grows, so the
        // difference cannot go negative even while other warps move the head
        // (read the other way round, a stale mark below a newer head would
        // wrap and hand out unpublished entries)
        h = *reinterpret_cast<volatile uint32_t *>(&st.near_head);
        __threadfence_block();
        const uint32_t cm = *reinterpret_cast<volatile uint32_t *>(&st.near_commit);
        if ((int32_t)(cm - h) > 0) {
          const uint32_t avail = cm - h;
          take = min(32u, max(1u, (avail + (uint32_t)nw - 1u) / (uint32_t)nw));
          if (atomicCAS(&st.near_head, h, h + take) == h) break;
          continue;
        }
        const uint32_t pend = *reinterpret_cast<volatile uint32_t *>(&st.pending);
        if (pend == 0) {
          stop = 1;
          break;
        }
        if (cm != seen_commit || pend != seen_pending) {
          seen_commit = cm;
          seen_pending = pend;
          idle = 0;
        }
        if (++idle > P.wait_limit) {
          fail_query(st, VINE_ERR_TIMEOUT, kSiteAsync);
          stop = 1;
          break;
        }
        if ((idle & 1023) == 0 && over_time(P, st)) {
          stop = 1;
          break;
        }
        __nanosleep(32);
      }
    }
    if (__shfl_sync(FULL, stop, 0)) break;
    h = __shfl_sync(FULL, h, 0);
    take = __shfl_sync(FULL, take, 0);
    __threadfence_block();  // entries below near_commit are visible

    float dv = 0.0f;
    int beg = 0, deg = 0;
    int v = -1;
    if ((uint32_t)lane < take) {
      v = (int)__ldcg(&c.nearq[(h + (uint32_t)lane) & P.near_mask]);
      if ((uint32_t)v >= (uint32_t)P.g.n) {
        fail_query(st, VINE_ERR_INTERNAL, kSiteRing);  // protocol slip: stop, do not follow
        v = -1;
      }
    }
    if (v >= 0) {
      const int r0 = __ldg(&P.g.rrow[v]);
      const int r1 = __ldg(&P.g.rrow[v + 1]);
      dv = reverse_dist(c, which, v);
      if (dv <= radius) {
        beg = r0;
        deg = r1 - r0;
      }
    }
    int incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const int excl = incl - deg;
    if (lane == 0)
      atomicAdd(reinterpret_cast<unsigned long long *>(&st.n_relaxed), (unsigned long long)total);
    for (int e0 = 0; e0 < total; e0 += 32) {
      const int e = e0 + lane;
      int k = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int ex = __shfl_sync(FULL, excl, (k + step) & 31);
        if (k + step < 32 && ex <= e) k += step;
      }
      const int obeg = __shfl_sync(FULL, beg, k);
      const int oex = __shfl_sync(FULL, excl, k);
      const float odv = __shfl_sync(FULL, dv, k);
      bool push = false;
      int u = 0;
      if (e < total) {
        const int j = obeg + (e - oex);
        u = __ldg(&P.g.rcol[j]);
        const float2 w = __ldg(&P.g.rw[j]);
        const float nd = odv + (which == 0 ? w.y : w.x);
        if (nd <= radius) {
          VState *su = &c.vs[u];
          bool improved = false;
          if (which == 0) {
            bool claimed = false;
            improved = relax_pair(&su->e_del, st.epoch, nd, &claimed);
            if (claimed) atomicExch(reinterpret_cast<unsigned int *>(&su->hlen), kInfBits);
          } else if (__ldcg(&su->e_del) == st.epoch) {
            const unsigned old =
                atomicMin(reinterpret_cast<unsigned int *>(&su->hlen), __float_as_uint(nd));
            improved = __float_as_uint(nd) < old;
          }
          if (improved) {
            // ring while it has room for every warp's pushes, else far pile
            const uint32_t hd = *reinterpret_cast<volatile uint32_t *>(&st.near_head);
            __threadfence_block();
            const uint32_t used = *reinterpret_cast<volatile uint32_t *>(&st.near_tail) - hd;
            if (nd < hi && used + 2u * (uint32_t)blockDim.x < cap) {
              push = true;
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
        }
      }
      async_push_vertex(c, push, u);
    }
    __syncwarp();
    if (lane == 0) atomicSub(&st.pending, take);
  }
}

// Far-pile items per thread whose loads are issued together when a bucket
// opens (more would spill registers around the inlined insert path).
constexpr int kSplitBatch = 2;

// ------------------------------------------------- bulk-staged label tiles
//
// When a bucket opens, the far bins (and, when the band is rebuilt, the rest
// pile) are read tile by tile: contiguous runs of 16-byte labels.  Each tile
// is brought into shared memory by 1-D bulk copies (cp.async.bulk, the TMA
// engine's untiled form; no multicast: the source is this GPU's own memory)
// that complete on an mbarrier, double-buffered so the next tile streams in
// while the block works on the current one.  The labels a tile writes back
// (compacted in place) land below every position a later tile reads, so the
// prefetch never races the write-back.

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global memory to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Generic-proxy writes of the calling thread become visible to later bulk
// copies (async proxy) that read the same global / shared memory.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Two tile buffers and their barriers; `parity` and `busy` are per-thread
// copies of the same values (every thread waits on every tile).
struct TileStage {
  Label *buf[2];
  uint64_t *bar[2];
  uint32_t parity;  // bit k: phase parity the next wait on buffer k expects
  uint32_t busy;    // bit k: a copy into buffer k is in flight
};

// Waits until buffer k's copies have landed (all threads).  Bounded: after
// wait_limit polls the query fails with VINE_ERR_TIMEOUT and the worker is
// marked so that it takes no further query (its buffer may still be written).
__device__ __forceinline__ bool tile_wait(const SearchParams &P, QueryState &st, TileStage &ts,
                                          int k) {
  if (!(ts.busy >> k & 1u)) return true;
  const uint32_t par = ts.parity >> k & 1u;
  bool ok = false;
  for (long long i = 0; i < P.wait_limit; ++i) {
    if (mbar_try_wait(ts.bar[k], par)) {
      ok = true;
      break;
    }
    if (i > 8) __nanosleep(64);
  }
  ts.busy &= ~(1u << k);
  ts.parity ^= 1u << k;
  if (!ok) {
    fail_query(st, VINE_ERR_TIMEOUT, kSiteTile);
    st.tile_broken = 1;
  }
  return ok;
}

// Waits for every copy still in flight (before leaving a staged loop early).
__device__ __forceinline__ void tile_drain(const SearchParams &P, QueryState &st, TileStage &ts) {
  tile_wait(P, st, ts, 0);
  tile_wait(P, st, ts, 1);
}

// Stages labels [base, base + cnt) of a contiguous pile into buffer k
// (thread 0 issues; every thread records the copy as in flight).
__device__ __forceinline__ void tile_issue_pile(TileStage &ts, int k, const Label *pile,
                                                uint32_t base, uint32_t cnt) {
  if (threadIdx.x == 0) {
    fence_proxy_async_shared();  // the block's reads of this buffer are done
    mbar_expect(ts.bar[k], cnt * (uint32_t)sizeof(Label));
    bulk_load(ts.buf[k], pile + base, cnt * (uint32_t)sizeof(Label), ts.bar[k]);
  }
  ts.busy |= 1u << k;
}

// Stages positions [base, base + cnt) of the scanned bins, seen as one
// sequence (bin j holds positions [pre[j], pre[j + 1])), into buffer k.
__device__ __forceinline__ void tile_issue_bins(TileStage &ts, int k, const Label *far,
                                                int64_t bin_cap, const uint32_t *pre, int last,
                                                uint32_t base, uint32_t cnt) {
  if (threadIdx.x == 0) {
    fence_proxy_async_shared();
    mbar_expect(ts.bar[k], cnt * (uint32_t)sizeof(Label));
    const uint32_t end = base + cnt;
    for (int j = 0; j <= last; ++j) {
      const uint32_t a = max(base, pre[j]), b = min(end, pre[j + 1]);
      if (a >= b) continue;
      bulk_load(ts.buf[k] + (a - base), far + (size_t)j * (size_t)bin_cap + (a - pre[j]),
                (b - a) * (uint32_t)sizeof(Label), ts.bar[k]);
    }
  }
  ts.busy |= 1u << k;
}

__global__ void __launch_bounds__(512, 1) batch_kernel(SearchParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int H = 1 << P.table_log2;
  const int NL = 1 << P.lock_log2;
  // round buffers only exist for block-synchronous rounds: in the default
  // mode their shared memory is left to the L1 cache
  const int RC = P.sync_rounds ? P.round_cap : 0;
  int32_t *tv = reinterpret_cast<int32_t *>(smem);
  float2 *tw = reinterpret_cast<float2 *>(tv + H);
  uint32_t *ti = reinterpret_cast<uint32_t *>(tw + H);
  int *locks = reinterpret_cast<int *>(ti + H);
  uint32_t *r_idx = reinterpret_cast<uint32_t *>(locks + NL);
  int *r_vid = reinterpret_cast<int *>(r_idx + RC);
  float *r_d = reinterpret_cast<float *>(r_vid + RC);
  float *r_dl = r_d + RC;
  int *r_beg = reinterpret_cast<int *>(r_dl + RC);
  int *r_off = r_beg + RC;
  int *scan = r_off + RC;
  QueryState &st = *reinterpret_cast<QueryState *>(
      (reinterpret_cast<uintptr_t>(scan + kScanScratch) + 15) & ~(uintptr_t)15);
  TileStage ts;
  ts.buf[0] = reinterpret_cast<Label *>(
      (reinterpret_cast<uintptr_t>(&st + 1) + 127) & ~(uintptr_t)127);
  ts.buf[1] = ts.buf[0] + blockDim.x * kSplitBatch;
  ts.bar[0] = reinterpret_cast<uint64_t *>(ts.buf[1] + blockDim.x * kSplitBatch);
  ts.bar[1] = ts.bar[0] + 1;
  ts.parity = 0;
  ts.busy = 0;

  const int tid = threadIdx.x, G = blockDim.x;
  const int slot = blockIdx.x;
  Ctx c(P, st);
  const RoundBuf rb{r_idx, r_vid, r_d, r_dl, r_beg, r_off, scan, RC};
  c.vs = P.vs + (size_t)slot * P.g.n;
  c.nearq = P.nearq + (size_t)slot * 2 * (P.near_mask + 1u);  // uint2 entries
  c.far = P.far + (size_t)slot * P.far_cap * 4;
  c.rest = P.rest + (size_t)slot * P.rest_cap;
  c.far_key = P.far_key + (size_t)slot * P.far_cap * 4;
  c.rest_key = P.rest_key + (size_t)slot * P.rest_cap;
  c.sinks = P.sinklist + (size_t)slot * P.sink_cap;
  c.bt.tv = tv;
  c.bt.tw = tw;
  c.bt.ti = ti;
  c.bt.log2h = P.table_log2;
  c.bt.probe = P.probe;
  c.bt.locks = locks;
  c.bt.lock_mask = NL - 1;
  c.bt.vs = c.vs;
  c.bt.next = P.next;
  c.bt.chain_steps = P.stats ? &st.n_chain_steps : nullptr;
  c.bt.spin_limit = P.wait_limit;

  for (int i = tid; i < H; i += G) tv[i] = kEmpty;
  for (int i = tid; i < NL; i += G) locks[i] = 0;
  const bool stage = P.split_staging != 0;
  if (tid == 0) {
    if (stage) {
      mbar_init(ts.bar[0]);
      mbar_init(ts.bar[1]);
      fence_proxy_async_shared();  // the initialised barriers are visible to the copy engine
    }
    st.tile_broken = 0;
    st.chunk_fill = 0;
    st.chunk_end = 0;
    st.chunk_lock = 0;
    st.n_chunks = 0;
    st.cur_chunk = 0;
    st.bcur = P.bctr[slot];
  }
  __syncthreads();

  for (;;) {
    if (tid == 0) {
      if (st.tile_broken) {
        st.q = -1;  // a tile buffer may still be written: take no further query
      } else {
        const unsigned long long k = atomicAdd(P.queue, 1ull);
        st.q = (k < (unsigned long long)P.nq) ? (P.order ? P.order[k] : (int)k) : -1;
      }
    }
    __syncthreads();
    const int q = st.q;
    if (q < 0) break;

    // ------------------------------------------------------------- setup
    if (tid == 0) {
      st.t0 = clock64();
      st.g0 = global_ns();
      st.src = P.src[q];
      st.dst = P.dst[q];
      st.budget = P.budget[q];
      st.epoch = (uint32_t)*P.epoch_ptr + (uint32_t)q;
      st.bcur += 1;
      st.qbase = st.bcur;
      st.inc_key = ~0ull;
      st.inc_idx = 0xffffffffu;
      st.inc_lock = 0;
      st.chunk_lock = 0;
      for (int i = 0; i < 32; ++i) st.slab_fill[i] = st.slab_end[i] = 0;
      st.pending = 0;
      st.near_commit = 0;
      st.far_n = 0;
      st.far_wpos = 0;
      st.far_min_bits = kInfBits;
      st.rest_n = 0;
      st.rest_wpos = 0;
      st.rest_min_bits = kInfBits;
      st.band_hi = INFINITY;
      st.near_head = st.near_tail = 0;
      st.abort = 0;
      st.abort_site = 0;
      st.done = 0;
      st.n_expanded = st.n_relaxed = st.n_inserted = st.n_dominated = 0;
      st.n_buckets = st.n_rounds = st.n_spills = 0;
      st.n_chain_steps = 0;
      st.n_bound_rounds = st.bound_cycles = 0;
      st.split_cycles = st.split_items = st.policy_cycles = st.rest_items = 0;
      st.idle_cycles = st.publish_cycles = 0;
      st.load_cycles = st.relax_cycles = 0;
      st.hist_n = 0;
      st.sink_n = 0;
      st.b_labels = st.b_expanded = st.b_rounds = st.b_dominated = 0;
      st.b_candidates = st.b_spilled = st.b_relaxed = 0;
      st.r_live = 0;
      st.width = P.width0;
      st.ar_width = P.width0;
      st.split_cap = P.round_cap;
      for (int i = 0; i < kFeat; ++i) st.x_prev[i] = 0.0f;
      const int s = st.src, t = st.dst;
      const float L = st.budget;
      if (s < 0 || s >= P.g.n || t < 0 || t >= P.g.n || isnan(L)) {
        fail_query(st, VINE_ERR_INVALID, kSiteInvalid);
      } else if (0.0f > L) {
        st.done = 1;  // even the source label violates the budget
      } else {
        pool_rewind(P, st);
        pool_reserve(P, st, 1);
        if (!st.abort) {
          const uint32_t idx = st.chunk_fill++;
          P.pool[idx] = Label{s, 0.0f, 0.0f, -1};
          st.inc_idx = idx;  // the source label (placed below)
          if (s == t) {
            // the source label is the unique Pareto-optimal sink label
            st.inc_key = pack_key(0.0f, 0.0f);
            st.done = 1;
            if (P.mode == VINE_MODE_PARETO) {
              c.sinks[0] = idx;
              st.sink_n = 1;
            }
          }
        }
      }
    }
    __syncthreads();
    if (!st.done && !st.abort) {
      if (P.use_bounds) {
        const long long t_b = clock64();
        const long long r_b = st.n_rounds;
        cta_reverse_search(c, rb, 0, st.budget, P.delta_del);
        cta_reverse_search(c, rb, 1, INFINITY, P.delta_len);
        if (tid == 0) {
          st.bound_cycles = clock64() - t_b;
          st.n_bound_rounds = st.n_rounds - r_b;
        }
      }
      if (tid == 0 && !st.abort) {
        const VView sv = c.view(st.src);
        const uint32_t idx = st.inc_idx;
        st.inc_idx = 0xffffffffu;
        if (!sv.reach) {
          st.done = 1;  // the sink lies beyond the budget
        } else {
          st.lo = sv.hlen;
          st.hi_bits = __float_as_uint(sv.hlen + P.width0);
          st.band_lo = sv.hlen;
          st.band_hi = sv.hlen + P.width0 * (float)P.band_mult;
          st.bin_inv = (float)kBins / (st.band_hi - st.band_lo);
          if (!(st.bin_inv < INFINITY)) st.bin_inv = 0.0f;
          for (int j = 0; j < kBins; ++j) {
            st.bin_n[j] = 0;
            st.bin_min[j] = kInfBits;
          }
          const uint32_t s0 = group_base(st.src, P.table_log2);
          tv[s0] = st.src;
          tw[s0] = make_float2(0.0f, 0.0f);
          ti[s0] = idx;
          c.near_ring()[0] = make_uint2(idx, (uint32_t)st.src);
          st.near_head = 0;
          st.near_tail = 1;
          st.b_labels = 1;
        }
      }
      __syncthreads();
    }
    c.bt.epoch = st.epoch;
    c.bt.qbase = st.qbase;
    c.bt.bcur = st.bcur;

    // --------------------------------------------------- bucket / round loop
    while (!st.done && !st.abort) {
      const uint32_t avail = st.near_tail - st.near_head;
      if (avail == 0) {
        // ---- bucket finished: settle its table labels, pick the next bucket
        const long long t_pol = clock64();
        atomicAdd(&st.b_dominated, c.c_dominated);
        atomicAdd(&st.b_candidates, c.c_candidates);
        atomicAdd(&st.b_spilled, c.c_spills);
        atomicAdd(&st.b_labels, c.c_near);
        atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
        atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
        atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
        c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
        for (int i = tid; i < H; i += G) {
          const int32_t vid = tv[i];
          if (vid != kEmpty) {
            if (!(ti[i] & kDeadBit)) settle(&c.vs[vid], st.epoch, tw[i].y);
            tv[i] = kEmpty;
          }
        }
        if (tid == 0) {
          // band summary (scheduler features and the next bucket's key)
          uint32_t band_n = 0, bmin = kInfBits;
          for (int j = 0; j < kBins; ++j) {
            const uint32_t n = min(st.bin_n[j], (uint32_t)P.bin_cap);
            band_n += n;
            if (n) bmin = min(bmin, st.bin_min[j]);
          }
          st.far_n = band_n;
          st.far_min_bits = bmin;
        }
        __syncthreads();
        if (tid < 32) policy_step(P, st);
        if (tid == 0) {
          st.n_buckets++;
          if (st.n_buckets > kMaxBuckets) fail_query(st, VINE_ERR_TIMEOUT, kSiteRounds);
          over_time(P, st);
          st.rb_band = 0;
          const float fmin = __uint_as_float(min(st.far_min_bits, st.rest_min_bits));
          if (st.far_n == 0 && st.rest_n == 0) {
            st.done = 1;
          } else if (P.mode == VINE_MODE_OPTIMAL && st.inc_key != ~0ull && fmin > key_d(st.inc_key)) {
            st.done = 1;
          } else {
            st.lo = fmaxf(bucket_hi(st), fmin);
            if (st.far_n == 0) {  // band ran dry: a new band starts at the next key
              st.band_lo = st.lo;
              st.band_hi = st.lo + st.width * (float)P.band_mult;
              if (!(st.band_hi > st.lo)) st.band_hi = nextafterf(st.lo, INFINITY);
              st.bin_inv = (float)kBins / (st.band_hi - st.band_lo);
              if (!(st.bin_inv < INFINITY)) st.bin_inv = 0.0f;  // degenerate band: one bin
              for (int j = 0; j < kBins; ++j) {
                st.bin_n[j] = 0;
                st.bin_min[j] = kInfBits;
              }
              st.rb_band = 1;
            } else if (__uint_as_float(st.rest_min_bits) < st.band_hi) {
              st.rb_band = 1;  // labels that found their bin full wait in the rest pile
            }
            if (st.rb_band) {
              st.rest_min_bits = kInfBits;
              st.rest_wpos = 0;
            }
            float hi = fminf(st.lo + st.width, st.band_hi);
            if (!(hi > st.lo)) hi = nextafterf(st.lo, INFINITY);
            st.hi_bits = __float_as_uint(hi);
            st.bcur += 1;  // chains of the finished bucket now count as settled
          }
          st.b_labels = st.b_expanded = st.b_rounds = st.b_dominated = 0;
          st.b_candidates = st.b_spilled = st.b_relaxed = 0;
          st.policy_cycles += clock64() - t_pol;
        }
        __syncthreads();
        if (st.done) break;
        const long long t_split = clock64();
        c.bt.bcur = st.bcur;
        if (st.rb_band) {
          // ---- move rest-pile labels below band_hi into their bins (in
          // ---- place, tile by tile; a label whose bin is full stays)
          const uint32_t rn = st.rest_n;
          const uint32_t rtile = (uint32_t)G * kSplitBatch;
          if (stage) {
            fence_proxy_async_global();  // this thread's pile writes, before the bulk reads
            __syncthreads();
            if (rn > 0) tile_issue_pile(ts, 0, c.rest, 0, min(rtile, rn));
          }
          for (uint32_t base = 0, t = 0; base < rn; base += rtile, ++t) {
            const int k = (int)(t & 1u);
            if (tid == 0) pool_reserve(P, st, rtile);  // for labels offered directly
            if (stage && base + rtile < rn)  // the other buffer was released by the last barrier
              tile_issue_pile(ts, k ^ 1, c.rest, base + rtile, min(rtile, rn - base - rtile));
            __syncthreads();
            const bool landed = stage ? tile_wait(P, st, ts, k) : true;
            if (__syncthreads_or(!landed || st.abort)) {  // the same decision in every thread
              if (stage) tile_drain(P, st, ts);
              break;
            }
            Label item[kSplitBatch];
            float f[kSplitBatch];
#pragma unroll
            for (int b = 0; b < kSplitBatch; ++b) {
              const uint32_t i = base + (uint32_t)(b * G + tid);
              if (i < rn) {
                item[b] = stage ? ts.buf[k][b * G + tid] : c.rest[i];
                f[b] = c.rest_key[i];  // stored with the label: no h lookup
              }
            }
            __syncthreads();  // the whole tile (labels and keys) is read before it is overwritten
#pragma unroll
            for (int b = 0; b < kSplitBatch; ++b) {
              if (base + (uint32_t)(b * G + tid) >= rn) break;
              if (P.mode == VINE_MODE_OPTIMAL &&
                  f[b] > key_d(*reinterpret_cast<volatile unsigned long long *>(&st.inc_key))) {
                // beaten by the incumbent: cannot lead to a better answer
              } else if (!(f[b] < st.band_hi && push_bin(c, item[b], f[b]))) {
                if (f[b] < bucket_hi(st)) {
                  // it belongs to the opening bucket but its bin is full:
                  // offer it now (a far label below hi always enters)
                  const Label &it = item[b];
                  offer(c, it.vid, it.d, it.dl, (uint32_t)it.parent, true);
                } else {
                  const uint32_t w = warp_agg_inc(&st.rest_wpos);
                  c.rest[w] = item[b];
                  c.rest_key[w] = f[b];
                  atomicMin(&st.rest_min_bits, __float_as_uint(f[b]));
                }
              }
            }
            __syncthreads();
          }
          if (tid == 0) {
            st.split_items += rn;
            st.rest_items += rn;
            st.rest_n = st.rest_wpos;
          }
          __syncthreads();
        }
        if (tid == 0) {
          // bins that can hold keys below hi are scanned, as one sequence
          const int last = band_bin(st, bucket_hi(st));
          uint32_t run = 0;
          for (int j = 0; j <= last; ++j) {
            st.bin_pre[j] = run;
            run += min(st.bin_n[j], (uint32_t)P.bin_cap);
            st.bin_n[j] = min(st.bin_n[j], (uint32_t)P.bin_cap);
            st.bin_wpos[j] = 0;
            st.bin_min[j] = kInfBits;
          }
          st.bin_pre[last + 1] = run;
          st.bin_last = last;
        }
        __syncthreads();
        // ---- split the scanned bins: labels below hi enter the bucket
        const int last = st.bin_last;
        const uint32_t fn = st.bin_pre[last + 1];
        const uint32_t tile = (uint32_t)G * kSplitBatch;
        if (stage) {
          fence_proxy_async_global();  // this thread's bin writes, before the bulk reads
          __syncthreads();
          if (fn > 0) tile_issue_bins(ts, 0, c.far, P.bin_cap, st.bin_pre, last, 0, min(tile, fn));
        }
        for (uint32_t base = 0, t = 0; base < fn; base += tile, ++t) {
          const int k = (int)(t & 1u);
          if (tid == 0) pool_reserve(P, st, tile);
          if (stage && base + tile < fn)  // the other buffer was released by the last barrier
            tile_issue_bins(ts, k ^ 1, c.far, P.bin_cap, st.bin_pre, last, base + tile,
                            min(tile, fn - base - tile));
          __syncthreads();
          const bool landed = stage ? tile_wait(P, st, ts, k) : true;
          if (__syncthreads_or(!landed || st.abort)) {  // the same decision in every thread
            if (stage) tile_drain(P, st, ts);
            break;
          }
          Label item[kSplitBatch];
          float fk[kSplitBatch];
          VView sv[kSplitBatch];
          int bj[kSplitBatch];
          const float hi_open = bucket_hi(st);
#pragma unroll
          for (int b = 0; b < kSplitBatch; ++b) {
            const uint32_t i = base + (uint32_t)(b * G + tid);
            bj[b] = 0;
            if (i < fn) {
              int j = 0;
              while (j < last && st.bin_pre[j + 1] <= i) ++j;
              bj[b] = j;
              const size_t at = (size_t)j * (size_t)P.bin_cap + (i - st.bin_pre[j]);
              item[b] = stage ? ts.buf[k][b * G + tid] : c.far[at];
              fk[b] = c.far_key[at];
            }
          }
          // only labels entering the bucket need their vertex's state
#pragma unroll
          for (int b = 0; b < kSplitBatch; ++b)
            if (base + (uint32_t)(b * G + tid) < fn && fk[b] < hi_open) sv[b] = c.view(item[b].vid);
          __syncthreads();  // the whole tile (labels and keys) is read before it is overwritten
          const float inc_d =
              key_d(*reinterpret_cast<volatile unsigned long long *>(&st.inc_key));
#pragma unroll
          for (int b = 0; b < kSplitBatch; ++b) {
            if (base + (uint32_t)(b * G + tid) >= fn) break;
            const Label &it = item[b];
            bool stay;
            if (fk[b] < hi_open) {
              stay = offer_with(c, it.vid, it.d, it.dl, (uint32_t)it.parent, true, sv[b]);
            } else {
              // beyond the bucket: stays unless the incumbent beats its key
              stay = !(P.mode == VINE_MODE_OPTIMAL && fk[b] > inc_d);
            }
            if (stay) {
              // stays in its bin (compacted in place)
              namespace cg = cooperative_groups;
              cg::coalesced_group act = cg::coalesced_threads();
              cg::coalesced_group grp = cg::labeled_partition(act, bj[b]);
              uint32_t wb = 0;
              if (grp.thread_rank() == 0) wb = atomicAdd(&st.bin_wpos[bj[b]], grp.size());
              const uint32_t w = grp.shfl(wb, 0) + grp.thread_rank();
              const size_t at = (size_t)bj[b] * (size_t)P.bin_cap + w;
              c.far[at] = it;
              c.far_key[at] = fk[b];
              atomicMin(&st.bin_min[bj[b]], __float_as_uint(fk[b]));
            }
          }
          __syncthreads();  // the tile's arena allocations end before the next reservation
        }
        __syncthreads();
        if (tid == 0) {
          for (int j = 0; j <= last; ++j) st.bin_n[j] = st.bin_wpos[j];
          st.split_items += fn;
          st.split_cycles += clock64() - t_split;
        }
        __syncthreads();
        continue;
      }

      if (!P.sync_rounds) {
        // ---- the whole bucket, warps pulling work from the near ring
        if (tid == 0) {
          st.near_commit = st.near_tail;
          st.pending = st.near_tail - st.near_head;
        }
        __syncthreads();
        const long long t_async = clock64();
        bucket_async(c);
        __syncthreads();
        if (tid == 0) st.relax_cycles += clock64() - t_async;
        continue;
      }
      // ---- one expansion round over up to split_cap near labels
      const int n_round = (int)min((uint32_t)min(RC, st.split_cap), avail);
      const uint32_t first = st.near_head;
      __syncthreads();
      if (tid == 0) {
        st.near_head += (uint32_t)n_round;
        st.n_rounds++;
        st.b_rounds++;
        if (st.n_rounds > kMaxRounds) fail_query(st, VINE_ERR_TIMEOUT, kSiteRounds);
        over_time(P, st);
      }
      expand_block(c, rb, first, n_round);  // reserves the arena after its scan
      if (tid == 0) {
        st.n_expanded += st.r_live;
        st.b_expanded += st.r_live;
        st.r_live = 0;
      }
      __syncthreads();
    }
    __syncthreads();

    // ------------------------------------------------------------- finish
    atomicAdd((unsigned long long *)&st.n_dominated, (unsigned long long)c.c_dominated);
    atomicAdd((unsigned long long *)&st.n_inserted, (unsigned long long)(c.c_near + c.c_far));
    atomicAdd((unsigned long long *)&st.n_spills, (unsigned long long)c.c_spills);
    c.c_dominated = c.c_candidates = c.c_spills = c.c_near = c.c_far = 0;
    for (int i = tid; i < H; i += G) tv[i] = kEmpty;
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
      copy_out_path(P, st, q, st.abort == 0 && st.inc_key != ~0ull);
      const bool ok = st.abort == 0;
      const bool found = ok && st.inc_key != ~0ull;
      P.status[q] = ok ? VINE_OK : st.abort;
      P.found[q] = found ? 1 : 0;
      P.cost[q] = found ? key_d(st.inc_key) : INFINITY;
      P.odelay[q] = found ? key_dl(st.inc_key) : INFINITY;
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
        s[VINE_STAT_ABORT_SITE] = st.abort_site;
        s[VINE_STAT_BOUND_ROUNDS] = st.n_bound_rounds;
        s[VINE_STAT_BOUND_CYCLES] = st.bound_cycles;
        s[VINE_STAT_SPLIT_CYCLES] = st.split_cycles;
        s[VINE_STAT_SPLIT_ITEMS] = st.split_items;
        s[VINE_STAT_POLICY_CYCLES] = st.policy_cycles;
        s[VINE_STAT_LOAD_CYCLES] = st.load_cycles;
        s[VINE_STAT_RELAX_CYCLES] = st.relax_cycles;
        s[VINE_STAT_CHAIN_STEPS] = (long long)st.n_chain_steps;
        s[VINE_STAT_START_NS] = (long long)st.g0;
        s[VINE_STAT_TIME_NS] = (long long)(global_ns() - st.g0);
        s[VINE_STAT_REST_ITEMS] = st.rest_items;
        s[VINE_STAT_IDLE_CYCLES] = (long long)st.idle_cycles;
        s[VINE_STAT_PUBLISH_CYCLES] = (long long)st.publish_cycles;
      }
    }
    __syncthreads();
  }
  if (tid == 0) P.bctr[slot] = st.bcur;
}

// Hands this call its block of query epochs: counters[5] = base,
// counters[4] += nq.  Kept on the device so that a captured launch sequence
// gets fresh epochs on every replay.
__global__ void epoch_kernel(unsigned long long *counters, int32_t nq) {
  counters[5] = counters[4];
  counters[4] += (unsigned long long)nq;
}

size_t batch_smem_bytes(int table_log2, int lock_log2, int round_cap, int block_threads,
                        int staging) {
  size_t b = ((sizeof(int32_t) + sizeof(float2) + sizeof(uint32_t)) << table_log2) +
             (sizeof(int) << lock_log2) +
             (size_t)round_cap * 24 + kScanScratch * sizeof(int);
  b = (b + 15) & ~(size_t)15;
  b += sizeof(QueryState) + 16;
  if (!staging) return b;
  // two staged label tiles (128-byte aligned) and their barriers
  return b + 128 + 2 * (size_t)block_threads * kSplitBatch * sizeof(Label) + 2 * sizeof(uint64_t);
}

int lock_log2_for(int table_log2) { return std::max(5, table_log2 - 1); }

}  // namespace

void BatchWorkspace::release() {
  cudaFree(vs);
  cudaFree(nearq);
  cudaFree(far);
  cudaFree(sinklist);
  cudaFree(bctr);
  cudaFree(next);
  cudaFree(rest);
  cudaFree(far_key);
  cudaFree(rest_key);
  cudaFree(chunks);
  cudaFree(path_arena);
  cudaFree(path_start);
  cudaFree(path_len);
  cudaFree(pool);
  cudaFree(counters);
  cudaFree(order);
  cudaFree(trace);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  *this = BatchWorkspace();
}

static int ensure_batch_workspace(vine_graph *g, const Resolved &r, int32_t nq) {
  BatchWorkspace &w = g->batch;
  const vine_config &c = r.cfg;
  const int64_t near_cap = int64_t(1) << 22;
  const int sink_cap = 4096;
  const bool same = w.slots == r.slots && w.far_cap == c.far_capacity && w.near_cap == near_cap &&
                    w.pool_cap == c.pool_labels;
  if (!same) {
    w.release();
    const size_t n = (size_t)g->n;
    VINE_CUDA_TRY(cudaMalloc(&w.vs, sizeof(VState) * n * r.slots));
    VINE_CUDA_TRY(cudaMemset(w.vs, 0, sizeof(VState) * n * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.nearq, sizeof(uint2) * (size_t)near_cap * r.slots));
    // the forward band: kBins bins sharing 4 x far_capacity labels (the
    // reverse bound searches use the first far_capacity labels as one pile)
    VINE_CUDA_TRY(cudaMalloc(&w.far, sizeof(Label) * (size_t)c.far_capacity * 4 * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.far_key, sizeof(float) * (size_t)c.far_capacity * 4 * r.slots));
    w.rest_cap = 4 * c.far_capacity;
    VINE_CUDA_TRY(cudaMalloc(&w.rest, sizeof(Label) * (size_t)w.rest_cap * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.rest_key, sizeof(float) * (size_t)w.rest_cap * r.slots));
    w.max_chunks = 4096;
    VINE_CUDA_TRY(cudaMalloc(&w.chunks, sizeof(uint2) * (size_t)w.max_chunks * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.sinklist, sizeof(uint32_t) * (size_t)sink_cap * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.bctr, sizeof(uint32_t) * r.slots));
    VINE_CUDA_TRY(cudaMemset(w.bctr, 0, sizeof(uint32_t) * r.slots));
    VINE_CUDA_TRY(cudaMalloc(&w.pool, sizeof(Label) * (size_t)c.pool_labels));
    VINE_CUDA_TRY(cudaMalloc(&w.next, sizeof(uint32_t) * (size_t)c.pool_labels));
    VINE_CUDA_TRY(cudaMalloc(&w.counters, sizeof(unsigned long long) * 8));
    const unsigned long long init[8] = {0, 0, 0, 0, 1, 1, 0, 0};
    VINE_CUDA_TRY(cudaMemcpy(w.counters, init, sizeof(init), cudaMemcpyHostToDevice));
    w.slots = r.slots;
    w.far_cap = c.far_capacity;
    w.near_cap = near_cap;
    w.sink_cap = sink_cap;
    w.pool_cap = c.pool_labels;
    w.epoch_next = 1;
  }
  if (w.q_cap < nq) {
    cudaFree(w.order);
    cudaFree(w.path_start);
    cudaFree(w.path_len);
    cudaFree(w.path_arena);
    w.order = nullptr;
    w.path_start = nullptr;
    w.path_len = nullptr;
    w.path_arena = nullptr;
    const int64_t cap = std::max<int64_t>(nq, 1024);
    VINE_CUDA_TRY(cudaMalloc(&w.order, sizeof(int32_t) * (size_t)cap));
    VINE_CUDA_TRY(cudaMalloc(&w.path_start, sizeof(int64_t) * (size_t)cap));
    VINE_CUDA_TRY(cudaMalloc(&w.path_len, sizeof(int32_t) * (size_t)cap));
    w.path_cap = cap * 4096;
    VINE_CUDA_TRY(cudaMalloc(&w.path_arena, sizeof(int32_t) * (size_t)w.path_cap));
    w.q_cap = cap;
  }
  if (c.trace && w.trace == nullptr) {
    w.trace_cap = 1 << 20;
    VINE_CUDA_TRY(cudaMalloc(&w.trace, sizeof(float) * VINE_TRACE_COLS * (size_t)w.trace_cap));
  }
  return VINE_OK;
}

int batch_prepare(vine_graph *g, const Resolved &r, int32_t nq, cudaStream_t stream) {
  VINE_TRY(ensure_batch_workspace(g, r, nq));
  BatchWorkspace &w = g->batch;
  if (w.epoch_next > 0xF0000000u - (uint32_t)nq) {
    // epochs would wrap: forget every tag (and any captured launch sequence)
    VINE_CUDA_TRY(cudaMemsetAsync(w.vs, 0, sizeof(VState) * (size_t)g->n * w.slots, stream));
    VINE_CUDA_TRY(cudaMemsetAsync(w.bctr, 0, sizeof(uint32_t) * w.slots, stream));
    const unsigned long long one = 1;
    VINE_CUDA_TRY(cudaMemcpyAsync(w.counters + 4, &one, sizeof(one), cudaMemcpyHostToDevice, stream));
    VINE_CUDA_TRY(cudaStreamSynchronize(stream));
    w.epoch_next = 1;
    if (w.graph_exec) {
      cudaGraphExecDestroy(w.graph_exec);
      w.graph_exec = nullptr;
      w.graph_key = 0;
    }
  }
  w.epoch_next += (uint32_t)nq;
  const size_t smem = batch_smem_bytes(r.cfg.table_log2, lock_log2_for(r.cfg.table_log2),
                                       r.cfg.sync_rounds ? r.round_cap : 0, r.cfg.block_threads,
                                       r.cfg.split_staging);
  VINE_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  return VINE_OK;
}

int batch_enqueue(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
                  const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
                  cudaStream_t stream, PathOut *paths) {
  const vine_config &c = r.cfg;
  BatchWorkspace &w = g->batch;
  SearchParams P;
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
  P.vs = w.vs;
  P.nearq = w.nearq;
  P.near_mask = (uint32_t)(w.near_cap - 1);
  P.far = w.far;
  P.far_cap = w.far_cap;
  P.rest = w.rest;
  P.rest_cap = w.rest_cap;
  P.far_key = w.far_key;
  P.rest_key = w.rest_key;
  P.band_mult = c.band_mult;
  P.chunks = w.chunks;
  P.max_chunks = w.max_chunks;
  P.path_arena = w.path_arena;
  P.path_cap = w.path_cap;
  P.path_top = w.counters + 2;
  P.path_start = w.path_start;
  P.path_len = w.path_len;
  P.sinklist = w.sinklist;
  P.sink_cap = w.sink_cap;
  P.bctr = w.bctr;
  P.pool = w.pool;
  P.next = w.next;
  P.pool_top = w.counters + 0;
  P.pool_cap = w.pool_cap;
  P.chunk = 1u << r.chunk_log2;
  P.queue = w.counters + 1;
  P.epoch_ptr = w.counters + 5;
  P.mode = c.mode;
  P.policy = c.policy;
  P.use_bounds = c.use_bounds;
  P.width0 = r.width0;
  P.ar_scale = c.ar_scale;
  P.len_scale = std::max(1.0f, g->mean_len);
  P.sync_rounds = c.sync_rounds;
  P.binned = 1;
  P.bin_cap = c.far_capacity * 4 / kBins;
  P.delta_del = std::max(1.0f, 4.0f * g->mean_delay);
  P.delta_len = std::max(1.0f, 4.0f * g->mean_len);
  P.round_cap = r.round_cap;
  P.table_log2 = c.table_log2;
  P.lock_log2 = lock_log2_for(c.table_log2);
  P.probe = 16;
  P.grid_scope = 0;
  P.split_staging = c.split_staging;
  P.wait_limit = c.wait_limit;
  P.time_limit_ns = c.time_limit_ms > 0 ? (unsigned long long)c.time_limit_ms * 1000000ull : 0ull;
  P.mlp = (c.policy == VINE_POLICY_MLP && c.mlp) ? c.mlp->params : nullptr;
  P.trace = c.trace ? w.trace : nullptr;
  P.trace_top = w.counters + 3;
  P.trace_cap = w.trace_cap;

  const size_t smem = batch_smem_bytes(c.table_log2, P.lock_log2, c.sync_rounds ? r.round_cap : 0,
                                       c.block_threads, c.split_staging);
  VINE_CUDA_TRY(cudaMemsetAsync(w.counters, 0, sizeof(unsigned long long) * 4, stream));
  epoch_kernel<<<1, 1, 0, stream>>>(w.counters, nq);
  if (c.order_queries) VINE_TRY(order_queries(nq, d_budget, w.order, stream));
  batch_kernel<<<r.slots, c.block_threads, smem, stream>>>(P);
  VINE_CUDA_TRY(cudaGetLastError());
  if (paths) {
    paths->arena = w.path_arena;
    paths->start = w.path_start;
    paths->len = w.path_len;
  }
  return VINE_OK;
}

int batch_run(vine_graph *g, const Resolved &r, int32_t nq, const int32_t *d_src,
              const int32_t *d_dst, const float *d_budget, const DeviceOutputs &out,
              cudaStream_t stream, PathOut *paths) {
  VINE_TRY(batch_prepare(g, r, nq, stream));
  return batch_enqueue(g, r, nq, d_src, d_dst, d_budget, out, stream, paths);
}

int batch_slots(const vine_graph *g, const vine_config &c, int round_cap, int *slots) {
  const size_t smem =
      batch_smem_bytes(c.table_log2, lock_log2_for(c.table_log2), c.sync_rounds ? round_cap : 0,
                       c.block_threads, c.split_staging);
  VINE_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  int per_sm = 0;
  VINE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel,
                                                              c.block_threads, smem));
  if (per_sm < 1) return fail(VINE_ERR_INVALID, "batch kernel does not fit on an SM with this configuration");
  if (c.ctas_per_sm > 0) per_sm = std::min(per_sm, c.ctas_per_sm);
  *slots = per_sm * g->sm_count;
  if (c.max_workers > 0) *slots = std::min(*slots, c.max_workers);
  return VINE_OK;
}

}  // namespace vine
