// Auxiliary kernels of the engines: query ordering and path extraction.
// The reference never extracts a path for CSP=1 (ck_CSPP_path,
// algorithm/cspp.cuh:327-373, is never launched and the father_id / pre
// fields it walks are commented out, include/label.hpp:176-177).  Here every
// accepted label stores its parent's arena index, each worker copies its
// answer's path out at the end of the query, and these kernels pack the
// paths in query order.

#include "engine_host.h"

namespace vine {

namespace {

// Orders queries by decreasing budget (classes 1/128 of an octave wide), a
// cheap proxy for query difficulty: the longest queries start first, so the
// persistent workers finish together (longest-processing-time-first).
constexpr int kOrderBins = 4096;

__device__ __forceinline__ int budget_bin(float b) {
  if (!(b > 0.0f) || !isfinite(b)) return 0;
  return min(kOrderBins - 1, (int)(log2f(b + 1.0f) * 128.0f));
}

__global__ void order_kernel(int32_t nq, const float *budget, int32_t *order) {
  __shared__ int hist[kOrderBins];
  __shared__ int warp_tot[32];
  for (int i = threadIdx.x; i < kOrderBins; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < nq; i += blockDim.x)
    atomicAdd(&hist[kOrderBins - 1 - budget_bin(budget[i])], 1);
  __syncthreads();
  // exclusive scan of the histogram: each thread owns a contiguous run of bins
  const int per = kOrderBins / blockDim.x;  // blockDim.x divides kOrderBins
  const int b0 = threadIdx.x * per;
  int run = 0;
  for (int k = 0; k < per; ++k) run += hist[b0 + k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int v = lane < nw ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane < nw) warp_tot[lane] = v;  // inclusive warp totals
  }
  __syncthreads();
  int base = (incl - run) + (warp > 0 ? warp_tot[warp - 1] : 0);
  for (int k = 0; k < per; ++k) {
    const int h = hist[b0 + k];
    hist[b0 + k] = base;
    base += h;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nq; i += blockDim.x)
    order[atomicAdd(&hist[kOrderBins - 1 - budget_bin(budget[i])], 1)] = i;
}

__global__ void path_len_kernel(const int32_t *len, int32_t nq, int64_t *off) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nq) off[q] = len[q];
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

// One warp per query copies its path segment.
__global__ void path_gather_kernel(const int32_t *arena, const int64_t *start,
                                   const int32_t *len, int32_t nq, const int64_t *off,
                                   int32_t *path) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;
  const int64_t s = start[q], o = off[q];
  for (int32_t i = lane; i < len[q]; i += 32) path[o + i] = arena[s + i];
}

}  // namespace

int order_queries(int32_t nq, const float *d_budget, int32_t *d_order, cudaStream_t stream) {
  if (nq <= 0) return VINE_OK;
  order_kernel<<<1, 1024, 0, stream>>>(nq, d_budget, d_order);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

int path_offsets(const PathOut &p, int32_t nq, int64_t *d_offsets, cudaStream_t stream) {
  if (nq <= 0) {
    VINE_CUDA_TRY(cudaMemsetAsync(d_offsets, 0, sizeof(int64_t), stream));
    return VINE_OK;
  }
  path_len_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(p.len, nq, d_offsets);
  scan_i64_kernel<<<1, 1024, 0, stream>>>(d_offsets, nq);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

int path_gather(const PathOut &p, int32_t nq, const int64_t *d_offsets, int32_t *d_path,
                cudaStream_t stream) {
  if (nq <= 0) return VINE_OK;
  path_gather_kernel<<<(nq * 32 + 255) / 256, 256, 0, stream>>>(p.arena, p.start, p.len, nq,
                                                                 d_offsets, d_path);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

}  // namespace vine
