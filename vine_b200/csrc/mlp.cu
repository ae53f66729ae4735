// Learned bucket scheduler: a 16-64-64-2 ReLU MLP in FP32, trained on the
// GPU by the kernels below (forward, backward, Adam).  The reference chooses
// its bucket width only through the AR model (algorithm/cspp.cuh:254-284);
// the network augments that policy.  It only changes how work is ordered, so
// exactness never depends on it (its outputs are clamped and a non-finite
// output falls back to the AR rule inside the search kernel).
//
// The contraction is 5.3 kFLOP per row, far too small for tensor cores to
// pay off; the kernels tile 32 rows per block in shared memory and let each
// thread own a fixed subset of parameters, so gradient accumulation inside a
// block needs no atomics (one atomicAdd per parameter per block at the end).

#include "engine_host.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

namespace vine {
namespace {

constexpr int kTile = 32;
constexpr int kThreads = 128;
constexpr int kW1 = 0, kB1 = kW1 + kHid * kFeat, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid,
              kW3 = kB2 + kHid, kB3 = kW3 + kOut * kHid;

size_t fb_smem_bytes() {
  return sizeof(float) * (2 * (size_t)kMlpParams + kTile * kFeat + 4 * kTile * kHid + 2 * kTile * kOut);
}

// Forward (and optionally backward) over rows idx[0..n) (or 0..n when idx is
// null).  Loss = (1/norm) * sum over rows and outputs of (y - t)^2.
__global__ void __launch_bounds__(kThreads) mlp_fb_kernel(const float *__restrict__ params,
                                                          const float *__restrict__ X,
                                                          const float *__restrict__ T,
                                                          const int32_t *__restrict__ idx, int n,
                                                          float inv_norm, float *grad, float *loss,
                                                          float *Y, int backward) {
  extern __shared__ float sm[];
  float *sW = sm;
  float *sG = sW + kMlpParams;
  float *sX = sG + kMlpParams;
  float *sH1 = sX + kTile * kFeat;
  float *sH2 = sH1 + kTile * kHid;
  float *sD1 = sH2 + kTile * kHid;
  float *sD2 = sD1 + kTile * kHid;
  float *sY = sD2 + kTile * kHid;
  float *sDY = sY + kTile * kOut;
  const int tid = threadIdx.x;
  for (int p = tid; p < kMlpParams; p += kThreads) {
    sW[p] = params[p];
    sG[p] = 0.0f;
  }
  float loss_local = 0.0f;
  __syncthreads();
  const int ntiles = (n + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * kTile;
    for (int o = tid; o < kTile * kFeat; o += kThreads) {
      const int r = o / kFeat, i = o % kFeat;
      const int row = r0 + r;
      float v = 0.0f;
      if (row < n) v = X[(size_t)(idx ? idx[row] : row) * kFeat + i];
      sX[o] = v;
    }
    __syncthreads();
    for (int o = tid; o < kTile * kHid; o += kThreads) {
      const int r = o / kHid, j = o % kHid;
      float acc = sW[kB1 + j];
      for (int i = 0; i < kFeat; ++i) acc += sW[kW1 + j * kFeat + i] * sX[r * kFeat + i];
      sH1[o] = fmaxf(acc, 0.0f);
    }
    __syncthreads();
    for (int o = tid; o < kTile * kHid; o += kThreads) {
      const int r = o / kHid, j = o % kHid;
      float acc = sW[kB2 + j];
      for (int i = 0; i < kHid; ++i) acc += sW[kW2 + j * kHid + i] * sH1[r * kHid + i];
      sH2[o] = fmaxf(acc, 0.0f);
    }
    __syncthreads();
    for (int o = tid; o < kTile * kOut; o += kThreads) {
      const int r = o / kOut, k = o % kOut;
      float acc = sW[kB3 + k];
      for (int i = 0; i < kHid; ++i) acc += sW[kW3 + k * kHid + i] * sH2[r * kHid + i];
      sY[o] = acc;
      const int row = r0 + r;
      float dy = 0.0f;
      if (row < n) {
        const size_t src = (size_t)(idx ? idx[row] : row);
        if (Y) Y[(size_t)row * kOut + k] = acc;
        if (T) {
          const float e = acc - T[src * kOut + k];
          loss_local += e * e;
          dy = 2.0f * e * inv_norm;
        }
      }
      sDY[o] = dy;
    }
    __syncthreads();
    if (!backward) continue;
    for (int o = tid; o < kTile * kHid; o += kThreads) {
      const int r = o / kHid, j = o % kHid;
      float acc = 0.0f;
      for (int k = 0; k < kOut; ++k) acc += sDY[r * kOut + k] * sW[kW3 + k * kHid + j];
      sD2[o] = sH2[o] > 0.0f ? acc : 0.0f;
    }
    __syncthreads();
    for (int o = tid; o < kTile * kHid; o += kThreads) {
      const int r = o / kHid, i = o % kHid;
      float acc = 0.0f;
      for (int j = 0; j < kHid; ++j) acc += sD2[r * kHid + j] * sW[kW2 + j * kHid + i];
      sD1[o] = sH1[o] > 0.0f ? acc : 0.0f;
    }
    __syncthreads();
    // parameter gradients; parameter p is owned by thread p % kThreads
    for (int p = tid; p < kMlpParams; p += kThreads) {
      float g = 0.0f;
      if (p < kB1) {
        const int j = (p - kW1) / kFeat, i = (p - kW1) % kFeat;
        for (int r = 0; r < kTile; ++r) g += sD1[r * kHid + j] * sX[r * kFeat + i];
      } else if (p < kW2) {
        const int j = p - kB1;
        for (int r = 0; r < kTile; ++r) g += sD1[r * kHid + j];
      } else if (p < kB2) {
        const int j = (p - kW2) / kHid, i = (p - kW2) % kHid;
        for (int r = 0; r < kTile; ++r) g += sD2[r * kHid + j] * sH1[r * kHid + i];
      } else if (p < kW3) {
        const int j = p - kB2;
        for (int r = 0; r < kTile; ++r) g += sD2[r * kHid + j];
      } else if (p < kB3) {
        const int k = (p - kW3) / kHid, i = (p - kW3) % kHid;
        for (int r = 0; r < kTile; ++r) g += sDY[r * kOut + k] * sH2[r * kHid + i];
      } else {
        const int k = p - kB3;
        for (int r = 0; r < kTile; ++r) g += sDY[r * kOut + k];
      }
      sG[p] += g;
    }
    __syncthreads();
  }
  if (backward && grad) {
    for (int p = tid; p < kMlpParams; p += kThreads) atomicAdd(&grad[p], sG[p]);
  }
  if (loss) {
    for (int o = 16; o > 0; o >>= 1) loss_local += __shfl_down_sync(0xffffffffu, loss_local, o);
    if ((tid & 31) == 0) atomicAdd(loss, loss_local * inv_norm);
  }
}

__global__ void adam_kernel(float *p, float *m, float *v, const float *g, int n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

int fb_launch(const vine_mlp *m, const float *dX, const float *dT, const int32_t *didx, int n,
              float inv_norm, float *dgrad, float *dloss, float *dY, bool backward,
              cudaStream_t s) {
  // the shared-memory opt-in is a per-device attribute: set it once per device
  static std::mutex mu;
  static bool attr[64] = {};
  const int dev = m->device;
  if (dev < 0 || dev >= 64) return fail(VINE_ERR_INVALID, "device out of range");
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!attr[dev]) {
      VINE_CUDA_TRY(cudaFuncSetAttribute(mlp_fb_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fb_smem_bytes()));
      attr[dev] = true;
    }
  }
  const int ntiles = (n + kTile - 1) / kTile;
  const int grid = std::max(1, std::min(ntiles, 296));
  mlp_fb_kernel<<<grid, kThreads, fb_smem_bytes(), s>>>(m->params, dX, dT, didx, n, inv_norm,
                                                        dgrad, dloss, dY, backward ? 1 : 0);
  VINE_CUDA_TRY(cudaGetLastError());
  return VINE_OK;
}

template <typename T>
struct DevBuf {
  T *p = nullptr;
  ~DevBuf() { cudaFree(p); }
  int alloc(size_t n) {
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess)
      return fail(VINE_ERR_CUDA, "allocation failed");
    return VINE_OK;
  }
};

}  // namespace
}  // namespace vine

using namespace vine;

extern "C" {

int vine_mlp_create(int32_t device, uint64_t seed, const float *params, vine_mlp **out) {
  if (!out) return fail(VINE_ERR_INVALID, "null output");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(VINE_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(VINE_ERR_INVALID, "device out of range");
  VINE_CUDA_TRY(cudaSetDevice(device));
  std::vector<float> p(kMlpParams, 0.0f);
  if (params) {
    std::memcpy(p.data(), params, sizeof(float) * kMlpParams);
  } else {
    // He-uniform weights, zero biases; one mt19937_64 stream in layout order
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int count, int fan_in) {
      const double a = std::sqrt(6.0 / fan_in);
      for (int i = 0; i < count; ++i) {
        const double u = (double)(rng() >> 11) * (1.0 / 9007199254740992.0);
        p[off + i] = (float)((2.0 * u - 1.0) * a);
      }
    };
    fill(kW1, kHid * kFeat, kFeat);
    fill(kW2, kHid * kHid, kHid);
    fill(kW3, kOut * kHid, kHid);
  }
  auto *m = new vine_mlp();
  m->device = device;
  if (cudaMalloc(&m->params, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->adam_m, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMalloc(&m->adam_v, sizeof(float) * kMlpParams) != cudaSuccess) {
    vine_mlp_destroy(m);
    return fail(VINE_ERR_CUDA, "parameter allocation failed");
  }
  if (cudaMemcpy(m->params, p.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->adam_m, 0, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaMemset(m->adam_v, 0, sizeof(float) * kMlpParams) != cudaSuccess ||
      cudaStreamSynchronize(0) != cudaSuccess) {  // the upload has landed before any stream uses it
    vine_mlp_destroy(m);
    return fail(VINE_ERR_CUDA, "parameter upload failed");
  }
  *out = m;
  return VINE_OK;
}

void vine_mlp_destroy(vine_mlp *m) {
  if (!m) return;
  cudaSetDevice(m->device);
  cudaFree(m->params);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  delete m;
}

int vine_mlp_get_params(const vine_mlp *m, float *params) {
  if (!m || !params) return fail(VINE_ERR_INVALID, "bad arguments");
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  VINE_CUDA_TRY(cudaMemcpy(params, m->params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  return VINE_OK;
}

int vine_mlp_set_params(vine_mlp *m, const float *params) {
  if (!m || !params) return fail(VINE_ERR_INVALID, "bad arguments");
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  VINE_CUDA_TRY(cudaMemcpy(m->params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
  // a copy from pageable memory may return before the DMA lands; wait for the
  // legacy stream so a kernel on a non-blocking caller stream sees the values
  VINE_CUDA_TRY(cudaStreamSynchronize(0));
  return VINE_OK;
}

int vine_mlp_forward(const vine_mlp *m, int32_t n, const float *x, float *y) {
  if (!m || n < 0 || (n > 0 && (!x || !y))) return fail(VINE_ERR_INVALID, "bad arguments");
  if (n == 0) return VINE_OK;
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  DevBuf<float> dX, dY;
  VINE_TRY(dX.alloc((size_t)n * kFeat));
  VINE_TRY(dY.alloc((size_t)n * kOut));
  VINE_CUDA_TRY(cudaMemcpy(dX.p, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice));
  VINE_TRY(fb_launch(m, dX.p, nullptr, nullptr, n, 1.0f, nullptr, nullptr, dY.p, false, 0));
  VINE_CUDA_TRY(cudaMemcpy(y, dY.p, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost));
  return VINE_OK;
}

int vine_mlp_loss_grad(const vine_mlp *m, int32_t n, const float *x, const float *y_target,
                       float *loss, float *grad) {
  if (!m || n <= 0 || !x || !y_target || !loss || !grad) return fail(VINE_ERR_INVALID, "bad arguments");
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  DevBuf<float> dX, dT, dG, dL;
  VINE_TRY(dX.alloc((size_t)n * kFeat));
  VINE_TRY(dT.alloc((size_t)n * kOut));
  VINE_TRY(dG.alloc(kMlpParams));
  VINE_TRY(dL.alloc(1));
  VINE_CUDA_TRY(cudaMemcpy(dX.p, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice));
  VINE_CUDA_TRY(cudaMemcpy(dT.p, y_target, sizeof(float) * n * kOut, cudaMemcpyHostToDevice));
  VINE_CUDA_TRY(cudaMemset(dG.p, 0, sizeof(float) * kMlpParams));
  VINE_CUDA_TRY(cudaMemset(dL.p, 0, sizeof(float)));
  VINE_TRY(fb_launch(m, dX.p, dT.p, nullptr, n, 1.0f / n, dG.p, dL.p, nullptr, true, 0));
  VINE_CUDA_TRY(cudaMemcpy(grad, dG.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  VINE_CUDA_TRY(cudaMemcpy(loss, dL.p, sizeof(float), cudaMemcpyDeviceToHost));
  return VINE_OK;
}

int vine_mlp_train(vine_mlp *m, int32_t n, const float *x, const float *y_target, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float *final_loss) {
  if (!m || n <= 0 || !x || !y_target || epochs < 0 || batch <= 0 || !(lr > 0.0f))
    return fail(VINE_ERR_INVALID, "bad arguments");
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  DevBuf<float> dX, dT, dG, dL;
  DevBuf<int32_t> dI;
  VINE_TRY(dX.alloc((size_t)n * kFeat));
  VINE_TRY(dT.alloc((size_t)n * kOut));
  VINE_TRY(dG.alloc(kMlpParams));
  VINE_TRY(dL.alloc(1));
  VINE_TRY(dI.alloc((size_t)n));
  VINE_CUDA_TRY(cudaMemcpy(dX.p, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice));
  VINE_CUDA_TRY(cudaMemcpy(dT.p, y_target, sizeof(float) * n * kOut, cudaMemcpyHostToDevice));
  std::vector<int32_t> perm(n);
  for (int32_t i = 0; i < n; ++i) perm[i] = i;
  std::mt19937_64 rng(seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int e = 0; e < epochs; ++e) {
    for (int32_t i = n - 1; i > 0; --i) {  // Fisher-Yates with a fixed stream
      const int32_t j = (int32_t)(rng() % (uint64_t)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    VINE_CUDA_TRY(cudaMemcpy(dI.p, perm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    for (int32_t b0 = 0; b0 < n; b0 += batch) {
      const int32_t nb = std::min(batch, n - b0);
      VINE_CUDA_TRY(cudaMemsetAsync(dG.p, 0, sizeof(float) * kMlpParams, 0));
      VINE_TRY(fb_launch(m, dX.p, dT.p, dI.p + b0, nb, 1.0f / nb, dG.p, nullptr, nullptr, true, 0));
      m->step++;
      const float c1 = 1.0f - std::pow(b1, (float)m->step);
      const float c2 = 1.0f - std::pow(b2, (float)m->step);
      adam_kernel<<<(kMlpParams + 255) / 256, 256>>>(m->params, m->adam_m, m->adam_v, dG.p,
                                                     kMlpParams, lr, b1, b2, c1, c2, eps);
      VINE_CUDA_TRY(cudaGetLastError());
    }
  }
  VINE_CUDA_TRY(cudaMemset(dL.p, 0, sizeof(float)));
  VINE_TRY(fb_launch(m, dX.p, dT.p, nullptr, n, 1.0f / n, nullptr, dL.p, nullptr, false, 0));
  float l = 0.0f;
  VINE_CUDA_TRY(cudaMemcpy(&l, dL.p, sizeof(float), cudaMemcpyDeviceToHost));
  if (final_loss) *final_loss = l;
  return VINE_OK;
}

// ------------------------------------------- no-allocation loss / gradient
//
// Callers that may not allocate device memory (a scheduler-refinement loop
// running beside a seconds-long batch solve, where cudaFree would wait for
// the whole device; a process whose HBM the label arena already holds) use
// vine_mlp_loss_grad_noalloc.  Its staging buffers live in one fixed array
// in the library image instead of cudaMalloc'd memory.
//
// Scratch layout (floats; every region starts on a 256-byte boundary):
//   [0]                          loss accumulator      (zeroed by each call)
//   [kNaGrad, +kMlpParams)       gradient accumulator  (zeroed by each call)
//   [kNaX, +maxrows * 16)        x rows                (overwritten by each call)
//   [kNaT, +maxrows * 2)         targets               (overwritten by each call)

}  // extern "C"

namespace vine {
namespace {

constexpr int kNaMaxRows = VINE_MLP_NOALLOC_MAX_ROWS;
constexpr size_t kNaAlign = 64;  // floats: 256 bytes
constexpr size_t kNaGrad = kNaAlign;
constexpr size_t kNaX = kNaGrad + ((kMlpParams + kNaAlign - 1) / kNaAlign) * kNaAlign;
constexpr size_t kNaT = kNaX + (size_t)kNaMaxRows * kFeat;
constexpr size_t kNaFloats = kNaT + (size_t)kNaMaxRows * kOut;  // 79,232 floats = 309.5 KiB
static_assert(kNaFloats == 79232, "no-allocation scratch size changed: update the documented size");

static __device__ __align__(256) float g_noalloc_scratch[kNaFloats];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mu;
float *g_na_ptr[kNaMaxDevices] = {};

// Device address of the scratch array on `device` (the current device),
// looked up once per device.
int noalloc_scratch(int device, float **out) {
  if (device < 0 || device >= kNaMaxDevices) return fail(VINE_ERR_INVALID, "device out of range");
  std::lock_guard<std::mutex> lock(g_na_mu);
  if (g_na_ptr[device] == nullptr) {
    float *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(VINE_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                     cudaGetErrorString(e));
    g_na_ptr[device] = p;
  }
  *out = g_na_ptr[device];
  return VINE_OK;
}

}  // namespace
}  // namespace vine

extern "C" {

int vine_mlp_loss_grad_noalloc(const vine_mlp *m, int32_t n, const float *x,
                               const float *y_target, float *loss, float *grad, void *stream) {
  if (!m || !x || !y_target || !loss || !grad) return fail(VINE_ERR_INVALID, "bad arguments");
  if (n < 1 || n > kNaMaxRows)
    return fail(VINE_ERR_INVALID, "vine_mlp_loss_grad_noalloc: n = " + std::to_string(n) +
                                      " rows, allowed 1.." + std::to_string(kNaMaxRows) +
                                      " (VINE_MLP_NOALLOC_MAX_ROWS)");
  VINE_CUDA_TRY(cudaSetDevice(m->device));
  float *scratch = nullptr;
  VINE_TRY(noalloc_scratch(m->device, &scratch));
  cudaStream_t s = (cudaStream_t)stream;
  float *dL = scratch, *dG = scratch + kNaGrad, *dX = scratch + kNaX, *dT = scratch + kNaT;
  VINE_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(float) * kNaX, s));  // loss + gradient
  VINE_CUDA_TRY(cudaMemcpyAsync(dX, x, sizeof(float) * (size_t)n * kFeat, cudaMemcpyHostToDevice, s));
  VINE_CUDA_TRY(cudaMemcpyAsync(dT, y_target, sizeof(float) * (size_t)n * kOut,
                                cudaMemcpyHostToDevice, s));
  VINE_TRY(fb_launch(m, dX, dT, nullptr, n, 1.0f / n, dG, dL, nullptr, true, s));
  VINE_CUDA_TRY(cudaMemcpyAsync(grad, dG, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, s));
  VINE_CUDA_TRY(cudaMemcpyAsync(loss, dL, sizeof(float), cudaMemcpyDeviceToHost, s));
  VINE_CUDA_TRY(cudaStreamSynchronize(s));
  return VINE_OK;
}

}  // extern "C"
