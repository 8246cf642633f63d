// sph_mlp.cu - the learned near-wall closure network: 16 -> 64 -> 64 -> 4,
// SiLU, trained and evaluated with BF16 operands on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation). FP32 master weights and Adam state;
// BF16 copies feed the matrix products. No reference counterpart.
//
// Parameter layout (5,508 floats): W1[64][16], b1[64], W2[64][64], b2[64],
// W3[4][64], b3[4]; W[out][in], so y = W x + b.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sph_cuda.h"
#include "sph_mlp.cuh"

using namespace sphmlp;

struct SphMlp {
  int dev = 0;
  cudaStream_t st = nullptr;
  float* w = nullptr;        // FP32 master parameters
  float* m = nullptr;        // Adam first moment
  float* v = nullptr;        // Adam second moment
  __nv_bfloat16* wb = nullptr;  // BF16 copies of W1, W2, W3 (biases stay FP32)
  float* grad = nullptr;     // summed gradient of a mini-batch
  float* part = nullptr;     // per-CTA gradient partials
  int part_rows = 0;
  float* loss = nullptr;     // per-CTA loss partials
  int64_t step = 0;
  int sms = 148;             // SMs of the device (queried at creation)
  std::vector<void*> allocs;
};

namespace {

template <class T>
cudaError_t mal(SphMlp* h, T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) h->allocs.push_back(*p);
  return e;
}

int status(cudaError_t e) {
  if (e == cudaSuccess) return SPH_OK;
  return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

// Per CTA: kWarps warps x 16 samples. Forward and backward of the closure
// network on BF16 tensor-core tiles; each CTA writes its gradient sum (and
// loss sum) to its row of `part` (deterministic, no atomics).
constexpr int kWarps = 4;
constexpr int kCtaSamples = kWarps * 16;

struct WarpSmem {
  __nv_bfloat16 x[16 * 16];
  float z1[16 * 64];
  __nv_bfloat16 h1[16 * 64];
  float z2[16 * 64];
  __nv_bfloat16 h2[16 * 64];
  __nv_bfloat16 dy[16 * 16];   // dL/dy in bf16, outputs padded to 16
  __nv_bfloat16 dz[16 * 64];   // dL/dz2, then dL/dz1
  float y[16 * 4];
};

struct CtaSmem {
  __nv_bfloat16 w1[64 * 16];
  __nv_bfloat16 w2[64 * 64];
  __nv_bfloat16 w3[16 * 64];   // W3 padded to 16 output rows
  float b[kParamBias];          // b1, b2, b3
  float g[kWarps][kParams];     // per-warp gradient
  WarpSmem wp[kWarps];
};

__global__ void __launch_bounds__(kWarps * 32)
k_mlp_train(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ w, const float* __restrict__ x,
            const float* __restrict__ t, const uint32_t* __restrict__ perm, int n, int batch_lo,
            int batch_n, float* __restrict__ part, float* __restrict__ loss_part, int want_grad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CtaSmem& S = *reinterpret_cast<CtaSmem*>(smem_raw);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_weights_smem(wb, w, S.w1, S.w2, S.w3, S.b);
  for (int i = threadIdx.x; i < kWarps * kParams; i += blockDim.x) (&S.g[0][0])[i] = 0.0f;
  __syncthreads();
  WarpSmem& W = S.wp[warp];
  int base = blockIdx.x * kCtaSamples + warp * 16;  // within the mini-batch
  // gather 16 samples (rows past the batch are zero with zero target weight)
  for (int q = lane; q < 16 * 16; q += 32) {
    int r = q >> 4, c = q & 15;
    int j = base + r;
    float v = 0.0f;
    if (j < batch_n) {
      int s = (int)perm[batch_lo + j];
      v = x[(size_t)s * kIn + c];
    }
    W.x[q] = __float2bfloat16_rn(v);
  }
  __syncwarp();
  forward_tile(W.x, S.w1, S.w2, S.w3, S.b, W.z1, W.h1, W.z2, W.h2, W.y, lane);
  // dL/dy of the mean squared error over batch_n x 4 outputs
  float lsum = 0.0f;
  const float scale = 2.0f / (float)(batch_n * kOut);
  for (int q = lane; q < 16 * 16; q += 32) {
    int r = q >> 4, c = q & 15;
    int j = base + r;
    float d = 0.0f;
    if (j < batch_n && c < kOut) {
      int s = (int)perm[batch_lo + j];
      float e = W.y[r * 4 + c] - t[(size_t)s * kOut + c];
      lsum += e * e;
      d = scale * e;
    }
    W.dy[q] = __float2bfloat16_rn(d);
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  __syncwarp();
  if (want_grad) backward_tile(W.x, S.w2, S.w3, W.z1, W.h1, W.z2, W.h2, W.dy, W.dz, S.g[warp], lane);
  __syncthreads();
  for (int i = threadIdx.x; i < kParams && want_grad; i += blockDim.x) {
    float a = 0.0f;
    for (int q = 0; q < kWarps; ++q) a += S.g[q][i];
    part[(size_t)blockIdx.x * kParams + i] = a;
  }
  __shared__ float ls[kWarps];
  if (lane == 0) ls[warp] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f;
    for (int q = 0; q < kWarps; ++q) a += ls[q];
    loss_part[blockIdx.x] = a;
  }
}

// Sum the CTA partials in order, then one Adam step (bias-corrected) on the
// FP32 masters and refresh of the BF16 copies.
__global__ void k_adam(int ctas, const float* __restrict__ part, float* __restrict__ grad, float* __restrict__ w,
                       float* __restrict__ m, float* __restrict__ v, __nv_bfloat16* __restrict__ wb, float lr,
                       float b1, float b2, float eps, float c1, float c2, int apply) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  float g = 0.0f;
  for (int c = 0; c < ctas; ++c) g += part[(size_t)c * kParams + i];
  grad[i] = g;
  if (!apply) return;
  float mi = b1 * m[i] + (1.0f - b1) * g;
  float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  float mh = mi / c1, vh = vi / c2;
  float wi = w[i] - lr * mh / (sqrtf(vh) + eps);
  w[i] = wi;
  int bi = bf16_index(i);
  if (bi >= 0) wb[bi] = __float2bfloat16_rn(wi);
}

__global__ void k_refresh_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  int bi = bf16_index(i);
  if (bi >= 0) wb[bi] = __float2bfloat16_rn(w[i]);
}

__global__ void __launch_bounds__(kWarps * 32)
k_mlp_forward(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ w, const float* __restrict__ x,
              int n, float* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CtaSmem& S = *reinterpret_cast<CtaSmem*>(smem_raw);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_weights_smem(wb, w, S.w1, S.w2, S.w3, S.b);
  __syncthreads();
  WarpSmem& W = S.wp[warp];
  for (int base = (blockIdx.x * kWarps + warp) * 16; base < n; base += gridDim.x * kWarps * 16) {
    for (int q = lane; q < 16 * 16; q += 32) {
      int r = q >> 4, c = q & 15;
      W.x[q] = __float2bfloat16_rn(base + r < n ? x[(size_t)(base + r) * kIn + c] : 0.0f);
    }
    __syncwarp();
    forward_tile(W.x, S.w1, S.w2, S.w3, S.b, W.z1, W.h1, W.z2, W.h2, W.y, lane);
    for (int q = lane; q < 16 * 4; q += 32) {
      int r = q >> 2;
      if (base + r < n) y[(size_t)(base + r) * kOut + (q & 3)] = W.y[q];
    }
    __syncwarp();
  }
}

int upload(SphMlp* h, const float* src, size_t count, float** dst) {
  cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(count, 1) * sizeof(float));
  if (e == cudaSuccess && count) e = cudaMemcpyAsync(*dst, src, count * sizeof(float), cudaMemcpyHostToDevice, h->st);
  return status(e);
}

int ensure_parts(SphMlp* h, int rows) {
  if (rows <= h->part_rows) return SPH_OK;
  if (h->part) cudaFree(h->part);
  if (h->loss) cudaFree(h->loss);
  cudaError_t e = cudaMalloc((void**)&h->part, (size_t)rows * kParams * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->loss, (size_t)rows * sizeof(float));
  h->part_rows = e == cudaSuccess ? rows : 0;
  return status(e);
}

}  // namespace

extern "C" {

int sph_mlp_create(int device, uint64_t seed, SphMlp** out) {
  if (!out) return SPH_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  SphMlp* h = new SphMlp();
  h->dev = device;
  cudaSetDevice(device);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) h->sms = sms;
  cudaError_t e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = mal(h, &h->w, kParams);
  if (e == cudaSuccess) e = mal(h, &h->m, kParams);
  if (e == cudaSuccess) e = mal(h, &h->v, kParams);
  if (e == cudaSuccess) e = mal(h, &h->wb, kBf16Count);
  if (e == cudaSuccess) e = mal(h, &h->grad, kParams);
  if (e == cudaSuccess && cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(CtaSmem)) != cudaSuccess)
    e = cudaErrorInvalidValue;
  if (e == cudaSuccess && cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(CtaSmem)) != cudaSuccess)
    e = cudaErrorInvalidValue;
  if (e != cudaSuccess) {
    sph_mlp_destroy(h);
    return status(e);
  }
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases
  std::vector<float> w(kParams);
  uint64_t s = seed;
  const int fan[3] = {kIn, kHid, kHid};
  const int off_w[3] = {kOffW1, kOffW2, kOffW3}, nw[3] = {kHid * kIn, kHid * kHid, kOut * kHid};
  const int off_b[3] = {kOffB1, kOffB2, kOffB3}, nb[3] = {kHid, kHid, kOut};
  for (int l = 0; l < 3; ++l) {
    double a = 1.0 / std::sqrt((double)fan[l]);
    for (int i = 0; i < nw[l]; ++i) w[off_w[l] + i] = (float)((2.0 * uniform01(s) - 1.0) * a);
    for (int i = 0; i < nb[l]; ++i) w[off_b[l] + i] = (float)((2.0 * uniform01(s) - 1.0) * a);
  }
  int st = sph_mlp_set_params(h, w.data());
  if (st != SPH_OK) {
    sph_mlp_destroy(h);
    return st;
  }
  *out = h;
  return SPH_OK;
}

void sph_mlp_destroy(SphMlp* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  if (h->st) cudaStreamSynchronize(h->st);
  for (void* p : h->allocs) cudaFree(p);
  if (h->part) cudaFree(h->part);
  if (h->loss) cudaFree(h->loss);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

int sph_mlp_set_params(SphMlp* h, const float* params) {
  if (!h || !params) return SPH_ERR_INVALID_ARG;
  cudaSetDevice(h->dev);
  cudaError_t e = cudaMemcpyAsync(h->w, params, kParams * sizeof(float), cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->m, 0, kParams * sizeof(float), h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->v, 0, kParams * sizeof(float), h->st);
  if (e == cudaSuccess) {
    k_refresh_bf16<<<(kParams + 255) / 256, 256, 0, h->st>>>(h->w, h->wb);
    e = cudaStreamSynchronize(h->st);
  }
  h->step = 0;
  return status(e);
}

int sph_mlp_get_params(SphMlp* h, float* params) {
  if (!h || !params) return SPH_ERR_INVALID_ARG;
  cudaSetDevice(h->dev);
  cudaError_t e = cudaMemcpyAsync(params, h->w, kParams * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  return status(e);
}

int sph_mlp_forward(SphMlp* h, const float* x, size_t n, float* y) {
  if (!h || (n && (!x || !y)) || n > 0x7fffffffull) return SPH_ERR_INVALID_ARG;
  if (n == 0) return SPH_OK;
  cudaSetDevice(h->dev);
  float *dx = nullptr, *dy = nullptr;
  int s = upload(h, x, n * kIn, &dx);
  cudaError_t e = s == SPH_OK ? cudaMalloc((void**)&dy, n * kOut * sizeof(float)) : cudaErrorUnknown;
  if (e == cudaSuccess) {
    int blocks = (int)std::min<size_t>((n + kCtaSamples - 1) / kCtaSamples, (size_t)h->sms * 4);
    k_mlp_forward<<<blocks, kWarps * 32, sizeof(CtaSmem), h->st>>>(h->wb, h->w, dx, (int)n, dy);
    e = cudaMemcpyAsync(y, dy, n * kOut * sizeof(float), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  }
  if (dx) cudaFree(dx);
  if (dy) cudaFree(dy);
  return s != SPH_OK ? s : status(e);
}

int sph_mlp_loss_grad(SphMlp* h, const float* x, const float* t, size_t n, float* loss, float* grad) {
  if (!h || !x || !t || n == 0 || n > (1u << 24)) return SPH_ERR_INVALID_ARG;
  cudaSetDevice(h->dev);
  float *dx = nullptr, *dt = nullptr;
  uint32_t* dp = nullptr;
  int s = upload(h, x, n * kIn, &dx);
  if (s == SPH_OK) s = upload(h, t, n * kOut, &dt);
  std::vector<uint32_t> perm(n);
  for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  cudaError_t e = s == SPH_OK ? cudaMalloc((void**)&dp, n * sizeof(uint32_t)) : cudaErrorUnknown;
  int ctas = (int)((n + kCtaSamples - 1) / kCtaSamples);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, perm.data(), n * 4, cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) e = ensure_parts(h, ctas) == SPH_OK ? cudaSuccess : cudaErrorMemoryAllocation;
  if (e == cudaSuccess) {
    k_mlp_train<<<ctas, kWarps * 32, sizeof(CtaSmem), h->st>>>(h->wb, h->w, dx, dt, dp, (int)n, 0, (int)n,
                                                               h->part, h->loss, 1);
    k_adam<<<(kParams + 255) / 256, 256, 0, h->st>>>(ctas, h->part, h->grad, h->w, h->m, h->v, h->wb, 0.0f,
                                                     0.9f, 0.999f, 1e-8f, 1.0f, 1.0f, 0);
    std::vector<float> lp(ctas);
    e = cudaMemcpyAsync(lp.data(), h->loss, ctas * sizeof(float), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess && grad) e = cudaMemcpyAsync(grad, h->grad, kParams * 4, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    double L = 0.0;
    for (float v : lp) L += v;
    if (loss) *loss = (float)(L / (double)(n * kOut));
  }
  if (dx) cudaFree(dx);
  if (dt) cudaFree(dt);
  if (dp) cudaFree(dp);
  return s != SPH_OK ? s : status(e);
}

int sph_mlp_train(SphMlp* h, const float* x, const float* t, size_t n, int batch, int epochs, float lr,
                  uint64_t shuffle_seed, float* epoch_loss) {
  if (!h || !x || !t || n == 0 || n > 0x7fffffffull || batch < 16 || epochs < 1 || !(lr > 0.0f))
    return SPH_ERR_INVALID_ARG;
  cudaSetDevice(h->dev);
  float *dx = nullptr, *dt = nullptr;
  uint32_t* dp = nullptr;
  int s = upload(h, x, n * kIn, &dx);
  if (s == SPH_OK) s = upload(h, t, n * kOut, &dt);
  cudaError_t e = s == SPH_OK ? cudaMalloc((void**)&dp, n * sizeof(uint32_t)) : cudaErrorUnknown;
  int ctas = (batch + kCtaSamples - 1) / kCtaSamples;
  if (e == cudaSuccess) e = ensure_parts(h, ctas) == SPH_OK ? cudaSuccess : cudaErrorMemoryAllocation;
  std::vector<uint32_t> perm(n);
  std::vector<float> lp(ctas);
  uint64_t rs = shuffle_seed;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    for (size_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(rs) % (i + 1)]);
    e = cudaMemcpyAsync(dp, perm.data(), n * 4, cudaMemcpyHostToDevice, h->st);
    double L = 0.0;
    for (size_t lo = 0; lo < n && e == cudaSuccess; lo += (size_t)batch) {
      int bn = (int)std::min<size_t>((size_t)batch, n - lo);
      int c = (bn + kCtaSamples - 1) / kCtaSamples;
      h->step += 1;
      float c1 = 1.0f - powf(b1, (float)h->step), c2 = 1.0f - powf(b2, (float)h->step);
      k_mlp_train<<<c, kWarps * 32, sizeof(CtaSmem), h->st>>>(h->wb, h->w, dx, dt, dp, (int)n, (int)lo, bn,
                                                              h->part, h->loss, 1);
      k_adam<<<(kParams + 255) / 256, 256, 0, h->st>>>(c, h->part, h->grad, h->w, h->m, h->v, h->wb, lr, b1,
                                                       b2, 1e-8f, c1, c2, 1);
      e = cudaMemcpyAsync(lp.data(), h->loss, c * sizeof(float), cudaMemcpyDeviceToHost, h->st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
      for (int q = 0; q < c; ++q) L += lp[q];
    }
    if (epoch_loss) epoch_loss[ep] = (float)(L / (double)(n * kOut));
  }
  if (dx) cudaFree(dx);
  if (dt) cudaFree(dt);
  if (dp) cudaFree(dp);
  return s != SPH_OK ? s : status(e);
}

}  // extern "C"
