// Test kernel: sph::div_h against CUDA's IEEE division over every float r in
// [lo, hi] (bit patterns u0..u1), for one smoothing length h.
#include "sph_kernels.cuh"

__global__ void k_div_check(float h, float inv_h, uint32_t u0, uint32_t u1, unsigned long long* bad,
                            uint32_t* first) {
  sph::SimConst k{};
  k.h = h;
  k.inv_h = inv_h;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = u0 + blockIdx.x * blockDim.x + threadIdx.x; u <= u1; u += stride) {
    const float r = __uint_as_float(u);
    if (__float_as_uint(sph::div_h(r, k)) != __float_as_uint(__fdiv_rn(r, h))) {
      atomicAdd(bad, 1ull);
      atomicMin(first, u);
    }
  }
}

// mismatches over [lo, hi] with inv_h = RN(1/h); first = the smallest failing r's bits (0xffffffff if none)
extern "C" int div_check(float h, float lo, float hi, unsigned long long* mismatches, uint32_t* first) {
  volatile float one = 1.0f;
  const float inv_h = one / h;
  unsigned long long* d_bad = nullptr;
  uint32_t* d_first = nullptr;
  if (cudaMalloc(&d_bad, sizeof(*d_bad)) != cudaSuccess) return 1;
  if (cudaMalloc(&d_first, sizeof(*d_first)) != cudaSuccess) return 1;
  cudaMemset(d_bad, 0, sizeof(*d_bad));
  cudaMemset(d_first, 0xff, sizeof(*d_first));
  uint32_t u0, u1;
  memcpy(&u0, &lo, 4);
  memcpy(&u1, &hi, 4);
  k_div_check<<<148 * 8, 256>>>(h, inv_h, u0, u1, d_bad, d_first);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(mismatches, d_bad, sizeof(*d_bad), cudaMemcpyDeviceToHost);
  cudaMemcpy(first, d_first, sizeof(*d_first), cudaMemcpyDeviceToHost);
  cudaFree(d_bad);
  cudaFree(d_first);
  return e == cudaSuccess ? 0 : 2;
}
