// sph_mlp.cuh - device pieces of the closure network (16 -> 64 -> 64 -> 4,
// SiLU): BF16 tensor-core tiles (mma.sync.m16n8k16, FP32 accumulation) over
// 16 samples per warp, operands staged in shared memory.
#pragma once
#include <cstdint>

#include <cuda_bf16.h>

namespace sphmlp {

constexpr int kIn = 16, kHid = 64, kOut = 4;
constexpr int kOffW1 = 0, kOffB1 = 1024, kOffW2 = 1088, kOffB2 = 5184, kOffW3 = 5248, kOffB3 = 5504;
constexpr int kParams = 5508;
constexpr int kParamBias = 132;   // b1 | b2 | b3 in shared memory
constexpr int kBf16Count = 5376;  // W1 | W2 | W3 in BF16

// Index of master parameter i in the BF16 weight array, -1 for biases.
__host__ __device__ inline int bf16_index(int i) {
  if (i < kOffB1) return i;
  if (i >= kOffW2 && i < kOffB2) return 1024 + (i - kOffW2);
  if (i >= kOffW3 && i < kOffB3) return 5120 + (i - kOffW3);
  return -1;
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C(16x8) += A(16x16) B(16x8) on the tensor cores, A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn] (BF16 in shared memory). Fragment layout of the
// PTX ISA for mma.m16n8k16: g = lane/4, t = lane%4; A rows g and g+8, columns
// 2t, 2t+1 (+8); B rows 2t, 2t+1 (+8), column g; C rows g, g+8, columns 2t, 2t+1.
__device__ __forceinline__ void mma_tile(const __nv_bfloat16* A, int sam, int sak, const __nv_bfloat16* B,
                                         int sbk, int sbn, float c[4], int lane) {
  int g = lane >> 2, t = lane & 3;
  int k0 = 2 * t;
  uint32_t a0 = pack2(A[g * sam + k0 * sak], A[g * sam + (k0 + 1) * sak]);
  uint32_t a1 = pack2(A[(g + 8) * sam + k0 * sak], A[(g + 8) * sam + (k0 + 1) * sak]);
  uint32_t a2 = pack2(A[g * sam + (k0 + 8) * sak], A[g * sam + (k0 + 9) * sak]);
  uint32_t a3 = pack2(A[(g + 8) * sam + (k0 + 8) * sak], A[(g + 8) * sam + (k0 + 9) * sak]);
  uint32_t b0 = pack2(B[k0 * sbk + g * sbn], B[(k0 + 1) * sbk + g * sbn]);
  uint32_t b1 = pack2(B[(k0 + 8) * sbk + g * sbn], B[(k0 + 9) * sbk + g * sbn]);
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Block-wide copy of the BF16 weights (W3 padded with zero rows to 16) and
// FP32 biases into shared memory.
__device__ __forceinline__ void load_weights_smem(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ w,
                                                  __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3,
                                                  float* b) {
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) w1[i] = wb[i];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) w2[i] = wb[1024 + i];
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) w3[i] = i < 256 ? wb[5120 + i] : __float2bfloat16_rn(0.0f);
  for (int i = threadIdx.x; i < kParamBias; i += blockDim.x)
    b[i] = i < 64 ? w[kOffB1 + i] : (i < 128 ? w[kOffB2 + i - 64] : w[kOffB3 + i - 128]);
}

// Forward pass of one 16-sample tile: x[16][16] (BF16) -> z1/h1, z2/h2
// ([16][64], FP32 pre-activations and BF16 activations) -> y[16][4] (FP32).
__device__ __forceinline__ void forward_tile(const __nv_bfloat16* x, const __nv_bfloat16* w1,
                                             const __nv_bfloat16* w2, const __nv_bfloat16* w3, const float* b,
                                             float* z1, __nv_bfloat16* h1, float* z2, __nv_bfloat16* h2,
                                             float* y, int lane) {
  int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma_tile(x, 16, 1, w1 + nt * 8 * 16, 1, 16, c, lane);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int r = g + (e >> 1) * 8, col = nt * 8 + 2 * t + (e & 1);
      float z = c[e] + b[col];
      z1[r * 64 + col] = z;
      h1[r * 64 + col] = __float2bfloat16_rn(silu(z));
    }
  }
  __syncwarp();
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) mma_tile(h1 + kt * 16, 64, 1, w2 + nt * 8 * 64 + kt * 16, 1, 64, c, lane);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int r = g + (e >> 1) * 8, col = nt * 8 + 2 * t + (e & 1);
      float z = c[e] + b[64 + col];
      z2[r * 64 + col] = z;
      h2[r * 64 + col] = __float2bfloat16_rn(silu(z));
    }
  }
  __syncwarp();
  {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) mma_tile(h2 + kt * 16, 64, 1, w3 + kt * 16, 1, 64, c, lane);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int r = g + (e >> 1) * 8, col = 2 * t + (e & 1);
      if (col < 4) y[r * 4 + col] = c[e] + b[128 + col];
    }
  }
  __syncwarp();
}

// One m16n8k16 step with the operands already in registers.
__device__ __forceinline__ void mma_regs(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ldg_pair(const __nv_bfloat16* p) {
  return __ldg(reinterpret_cast<const unsigned int*>(p));
}

// The forward pass of forward_tile with the activations kept in registers:
// the C fragment of two adjacent n-tiles of one layer is the A fragment of
// one k-tile of the next (rows g, g+8; columns 2t, 2t+1 and 2t+8, 2t+9), so
// only the input tile x[16][16] (BF16, shared) and the output y[16][4]
// (FP32, shared) leave the registers. The weights are read from global
// memory (wb: BF16 W1 | W2 | W3; the master FP32 parameters wf for the
// biases) and stay in L1. Same instructions, operands and rounding points as
// forward_tile, so the outputs are identical.
__device__ __forceinline__ void forward_tile_regs(const __nv_bfloat16* x, const __nv_bfloat16* __restrict__ wb,
                                                  const float* __restrict__ wf, float* y, int lane) {
  int g = lane >> 2, t = lane & 3;
  int k0 = 2 * t;
  uint32_t xa0 = pack2(x[g * 16 + k0], x[g * 16 + k0 + 1]);
  uint32_t xa1 = pack2(x[(g + 8) * 16 + k0], x[(g + 8) * 16 + k0 + 1]);
  uint32_t xa2 = pack2(x[g * 16 + k0 + 8], x[g * 16 + k0 + 9]);
  uint32_t xa3 = pack2(x[(g + 8) * 16 + k0 + 8], x[(g + 8) * 16 + k0 + 9]);
  const __nv_bfloat16* w1 = wb;
  const __nv_bfloat16* w2 = wb + 1024;
  const __nv_bfloat16* w3 = wb + 5120;
  uint32_t h1[16];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const __nv_bfloat16* wr = w1 + (nt * 8 + g) * 16 + k0;
    mma_regs(c, xa0, xa1, xa2, xa3, ldg_pair(wr), ldg_pair(wr + 8));
    float bl = __ldg(&wf[kOffB1 + nt * 8 + k0]), bh = __ldg(&wf[kOffB1 + nt * 8 + k0 + 1]);
    h1[(nt >> 1) * 4 + (nt & 1) * 2] = pack2(__float2bfloat16_rn(silu(c[0] + bl)), __float2bfloat16_rn(silu(c[1] + bh)));
    h1[(nt >> 1) * 4 + (nt & 1) * 2 + 1] =
        pack2(__float2bfloat16_rn(silu(c[2] + bl)), __float2bfloat16_rn(silu(c[3] + bh)));
  }
  uint32_t h2[16];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const __nv_bfloat16* wr = w2 + (nt * 8 + g) * 64 + kt * 16 + k0;
      mma_regs(c, h1[kt * 4], h1[kt * 4 + 1], h1[kt * 4 + 2], h1[kt * 4 + 3], ldg_pair(wr), ldg_pair(wr + 8));
    }
    float bl = __ldg(&wf[kOffB2 + nt * 8 + k0]), bh = __ldg(&wf[kOffB2 + nt * 8 + k0 + 1]);
    h2[(nt >> 1) * 4 + (nt & 1) * 2] = pack2(__float2bfloat16_rn(silu(c[0] + bl)), __float2bfloat16_rn(silu(c[1] + bh)));
    h2[(nt >> 1) * 4 + (nt & 1) * 2 + 1] =
        pack2(__float2bfloat16_rn(silu(c[2] + bl)), __float2bfloat16_rn(silu(c[3] + bh)));
  }
  float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    // output columns 4..7 of the padded W3 are zero rows
    uint32_t b0 = 0u, b1 = 0u;
    if (g < 4) {
      const __nv_bfloat16* wr = w3 + g * 64 + kt * 16 + k0;
      b0 = ldg_pair(wr);
      b1 = ldg_pair(wr + 8);
    }
    mma_regs(c, h2[kt * 4], h2[kt * 4 + 1], h2[kt * 4 + 2], h2[kt * 4 + 3], b0, b1);
  }
  if (t < 2) {
    float bl = __ldg(&wf[kOffB3 + k0]), bh = __ldg(&wf[kOffB3 + k0 + 1]);
    y[g * 4 + k0] = c[0] + bl;
    y[g * 4 + k0 + 1] = c[1] + bh;
    y[(g + 8) * 4 + k0] = c[2] + bl;
    y[(g + 8) * 4 + k0 + 1] = c[3] + bh;
  }
}

// Sum of a C-fragment column over the 16 rows (lanes with equal t), in lanes
// 0..3 (columns 2t, 2t+1).
__device__ __forceinline__ void colsum(float c[4], float& s0, float& s1) {
  s0 = c[0] + c[2];
  s1 = c[1] + c[3];
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
}

// Backward pass of one tile given dy[16][16] (BF16, dL/dy in columns 0..3):
// adds dL/dparams of the tile to gsum[kParams] (FP32, shared).
__device__ __forceinline__ void backward_tile(const __nv_bfloat16* x, const __nv_bfloat16* w2,
                                              const __nv_bfloat16* w3, const float* z1, const __nv_bfloat16* h1,
                                              const float* z2, const __nv_bfloat16* h2, const __nv_bfloat16* dy,
                                              __nv_bfloat16* dz, float* gsum, int lane) {
  int g = lane >> 2, t = lane & 3;
  // dW3[o][k] = sum_m dy[m][o] h2[m][k] (rows o >= 4 are padding)
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma_tile(dy, 1, 16, h2 + nt * 8, 64, 1, c, lane);
    if (g < 4) {
      gsum[kOffW3 + g * 64 + nt * 8 + 2 * t] += c[0];
      gsum[kOffW3 + g * 64 + nt * 8 + 2 * t + 1] += c[1];
    }
  }
  // db3
  if (lane < 4) {
    float s = 0.0f;
    for (int m = 0; m < 16; ++m) s += __bfloat162float(dy[m * 16 + lane]);
    gsum[kOffB3 + lane] += s;
  }
  // dz2 = (dy W3) * silu'(z2); db2
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma_tile(dy, 16, 1, w3 + nt * 8, 64, 1, c, lane);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int r = g + (e >> 1) * 8, col = nt * 8 + 2 * t + (e & 1);
      c[e] *= silu_grad(z2[r * 64 + col]);
      dz[r * 64 + col] = __float2bfloat16_rn(c[e]);
    }
    float s0, s1;
    colsum(c, s0, s1);
    if (lane < 4) {
      gsum[kOffB2 + nt * 8 + 2 * t] += s0;
      gsum[kOffB2 + nt * 8 + 2 * t + 1] += s1;
    }
  }
  __syncwarp();
  // dW2[o][k] = sum_m dz2[m][o] h1[m][k]
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma_tile(dz + mt * 16, 1, 64, h1 + nt * 8, 64, 1, c, lane);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int o = mt * 16 + g + (e >> 1) * 8, k = nt * 8 + 2 * t + (e & 1);
        gsum[kOffW2 + o * 64 + k] += c[e];
      }
    }
  // dz1 = (dz2 W2) * silu'(z1) (all tiles first: dz is overwritten after)
  float d1[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
    for (int e = 0; e < 4; ++e) d1[nt][e] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) mma_tile(dz + kt * 16, 64, 1, w2 + kt * 16 * 64 + nt * 8, 64, 1, d1[nt], lane);
  }
  __syncwarp();
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int r = g + (e >> 1) * 8, col = nt * 8 + 2 * t + (e & 1);
      d1[nt][e] *= silu_grad(z1[r * 64 + col]);
      dz[r * 64 + col] = __float2bfloat16_rn(d1[nt][e]);
    }
    float s0, s1;
    colsum(d1[nt], s0, s1);
    if (lane < 4) {
      gsum[kOffB1 + nt * 8 + 2 * t] += s0;
      gsum[kOffB1 + nt * 8 + 2 * t + 1] += s1;
    }
  }
  __syncwarp();
  // dW1[o][k] = sum_m dz1[m][o] x[m][k]
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma_tile(dz + mt * 16, 1, 64, x + nt * 8, 16, 1, c, lane);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int o = mt * 16 + g + (e >> 1) * 8, k = nt * 8 + 2 * t + (e & 1);
        gsum[kOffW1 + o * 16 + k] += c[e];
      }
    }
  __syncwarp();
}

}  // namespace sphmlp
