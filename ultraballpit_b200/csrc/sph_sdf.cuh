// GridSDF (orchestrator geometry.rs:99-175) on the device, exactly: the
// trilinear sample with f32::MAX off the grid and the normalised central
// difference gradient. Node (i, j, k) sits at origin + (i, j, k) * cell,
// index i * ny * nz + j * nz + k. Shared by the force extraction and the
// domain setup kernels.
#pragma once
#include <cstddef>

namespace sph {

// GridSDF::sample (geometry.rs:99-150) exactly, f32::MAX off the grid.
__device__ __forceinline__ float sdf_sample_exact(const float* __restrict__ d, const float origin[3],
                                                  float cell, const int dims[3], float px, float py,
                                                  float pz) {
  float gx = (px - origin[0]) / cell, gy = (py - origin[1]) / cell, gz = (pz - origin[2]) / cell;
  int i0 = (int)floorf(gx), j0 = (int)floorf(gy), k0 = (int)floorf(gz);
  if (i0 < 0 || j0 < 0 || k0 < 0) return 3.40282347e38f;
  if (i0 + 1 >= dims[0] || j0 + 1 >= dims[1] || k0 + 1 >= dims[2]) return 3.40282347e38f;
  float fx = gx - (float)i0, fy = gy - (float)j0, fz = gz - (float)k0;
  size_t ny = dims[1], nz = dims[2];
  size_t b = (size_t)i0 * ny * nz + (size_t)j0 * nz + (size_t)k0, si = ny * nz, sj = nz;
  float c00 = d[b] * (1.0f - fz) + d[b + 1] * fz;
  float c01 = d[b + sj] * (1.0f - fz) + d[b + sj + 1] * fz;
  float c10 = d[b + si] * (1.0f - fz) + d[b + si + 1] * fz;
  float c11 = d[b + si + sj] * (1.0f - fz) + d[b + si + sj + 1] * fz;
  float c0 = c00 * (1.0f - fy) + c01 * fy;
  float c1 = c10 * (1.0f - fy) + c11 * fy;
  return c0 * (1.0f - fx) + c1 * fx;
}

// GridSDF::gradient (geometry.rs:153-175): central differences at half a
// cell, normalised; zero where the magnitude is at most 1e-8.
__device__ __forceinline__ void sdf_gradient_exact(const float* __restrict__ d, const float origin[3], float cell,
                                                   const int dims[3], float px, float py, float pz,
                                                   float out[3]) {
  float h = cell * 0.5f;
  float gx = (sdf_sample_exact(d, origin, cell, dims, px + h, py, pz) -
              sdf_sample_exact(d, origin, cell, dims, px - h, py, pz)) / (2.0f * h);
  float gy = (sdf_sample_exact(d, origin, cell, dims, px, py + h, pz) -
              sdf_sample_exact(d, origin, cell, dims, px, py - h, pz)) / (2.0f * h);
  float gz = (sdf_sample_exact(d, origin, cell, dims, px, py, pz + h) -
              sdf_sample_exact(d, origin, cell, dims, px, py, pz - h)) / (2.0f * h);
  float mag = sqrtf(gx * gx + gy * gy + gz * gz);
  if (mag > 1e-8f) {
    out[0] = gx / mag;
    out[1] = gy / mag;
    out[2] = gz / mag;
  } else {
    out[0] = out[1] = out[2] = 0.0f;
  }
}

}  // namespace sph
