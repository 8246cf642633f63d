// sph_kernels.cuh - sm_100a kernels of the WCSPH step.
//
// Compiled with --fmad=false and IEEE division/square root so that every f32
// operation rounds exactly as the reference CPU kernel's (Rust never fuses
// a*b+c). Neighbour loops visit cells dz -> dy -> dx and, inside a cell,
// particles in ascending original index, which is the reference visit order
// (kernel/src/neighbor.rs:129-182); boundary terms are summed in ascending
// boundary index (sph.rs:148-156, 391-408; boundary.rs:161-179), and the
// Adami boundary pressure sums fluid terms in ascending fluid index
// (boundary.rs:109-123). Together these make the step bit-identical to the
// reference arithmetic.
//
// Storage: particles live sorted by (cell rank, original id), where the cell
// rank orders cells by 30-bit Morton code (or by linear hash). Per particle,
// float4 packs keep one 16-byte load per neighbour field:
//   pos    (x, y, z, m)           velout (v after kick 2, rho)
//   vel    (v after kick 1, -)    acc    (a, 0)
//   rv     (rho_old, m/rho_old)   rf     (rho_new, p/rho_new^2)
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "sph_cuda.h"
#include "sph_mlp.cuh"
#include "sph_sdf.cuh"

namespace sph {

constexpr uint32_t kIdMask = 0x7fffffffu;
constexpr uint32_t kAirBit = 0x80000000u;
constexpr float kWaterRho0 = 1000.0f;  // eos.rs:7
constexpr float kAirRho0 = 1.204f;     // eos.rs:10
constexpr int kAdamiCap = 256;         // fluid terms per boundary particle
constexpr int kCellCap = 4096;         // particles per cell for the id ranking
constexpr uint32_t kNbrCap = 128;      // listed neighbours per particle
// The neighbour kernels are latency-bound on gathered loads, so occupancy
// pays more than registers: k_forces and k_xsph_drift (whose replays put two
// neighbours' gathers in flight before using them) are capped at 56
// registers, k_density (whose warp scan holds its shared scratch per warp) at
// SPH_MAXNREG_DENSITY (__maxnreg__ below; each measured at 2M particles).

#ifndef SPH_MAXNREG_DENSITY
#define SPH_MAXNREG_DENSITY 64
#endif
#ifndef SPH_MAXNREG_FORCES
#define SPH_MAXNREG_FORCES 56
#endif
#ifndef SPH_MAXNREG_XSPH
#define SPH_MAXNREG_XSPH 56
#endif

enum : uint32_t { kFlagDelta = 1, kFlagXsph = 2, kFlagRepulsion = 4, kFlagClamp = 8 };
enum : uint32_t { kErrCellCap = 1, kErrAdamiCap = 2 };

// Step constants, each rounded in f32 exactly as the reference evaluates it.
struct SimConst {
  float h, support, radius_sq, cell;
  float inv_h;       // RN(1 / h)
  float gmin[3];
  int dims[3];
  float norm_h3;     // NORM / (h*h*h)        (sph.rs:45)
  float norm_h4;     // NORM / ((h*h*h)*h)    (sph.rs:80)
  float eta_sq;      // 0.01*h*h              (sph.rs:177, 442)
  float delta_coef;  // DELTA_SPH*h*c         (sph.rs:212)
  float neg_alpha_c; // -alpha*c              (sph.rs:472)
  float beta;
  float grav[3];
  float dmin[3], dmax[3];
  float b_water, b_air;  // rho0*c*c/gamma    (eos.rs:40)
  float r0, rep_d;       // 0.5h, 10*9.81*0.01 (boundary.rs:150-154)
  float c;
  float reach;           // Adami candidate reach, > 2h with margin
  float sdf_coef;
  uint32_t flags;
  // sqrtf is monotone: sqrtf(d2) < support  <=>  d2 <= sup_d2,
  // sqrtf(d2) < r0 <=> d2 <= r0_d2, sqrtf(d2) > 1e-12 <=> d2 > tiny_d2.
  float sup_d2, r0_d2, tiny_d2;
  // SDF wall mode (boundary_mode 1): node grid geometry
  int sdf_mode;
  float wall_inv_step;   // kWallN / 2h
  // wall particle mass / (rho0 (h / 1.3)^3): the homogenised wall layers
  // carry the fluid's particle mass; exactly 1 for mass rho0 dx^3
  float wall_scale;
  float wall_inv2, wall_inv3;  // kWallN2 / 2h, kWallN3 / 2h: edge and corner tables
  int has_geo;                 // SDF mode: an obstacle SDF is present
  float sdf_origin[3];
  float sdf_cell;
  int sdf_dims[3];
  // batch: this instance's index (dt and dt-maxima slots) and the offset of
  // its cells in the global cell tables (0 for a single simulation)
  int inst;
  int coff;
  int rows;  // the cells of an x-row are consecutive in the particle order
  float cfl;
  // geometry SDF for the closure features (boundary-particle mode) or the
  // SDF walls, at sdf_off in the device SDF array
  int feat_sdf;
  long long sdf_off;
};

// Constants provider of a single simulation: the constants ride in the
// kernel parameter space.
struct OneSim {
  SimConst k;
  __device__ __forceinline__ const SimConst& at(int) const { return k; }
};

// Constants provider of a batch: per-instance constants, and the instance
// of every slot (particles of an instance occupy a fixed slot range).
struct ManySim {
  const SimConst* __restrict__ tab;
  const uint16_t* __restrict__ inst;
  __device__ __forceinline__ const SimConst& at(int i) const { return tab[__ldg(&inst[i])]; }
};

// ---------------------------------------------------------------------------
// exact per-op helpers
// ---------------------------------------------------------------------------

// neighbor.rs:57-71
__device__ __forceinline__ int axis_cell(float p, float gmin, float cell, int dim) {
  float f = floorf((p - gmin) / cell);
  f = fmaxf(f, 0.0f);
  f = fminf(f, (float)(dim - 1));
  return (int)f;
}

__device__ __forceinline__ int cell_hash(int cx, int cy, int cz, const SimConst& k) {
  return cx + cy * k.dims[0] + cz * k.dims[0] * k.dims[1];
}

// r / h correctly rounded, from inv_h = RN(1/h) and two FMA residual
// corrections (Markstein's division by the fused multiply-add; Muller et al.,
// Handbook of Floating-Point Arithmetic, "Division using the FMA"): q1 =
// RN(q0 + RN(r - h q0) inv_h) is within an ulp of r / h, so its residual
// r - h q1 is exact and RN(q1 + (r - h q1) inv_h) is the correctly rounded
// quotient. That holds while the residuals do not underflow, i.e. for every
// r above 2^-100 or so (checked exhaustively against IEEE division for the
// smoothing lengths the tests use); the Wendland kernel and its gradient do
// not depend on q's low bits below r = 2^-36 (q < 2^-26 rounds out of
// 1 - q/2 and 1 + 2q, and the gradient is zero below r = 1e-12).
__device__ __forceinline__ float div_h(float r, const SimConst& k) {
  const float q0 = __fmul_rn(r, k.inv_h);
  const float q1 = __fmaf_rn(__fmaf_rn(-q0, k.h, r), k.inv_h, q0);
  return __fmaf_rn(__fmaf_rn(-q1, k.h, r), k.inv_h, q1);
}

// sph.rs:35-46 with NORM/h^3 precomputed (same rounding).
__device__ __forceinline__ float w_c2(float r, const SimConst& k) {
  float q = div_h(r, k);
  if (q >= 2.0f) return 0.0f;
  float omq = 1.0f - 0.5f * q;
  float t = omq * omq;
  float t4 = t * t;
  return k.norm_h3 * t4 * (1.0f + 2.0f * q);
}

// sph.rs:68-85
__device__ __forceinline__ void grad_c2(float dx, float dy, float dz, float r, const SimConst& k,
                                        float& gx, float& gy, float& gz) {
  float q = div_h(r, k);
  if (q >= 2.0f || r < 1.0e-12f) {
    gx = 0.0f; gy = 0.0f; gz = 0.0f;
    return;
  }
  float omq = 1.0f - 0.5f * q;
  float t3 = omq * omq * omq;
  float dw_dr = k.norm_h4 * (-5.0f * q) * t3;
  float inv_r = 1.0f / r;
  gx = dw_dr * dx * inv_r;
  gy = dw_dr * dy * inv_r;
  gz = dw_dr * dz * inv_r;
}

// Correctly rounded x^7: the double product carries < 4 ulp(double) of error,
// far inside half an f32 ulp (checked exhaustively on [0.5, 2]).
__device__ __forceinline__ float pow7_cr(float x) {
  double r = x, r2 = r * r, r4 = r2 * r2, r6 = r4 * r2;
  return (float)(r6 * r);
}

// eos.rs:39-47 (Water gamma 7, Air gamma 1.4)
__device__ __forceinline__ float tait(float rho, bool air, const SimConst& k) {
  float rest = air ? kAirRho0 : kWaterRho0;
  float b = air ? k.b_air : k.b_water;
  float ratio = rho / rest;
  float pw = air ? (float)pow((double)ratio, (double)1.4f) : pow7_cr(ratio);
  float p = b * (pw - 1.0f);
  return fmaxf(p, 0.0f);
}

// ---- SDF wall (boundary_mode 1; no reference counterpart) -----------------
// The walls stand in for the reference's 3 layers of wall particles on every
// face of the domain box (domain.rs:162-348) plus those of an obstacle given
// by its SDF, homogenised along each wall. wall_tab holds lattice sums built
// on the host (phi = sum W dx^3, grad = sum (-dW/dr)(z_a / r) dx^3 along the
// first argument's normal a):
//   [0, kWallN]           one 3-layer slab at distance d (lateral average),
//   kWallOff2 + ...       the edge column where two slabs meet, at (d_a, d_b)
//                         (average along the edge),
//   kWallOff3 + ...       the corner cube of three slabs, at (d_a, d_b, d_c),
// on [0, 2h] per argument, interpolated (bi-, tri-)linearly in f32. The box
// walls are the union of the face slabs: singles - edges + corner.
constexpr int kWallN = 512;
constexpr int kWallN2 = 64;
constexpr int kWallN3 = 24;
constexpr int kWallOff2 = kWallN + 1;
constexpr int kWallOff3 = kWallOff2 + (kWallN2 + 1) * (kWallN2 + 1);
constexpr int kWallTabSize = kWallOff3 + (kWallN3 + 1) * (kWallN3 + 1) * (kWallN3 + 1);
__device__ __forceinline__ float2 wall_lookup(const float2* __restrict__ tab, float inv_step, float d) {
  float u = fmaxf(d, 0.0f) * inv_step;
  if (!(u < (float)kWallN)) return make_float2(0.0f, 0.0f);
  int i = (int)u;
  float f = u - (float)i;
  float2 a = __ldg(&tab[i]), b = __ldg(&tab[i + 1]);
  return make_float2(a.x + f * (b.x - a.x), a.y + f * (b.y - a.y));
}

__device__ __forceinline__ float2 wall_lookup2(const float2* __restrict__ tab, float inv, float da, float db) {
  float u = fmaxf(da, 0.0f) * inv, v = fmaxf(db, 0.0f) * inv;
  if (!(u < (float)kWallN2) || !(v < (float)kWallN2)) return make_float2(0.0f, 0.0f);
  int i = (int)u, j = (int)v;
  float fu = u - (float)i, fv = v - (float)j;
  const float2* t = tab + kWallOff2 + i * (kWallN2 + 1) + j;
  float2 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + kWallN2 + 1), d = __ldg(t + kWallN2 + 2);
  float x0 = a.x + fv * (b.x - a.x), x1 = c.x + fv * (d.x - c.x);
  float y0 = a.y + fv * (b.y - a.y), y1 = c.y + fv * (d.y - c.y);
  return make_float2(x0 + fu * (x1 - x0), y0 + fu * (y1 - y0));
}

__device__ __forceinline__ float2 wall_lookup3(const float2* __restrict__ tab, float inv, float da, float db,
                                               float dc) {
  float u = fmaxf(da, 0.0f) * inv, v = fmaxf(db, 0.0f) * inv, w = fmaxf(dc, 0.0f) * inv;
  if (!(u < (float)kWallN3) || !(v < (float)kWallN3) || !(w < (float)kWallN3)) return make_float2(0.0f, 0.0f);
  int i = (int)u, j = (int)v, l = (int)w;
  float fu = u - (float)i, fv = v - (float)j, fw = w - (float)l;
  const int S = kWallN3 + 1;
  const float2* t = tab + kWallOff3 + (i * S + j) * S + l;
  float2 c000 = __ldg(t), c001 = __ldg(t + 1), c010 = __ldg(t + S), c011 = __ldg(t + S + 1);
  float2 c100 = __ldg(t + S * S), c101 = __ldg(t + S * S + 1), c110 = __ldg(t + S * S + S),
         c111 = __ldg(t + S * S + S + 1);
  float x00 = c000.x + fw * (c001.x - c000.x), x01 = c010.x + fw * (c011.x - c010.x);
  float x10 = c100.x + fw * (c101.x - c100.x), x11 = c110.x + fw * (c111.x - c110.x);
  float y00 = c000.y + fw * (c001.y - c000.y), y01 = c010.y + fw * (c011.y - c010.y);
  float y10 = c100.y + fw * (c101.y - c100.y), y11 = c110.y + fw * (c111.y - c110.y);
  float x0 = x00 + fv * (x01 - x00), x1 = x10 + fv * (x11 - x10);
  float y0 = y00 + fv * (y01 - y00), y1 = y10 + fv * (y11 - y10);
  return make_float2(x0 + fu * (x1 - x0), y0 + fu * (y1 - y0));
}

// The nearer face of the domain box on each axis: distance, inward normal
// sign (+1 at the lower face, -1 at the upper) and whether it is within 2h.
// Domains narrower than 4h, where both faces of an axis could be, are not
// supported by the SDF wall mode.
struct BoxFaces {
  float d[3], s[3];
  bool on[3];
};
__device__ __forceinline__ BoxFaces box_faces(const SimConst& k, float px, float py, float pz) {
  BoxFaces b;
  float p[3] = {px, py, pz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float dl = p[a] - k.dmin[a], dh = k.dmax[a] - p[a];
    if (dl <= dh) {
      b.d[a] = dl;
      b.s[a] = 1.0f;
    } else {
      b.d[a] = dh;
      b.s[a] = -1.0f;
    }
    b.on[a] = b.d[a] < k.support;
  }
  return b;
}

// Kernel mass of the SDF-mode walls at a particle, in units of the wall
// particle mass density: box faces (singles - edges + corner), then the
// obstacle at SDF distance dgeo.
__device__ __forceinline__ float sdf_wall_mass(const SimConst& k, const float2* __restrict__ tab,
                                               const BoxFaces& b, float dgeo) {
  float m = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (b.on[a]) m += wall_lookup(tab, k.wall_inv_step, b.d[a]).x;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = a + 1; c < 3; ++c)
      if (b.on[a] && b.on[c]) m -= wall_lookup2(tab, k.wall_inv2, b.d[a], b.d[c]).x;
  if (b.on[0] && b.on[1] && b.on[2]) m += wall_lookup3(tab, k.wall_inv3, b.d[0], b.d[1], b.d[2]).x;
  if (k.has_geo && dgeo < k.support) m += wall_lookup(tab, k.wall_inv_step, dgeo).x;
  return m;
}

// GridSDF::sample (orchestrator geometry.rs:99-150) with the grid coordinate
// clamped to [0, dims-1-1e-3]: points on or past the outer nodes interpolate
// in the last cell instead of returning f32::MAX.
__device__ __forceinline__ float sdf_sample_clamped(const float* __restrict__ d, const SimConst& k,
                                                    float px, float py, float pz) {
  float g[3] = {(px - k.sdf_origin[0]) / k.sdf_cell, (py - k.sdf_origin[1]) / k.sdf_cell,
                (pz - k.sdf_origin[2]) / k.sdf_cell};
  int i0[3];
  float fr[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] = fminf(fmaxf(g[a], 0.0f), (float)(k.sdf_dims[a] - 1) - 0.001f);
    i0[a] = (int)floorf(g[a]);
    fr[a] = g[a] - (float)i0[a];
  }
  size_t ny = (size_t)k.sdf_dims[1], nz = (size_t)k.sdf_dims[2];
  size_t base = (size_t)k.sdf_off + (size_t)i0[0] * ny * nz + (size_t)i0[1] * nz + (size_t)i0[2];
  size_t si = ny * nz, sj = nz;
  float c000 = __ldg(&d[base]), c001 = __ldg(&d[base + 1]);
  float c010 = __ldg(&d[base + sj]), c011 = __ldg(&d[base + sj + 1]);
  float c100 = __ldg(&d[base + si]), c101 = __ldg(&d[base + si + 1]);
  float c110 = __ldg(&d[base + si + sj]), c111 = __ldg(&d[base + si + sj + 1]);
  float fx = fr[0], fy = fr[1], fz = fr[2];
  float c00 = c000 * (1.0f - fz) + c001 * fz;
  float c01 = c010 * (1.0f - fz) + c011 * fz;
  float c10 = c100 * (1.0f - fz) + c101 * fz;
  float c11 = c110 * (1.0f - fz) + c111 * fz;
  float c0 = c00 * (1.0f - fy) + c01 * fy;
  float c1 = c10 * (1.0f - fy) + c11 * fy;
  return c0 * (1.0f - fx) + c1 * fx;
}

// GridSDF::gradient (geometry.rs:153-175) on the clamped sampler.
__device__ __forceinline__ void sdf_gradient_clamped(const float* __restrict__ d, const SimConst& k,
                                                     float px, float py, float pz, float& nx,
                                                     float& ny, float& nz) {
  float h = k.sdf_cell * 0.5f;
  float gx = (sdf_sample_clamped(d, k, px + h, py, pz) - sdf_sample_clamped(d, k, px - h, py, pz)) / (2.0f * h);
  float gy = (sdf_sample_clamped(d, k, px, py + h, pz) - sdf_sample_clamped(d, k, px, py - h, pz)) / (2.0f * h);
  float gz = (sdf_sample_clamped(d, k, px, py, pz + h) - sdf_sample_clamped(d, k, px, py, pz - h)) / (2.0f * h);
  float mag = sqrtf(gx * gx + gy * gy + gz * gz);
  if (mag > 1e-8f) { nx = gx / mag; ny = gy / mag; nz = gz / mag; }
  else { nx = 0.0f; ny = 0.0f; nz = 0.0f; }
}

// Distance to the nearest wall of the SDF mode (a box face or the obstacle)
// and its inward normal: the closure features' SDF in that mode.
__device__ __forceinline__ float wall_distance(const SimConst& k, const float* __restrict__ sdf, float px,
                                               float py, float pz) {
  BoxFaces b = box_faces(k, px, py, pz);
  float d = fminf(fminf(b.d[0], b.d[1]), b.d[2]);
  if (k.has_geo) d = fminf(d, sdf_sample_clamped(sdf, k, px, py, pz));
  return d;
}
__device__ __forceinline__ void wall_normal(const SimConst& k, const float* __restrict__ sdf, float px,
                                            float py, float pz, float& nx, float& ny, float& nz) {
  BoxFaces b = box_faces(k, px, py, pz);
  int a = b.d[0] <= b.d[1] ? (b.d[0] <= b.d[2] ? 0 : 2) : (b.d[1] <= b.d[2] ? 1 : 2);
  if (k.has_geo && sdf_sample_clamped(sdf, k, px, py, pz) < b.d[a]) {
    sdf_gradient_clamped(sdf, k, px, py, pz, nx, ny, nz);
    return;
  }
  nx = a == 0 ? b.s[0] : 0.0f;
  ny = a == 1 ? b.s[1] : 0.0f;
  nz = a == 2 ? b.s[2] : 0.0f;
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__device__ __forceinline__ uint32_t morton30(uint32_t cx, uint32_t cy, uint32_t cz) {
  return spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
}

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  // v >= 0 and not NaN: the IEEE bit pattern orders like an unsigned int.
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

// Visit the reference's 27-cell neighbourhood of (px,py,pz) on the cell table
// `ctab` (per linear cell: storage start, count), skipping slot `self`, and
// call f(slot, pj, dx, dy, dz, dist_sq) for every candidate with
// dist_sq <= (2h)^2.
template <class F>
__device__ __forceinline__ void for_each_neighbor(float px, float py, float pz, int self,
                                                  const float4* __restrict__ pos,
                                                  const uint2* __restrict__ ctab,
                                                  const SimConst& k, F&& f) {
  int cx = axis_cell(px, k.gmin[0], k.cell, k.dims[0]);
  int cy = axis_cell(py, k.gmin[1], k.cell, k.dims[1]);
  int cz = axis_cell(pz, k.gmin[2], k.cell, k.dims[2]);
  // Squared distance to the lower / upper face of the home cell per axis,
  // shrunk by a margin far above any rounding of the binning: a cell whose
  // box lies farther than 2h holds no particle with dist_sq <= (2h)^2, so
  // skipping it changes no sum.
  const float margin = 1.0e-5f * k.cell + 1.0e-6f;
  float lo2[3], hi2[3];
  {
    float p3[3] = {px, py, pz};
    int c3[3] = {cx, cy, cz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float face = k.gmin[a] + (float)c3[a] * k.cell;
      float dl = fmaxf(p3[a] - face - margin, 0.0f);
      float dh = fmaxf(face + k.cell - p3[a] - margin, 0.0f);
      lo2[a] = dl * dl;
      hi2[a] = dh * dh;
    }
  }
  for (int dz = -1; dz <= 1; ++dz) {
    int nz = cz + dz;
    if (nz < 0 || nz >= k.dims[2]) continue;
    float ez = dz < 0 ? lo2[2] : (dz > 0 ? hi2[2] : 0.0f);
    for (int dy = -1; dy <= 1; ++dy) {
      int ny = cy + dy;
      if (ny < 0 || ny >= k.dims[1]) continue;
      float ey = ez + (dy < 0 ? lo2[1] : (dy > 0 ? hi2[1] : 0.0f));
      if (ey > k.radius_sq) continue;
      int row = (ny + nz * k.dims[1]) * k.dims[0];
      for (int dx = -1; dx <= 1; ++dx) {
        int nx = cx + dx;
        if (nx < 0 || nx >= k.dims[0]) continue;
        if (ey + (dx < 0 ? lo2[0] : (dx > 0 ? hi2[0] : 0.0f)) > k.radius_sq) continue;
        uint2 se = __ldg(&ctab[k.coff + row + nx]);
        int end = (int)(se.x + se.y);
        int s = (int)se.x;
        auto test = [&](int t, const float4& pj) {
          if (t == self) return;
          float ddx = px - pj.x, ddy = py - pj.y, ddz = pz - pj.z;
          float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (d2 <= k.radius_sq) f(t, pj, ddx, ddy, ddz, d2);
        };
        // four candidate loads in flight before the (in-order) tests
        for (; s + 3 < end; s += 4) {
          float4 q0 = __ldg(&pos[s]), q1 = __ldg(&pos[s + 1]), q2 = __ldg(&pos[s + 2]), q3 = __ldg(&pos[s + 3]);
          test(s, q0);
          test(s + 1, q1);
          test(s + 2, q2);
          test(s + 3, q3);
        }
        for (; s < end; ++s) test(s, __ldg(&pos[s]));
      }
    }
  }
}

// Packed f32x2 arithmetic (sm_100): two IEEE f32 operations per instruction,
// each rounded exactly as its scalar form (explicit .rn, never contracted).
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// ((px - x)^2 + (py - y)^2) + (pz - z)^2 of two candidates at once, rounded
// as the reference's scalar expression.
__device__ __forceinline__ void dist2_pair(unsigned long long X, unsigned long long Y, unsigned long long Z,
                                           const float4& a, const float4& b, float& da, float& db) {
  unsigned long long dx = f2_sub(X, f2_pack(a.x, b.x));
  unsigned long long dy = f2_sub(Y, f2_pack(a.y, b.y));
  unsigned long long dz = f2_sub(Z, f2_pack(a.z, b.z));
  f2_unpack(f2_add(f2_add(f2_mul(dx, dx), f2_mul(dy, dy)), f2_mul(dz, dz)), da, db);
}

// Positions in the sorted order as three planes (x, y, z) of `stride` floats
// each, stride a multiple of 4 with zero padding past the last slot, so that
// four consecutive candidates' coordinates are one aligned 16-byte load and
// come packed for the f32x2 arithmetic. Written by k_reorder and k_restore
// beside the float4 state.
struct Planes {
  float* __restrict__ xyz;
  size_t stride;
};

// Neighbour lists are entry-major: entry c of slot i at nbr[c n + i]. The
// warp-cooperative scan below emits one entry per lane per step, so the
// lanes' stores of one step fill whole lines, and the replays read entry c of
// 32 consecutive slots with one coalesced load.
__device__ __forceinline__ size_t nbr_index(uint32_t c, int n, int i) {
  return (size_t)c * (size_t)n + (size_t)i;
}

// The per-thread form of the density pass's scan over the SoA planes, for a
// cell whose 27-cell neighbourhood holds more candidates than the warp scan's
// masks cover: the candidates of a range are taken in aligned groups of four
// (lanes outside [s, e) masked), each group's distances in two f32x2 pairs
// rounded exactly as the scalar expression, and the in-support slots stored
// in visit order (at most kNbrCap; the count is returned in full). The cells,
// rows and order visited are for_each_neighbor's.
// The grid constants record_neighbors reads (passed by value: a reference to
// a single simulation's constants would move them from the parameter space
// to the stack of every thread).
struct ScanGeo {
  float gmin[3];
  float cell, radius_sq;
  int dims[3];
  int coff, rows;
  __device__ __forceinline__ explicit ScanGeo(const SimConst& k)
      : gmin{k.gmin[0], k.gmin[1], k.gmin[2]}, cell(k.cell), radius_sq(k.radius_sq),
        dims{k.dims[0], k.dims[1], k.dims[2]}, coff(k.coff), rows(k.rows) {}
};
__device__ __noinline__ uint32_t record_neighbors(float px, float py, float pz, int self, Planes pl,
                                                  const uint2* __restrict__ ctab, const ScanGeo k,
                                                  uint32_t* __restrict__ nbr, int n) {
  int cx = axis_cell(px, k.gmin[0], k.cell, k.dims[0]);
  int cy = axis_cell(py, k.gmin[1], k.cell, k.dims[1]);
  int cz = axis_cell(pz, k.gmin[2], k.cell, k.dims[2]);
  const float margin = 1.0e-5f * k.cell + 1.0e-6f;  // as for_each_neighbor
  float lo2[3], hi2[3];
  {
    float p3[3] = {px, py, pz};
    int c3[3] = {cx, cy, cz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float face = k.gmin[a] + (float)c3[a] * k.cell;
      float dl = fmaxf(p3[a] - face - margin, 0.0f);
      float dh = fmaxf(face + k.cell - p3[a] - margin, 0.0f);
      lo2[a] = dl * dl;
      hi2[a] = dh * dh;
    }
  }
  const float* xs = pl.xyz;
  const float* ys = pl.xyz + pl.stride;
  const float* zs = pl.xyz + 2 * pl.stride;
  const unsigned long long X = f2_pack(px, px), Y = f2_pack(py, py), Z = f2_pack(pz, pz);
  const float r2 = k.radius_sq;
  uint32_t listed = 0;
  auto put = [&](bool ok, int slot) {
    if (ok) {
      if (listed < kNbrCap) nbr[nbr_index(listed, n, self)] = (uint32_t)slot;
      ++listed;
    }
  };
  auto range = [&](int s, int e) {
    for (int g = s & ~3; g < e; g += 4) {
      float4 qx = __ldg(reinterpret_cast<const float4*>(xs + g));
      float4 qy = __ldg(reinterpret_cast<const float4*>(ys + g));
      float4 qz = __ldg(reinterpret_cast<const float4*>(zs + g));
      unsigned long long dx01 = f2_sub(X, f2_pack(qx.x, qx.y)), dx23 = f2_sub(X, f2_pack(qx.z, qx.w));
      unsigned long long dy01 = f2_sub(Y, f2_pack(qy.x, qy.y)), dy23 = f2_sub(Y, f2_pack(qy.z, qy.w));
      unsigned long long dz01 = f2_sub(Z, f2_pack(qz.x, qz.y)), dz23 = f2_sub(Z, f2_pack(qz.z, qz.w));
      float d0, d1, d2, d3;
      f2_unpack(f2_add(f2_add(f2_mul(dx01, dx01), f2_mul(dy01, dy01)), f2_mul(dz01, dz01)), d0, d1);
      f2_unpack(f2_add(f2_add(f2_mul(dx23, dx23), f2_mul(dy23, dy23)), f2_mul(dz23, dz23)), d2, d3);
      const int lo = s - g, hi = e - g;
      put(d0 <= r2 && 0 >= lo && 0 < hi, g);
      put(d1 <= r2 && 1 >= lo && 1 < hi, g + 1);
      put(d2 <= r2 && 2 >= lo && 2 < hi, g + 2);
      put(d3 <= r2 && 3 >= lo && 3 < hi, g + 3);
    }
  };
  for (int dz = -1; dz <= 1; ++dz) {
    int nz = cz + dz;
    if (nz < 0 || nz >= k.dims[2]) continue;
    float ez = dz < 0 ? lo2[2] : (dz > 0 ? hi2[2] : 0.0f);
    for (int dy = -1; dy <= 1; ++dy) {
      int ny = cy + dy;
      if (ny < 0 || ny >= k.dims[1]) continue;
      float ey = ez + (dy < 0 ? lo2[1] : (dy > 0 ? hi2[1] : 0.0f));
      if (ey > r2) continue;
      int row = k.coff + (ny + nz * k.dims[1]) * k.dims[0];
      if (k.rows) {
        int xa = (cx > 0 && ey + lo2[0] <= r2) ? cx - 1 : cx;
        int xb = (cx + 1 < k.dims[0] && ey + hi2[0] <= r2) ? cx + 1 : cx;
        uint2 sa = __ldg(&ctab[row + xa]), sb = __ldg(&ctab[row + xb]);
        if (ny == cy && nz == cz) {  // the home row holds `self`: skip it by splitting the range
          range((int)sa.x, self);
          range(self + 1, (int)(sb.x + sb.y));
        } else {
          range((int)sa.x, (int)(sb.x + sb.y));
        }
      } else {
        for (int dx = -1; dx <= 1; ++dx) {
          int nx = cx + dx;
          if (nx < 0 || nx >= k.dims[0]) continue;
          if (ey + (dx < 0 ? lo2[0] : (dx > 0 ? hi2[0] : 0.0f)) > r2) continue;
          uint2 se = __ldg(&ctab[row + nx]);
          if (dx == 0 && ny == cy && nz == cz) {
            range((int)se.x, self);
            range(self + 1, (int)(se.x + se.y));
          } else {
            range((int)se.x, (int)(se.x + se.y));
          }
        }
      }
    }
  }
  return listed;
}

// Warp-cooperative neighbour scan of the density pass. The particles of one
// cell share one candidate sequence: its 27-cell neighbourhood as 9 x-row
// ranges (row cell order, where a row's cells are consecutive) or 27 cell
// ranges, concatenated in the reference's visit order (dz, dy, dx, then slot,
// i.e. ascending id within a cell). A warp takes its 32 slots cell by cell (a
// "segment" is the run of its slots in one cell): the lanes load 32
// consecutive candidates of the sequence at once, and for four of the
// segment's particles at a time every lane computes its candidate's squared
// distance to each (two f32x2 chains, rounded as the scalar expression); a
// ballot per particle gives that particle's 32-bit in-support mask for the
// word, and one lane stores the quad's four masks with one 16-byte store
// (per segment the masks lie word-major: word w of the segment's particle p
// at mask[base + w q + p], q its particle count rounded up to a quad). Each
// lane then turns its particle's masks, its own slot cleared, into its list,
// one entry per step, so that every active lane stores entry c at the same
// step (entry-major: the stores of a step coalesce). The list and its order
// equal for_each_neighbor's: a candidate outside support sets no bit, and the
// sequence visits the neighbourhood's cells in the reference's order.
constexpr int kScanWords = 24;   // mask words per particle: up to 768 candidates per neighbourhood
constexpr int kScanSegs = 4;     // segments whose masks are held at once
constexpr int kScanRanges = 27;  // candidate ranges per segment (9 in row order)
// masks of one batch: at most kScanWords words per quad-padded particle, and
// the batch's segments hold 32 particles plus at most 3 pads each
constexpr int kMaskWords = kScanWords * (32 + 3 * kScanSegs);
struct __align__(16) ScanWarp {
  float px[36], py[36], pz[36];                  // the segment's particles, padded to quads with NaN
  uint32_t mask[kMaskWords];                     // per segment [word][particle]
  uint32_t vstart[kScanSegs][kScanRanges + 1];   // sequence index of each range's first candidate; [R] = total
  uint32_t sstart[kScanSegs][kScanRanges];       // slot of each range's first candidate
  uint32_t mbase[kScanSegs], mquad[kScanSegs];   // each segment's mask base and particle stride
};
static_assert(sizeof(ScanWarp) % 16 == 0, "per-warp scratch keeps 16-byte alignment");
static_assert(offsetof(ScanWarp, py) % 16 == 0 && offsetof(ScanWarp, pz) % 16 == 0, "quad loads");

// Returns this lane's neighbour count (entries stored up to kNbrCap). Every
// lane of the warp calls it, `live` or not. A lane whose list comes from its
// masks also hands every neighbour, in list order, to two(s0, s1) (two at a
// time, their gathers in flight together) or one(s) (the last of an odd
// count), and sets `fed`; a lane of a neighbourhood too large for the masks
// takes the per-thread scan, and its caller replays the list.
template <class KP, class Two, class One>
__device__ __forceinline__ uint32_t scan_warp(const KP& kp, int i, bool live, Planes pl,
                                              const uint2* __restrict__ ctab, ScanWarp& S,
                                              uint32_t* __restrict__ nbr, int n, Two&& two, One&& one,
                                              bool& fed) {
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const float* xs = pl.xyz;
  const float* ys = xs + pl.stride;
  const float* zs = ys + pl.stride;
  const float nan = __int_as_float(0x7fc00000);
  float qx = 0.0f, qy = 0.0f, qz = 0.0f;
  int cx = 0, cy = 0, cz = 0;
  uint32_t key = 0xffffffffu;
  if (live) {
    const SimConst& k = kp.at(i);
    qx = xs[i];
    qy = ys[i];
    qz = zs[i];
    cx = axis_cell(qx, k.gmin[0], k.cell, k.dims[0]);
    cy = axis_cell(qy, k.gmin[1], k.cell, k.dims[1]);
    cz = axis_cell(qz, k.gmin[2], k.cell, k.dims[2]);
    key = (uint32_t)(k.coff + cell_hash(cx, cy, cz, k));  // global cell: instances never share one
  }
  const uint32_t prev = __shfl_up_sync(kAll, key, 1);
  const uint32_t heads = __ballot_sync(kAll, live && (lane == 0 || prev != key));
  const uint32_t livemask = __ballot_sync(kAll, live);  // a prefix of the lanes
  const int myhead = live ? 31 - __clz(heads & (lane == 31 ? kAll : (2u << lane) - 1u)) : 0;
  uint32_t listed = 0;
  uint32_t rem = heads;
  while (rem) {
    uint32_t batch = 0, t = rem;  // the next kScanSegs segments
    for (int q = 0; q < kScanSegs && t; ++q) {
      batch |= t & (0u - t);
      t &= t - 1u;
    }
    rem = t;
    __syncwarp();
    int seg = 0;
    uint32_t mbase = 0;  // the next segment's mask base (a multiple of 4 words)
    for (uint32_t bb = batch; bb; bb &= bb - 1u, ++seg) {
      const int hl = __ffs(bb) - 1;
      const uint32_t after = heads & ~(hl == 31 ? kAll : (2u << hl) - 1u);
      const int he = after ? __ffs(after) - 1 : 32 - __clz(livemask);
      const int m = he - hl;
      const int scx = __shfl_sync(kAll, cx, hl), scy = __shfl_sync(kAll, cy, hl), scz = __shfl_sync(kAll, cz, hl);
      const SimConst& k = kp.at(__shfl_sync(kAll, i, hl));
      const int R = k.rows ? 9 : 27;
      uint32_t len = 0, st = 0;
      if (lane < R) {  // lane r: range r of the sequence
        const int dz = k.rows ? lane / 3 - 1 : lane / 9 - 1;
        const int dy = k.rows ? lane % 3 - 1 : (lane / 3) % 3 - 1;
        const int nz = scz + dz, ny = scy + dy;
        if (nz >= 0 && nz < k.dims[2] && ny >= 0 && ny < k.dims[1]) {
          const int row = k.coff + (ny + nz * k.dims[1]) * k.dims[0];
          if (k.rows) {
            const int xa = scx > 0 ? scx - 1 : scx, xb = scx + 1 < k.dims[0] ? scx + 1 : scx;
            const uint2 sa = __ldg(&ctab[row + xa]), sb = __ldg(&ctab[row + xb]);
            st = sa.x;
            len = sb.x + sb.y - sa.x;
          } else {
            const int nx = scx + lane % 3 - 1;
            if (nx >= 0 && nx < k.dims[0]) {
              const uint2 se = __ldg(&ctab[row + nx]);
              st = se.x;
              len = se.y;
            }
          }
        }
      }
      uint32_t incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t total = __shfl_sync(kAll, incl, 31);
      if (lane < R) {
        S.vstart[seg][lane] = incl - len;
        S.sstart[seg][lane] = st;
      }
      if (lane == 0) S.vstart[seg][R] = total;
      const bool in_seg = lane >= hl && lane < he;
      if (in_seg) {
        S.px[lane - hl] = qx;
        S.py[lane - hl] = qy;
        S.pz[lane - hl] = qz;
      }
      if (lane >= m && lane < ((m + 3) & ~3)) {
        S.px[lane] = nan;
        S.py[lane] = nan;
        S.pz[lane] = nan;
      }
      const int nw = (int)((total + 31u) / 32u);
      const int q4 = (m + 3) & ~3;
      if (lane == 0) {
        S.mbase[seg] = mbase;
        S.mquad[seg] = (uint32_t)q4;
      }
      __syncwarp();
      if (nw <= kScanWords) {
        const float r2 = k.radius_sq;
        uint32_t* const mw = S.mask + mbase;
        int r = 0;
        float nxv = nan, nyv = nan, nzv = nan;
        auto fetch = [&](int w) {  // candidate 32 w + lane (NaN past the end: in no particle's support)
          const uint32_t v = (uint32_t)(w * 32 + lane);
          nxv = nan;
          nyv = nan;
          nzv = nan;
          if (v < total) {
            while (v >= S.vstart[seg][r + 1]) ++r;
            const uint32_t slot = S.sstart[seg][r] + (v - S.vstart[seg][r]);
            nxv = __ldg(&xs[slot]);
            nyv = __ldg(&ys[slot]);
            nzv = __ldg(&zs[slot]);
          }
        };
        fetch(0);
        for (int w = 0; w < nw; ++w) {
          const unsigned long long CX = f2_pack(nxv, nxv), CY = f2_pack(nyv, nyv), CZ = f2_pack(nzv, nzv);
          if (w + 1 < nw) fetch(w + 1);  // next word's candidates in flight
          uint32_t* const row = mw + w * q4;
          for (int p = 0; p < m; p += 4) {
            const float4 ax = *reinterpret_cast<const float4*>(&S.px[p]);
            const float4 ay = *reinterpret_cast<const float4*>(&S.py[p]);
            const float4 az = *reinterpret_cast<const float4*>(&S.pz[p]);
            const unsigned long long dx0 = f2_sub(f2_pack(ax.x, ax.y), CX), dx1 = f2_sub(f2_pack(ax.z, ax.w), CX);
            const unsigned long long dy0 = f2_sub(f2_pack(ay.x, ay.y), CY), dy1 = f2_sub(f2_pack(ay.z, ay.w), CY);
            const unsigned long long dz0 = f2_sub(f2_pack(az.x, az.y), CZ), dz1 = f2_sub(f2_pack(az.z, az.w), CZ);
            float d0, d1, d2, d3;
            f2_unpack(f2_add(f2_add(f2_mul(dx0, dx0), f2_mul(dy0, dy0)), f2_mul(dz0, dz0)), d0, d1);
            f2_unpack(f2_add(f2_add(f2_mul(dx1, dx1), f2_mul(dy1, dy1)), f2_mul(dz1, dz1)), d2, d3);
            const uint32_t M0 = __ballot_sync(kAll, d0 <= r2), M1 = __ballot_sync(kAll, d1 <= r2);
            const uint32_t M2 = __ballot_sync(kAll, d2 <= r2), M3 = __ballot_sync(kAll, d3 <= r2);
            if (lane == 0) *reinterpret_cast<uint4*>(row + p) = make_uint4(M0, M1, M2, M3);
          }
        }
        mbase += (uint32_t)(nw * q4);
      }
      __syncwarp();
    }
    // the batch's lanes turn their masks into their lists
    if (live && ((batch >> myhead) & 1u)) {
      const SimConst& k = kp.at(i);
      const int R = k.rows ? 9 : 27;
      const int s = __popc(batch & ((1u << myhead) - 1u));
      const uint32_t total = S.vstart[s][R];
      const int nw = (int)((total + 31u) / 32u);
      if (nw > kScanWords) {
        listed = record_neighbors(qx, qy, qz, i, pl, ctab, ScanGeo(k), nbr, n);
      } else {
        fed = true;
        const uint32_t q4 = S.mquad[s];
        const uint32_t* words = S.mask + S.mbase[s] + (lane - myhead);  // word w at words[w q4]
        // this lane's own slot in the sequence (its home range is range R/2), cleared from its masks
        const uint32_t vself = S.vstart[s][R / 2] + ((uint32_t)i - S.sstart[s][R / 2]);
        const int wself = (int)(vself >> 5);
        const uint32_t bself = ~(1u << (vself & 31u));
        int w = 0, r = 0;
        uint32_t M = words[0];
        if (wself == 0) M &= bself;
        uint32_t vnext = S.vstart[s][1];
        uint32_t delta = S.sstart[s][0] - S.vstart[s][0];  // slot - sequence index within range r
        size_t at = (size_t)i;
        // the next neighbour's slot, stored as the next entry; false when none is left
        auto next = [&](uint32_t& slot) {
          while (M == 0u && w + 1 < nw) {
            M = words[++w * q4];
            if (w == wself) M &= bself;
          }
          if (M == 0u) return false;
          const uint32_t v = (uint32_t)(w * 32 + __ffs(M) - 1);
          M &= M - 1u;
          while (v >= vnext) {
            ++r;
            vnext = S.vstart[s][r + 1];
            delta = S.sstart[s][r] - S.vstart[s][r];
          }
          slot = v + delta;
          if (listed < kNbrCap) nbr[at] = slot;
          at += (size_t)n;
          ++listed;
          return true;
        };
        uint32_t sa, sb;
        while (next(sa)) {
          if (!next(sb)) {
            one((int)sa);
            break;
          }
          two((int)sa, (int)sb);
        }
      }
    }
    __syncwarp();
  }
  return listed;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

__global__ void k_set_dt(float* dt, int ninst, float value) {
  for (int q = threadIdx.x; q < ninst; q += blockDim.x) dt[q] = value;
}

// One 32-byte gather record (two float4) in a single 256-bit load.
__device__ __forceinline__ void ld_record(const float4* __restrict__ p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

// Gather records of k_xsph_drift, one 32-byte pair per particle:
// rec[2i] = (x, y, z, m), rec[2i+1] = (v + a dt/2, rho), the half-kicked
// velocity computed as the reference's kick 1 does (lib.rs:301-305). The
// XSPH sum then gathers one sector per neighbour instead of three (it is
// bound by L1 throughput; the other neighbour passes are latency-bound and
// gain nothing from records).
template <class KP>
__global__ void __launch_bounds__(256)
k_xsph_prep(KP kp, int n, const float* __restrict__ dtp, const float4* __restrict__ pos,
            const float4* __restrict__ velout, const float4* __restrict__ acc, float4* __restrict__ rec,
            const uint32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || *err) return;
  float hdt = 0.5f * dtp[kp.at(i).inst];
  float4 v = velout[i], a = acc[i];
  rec[2 * i] = pos[i];
  rec[2 * i + 1] = make_float4(v.x + a.x * hdt, v.y + a.y * hdt, v.z + a.z * hdt, v.w);
}

// Kick 1 (lib.rs:301-305) + XSPH (sph.rs:236-280) + drift (lib.rs:313-317)
// + domain clamp (boundary.rs:239-291) + binning of the new position
// (neighbor.rs:89-101) into a rank-indexed histogram. Reads the sorted state,
// writes the unsorted "U" arrays in the same slot order.
template <class KP>
__global__ void __maxnreg__(SPH_MAXNREG_XSPH)
k_xsph_drift(KP kp, int n, const float* __restrict__ dtp, const float4* __restrict__ pos,
             const float4* __restrict__ velout, const float4* __restrict__ acc, const float4* __restrict__ rec,
             const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
             const uint32_t* __restrict__ rank_of_lin, float4* __restrict__ posU,
             float4* __restrict__ velU, uint32_t* __restrict__ idU, uint32_t* __restrict__ keyU,
             uint32_t* __restrict__ hist, const uint32_t* __restrict__ err,
             const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ ncount) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || *err) return;
  const SimConst& k = kp.at(i);
  float dt = dtp[k.inst];
  float hdt = 0.5f * dt;
  float4 pi = pos[i];
  float4 vi = velout[i];
  float4 ai = acc[i];
  float vx = vi.x + ai.x * hdt;
  float vy = vi.y + ai.y * hdt;
  float vz = vi.z + ai.z * hdt;
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  if (k.flags & kFlagXsph) {
    float rho_i = vi.w;
    // vh = the neighbour's half-kicked velocity and density (k_xsph_prep)
    auto term = [&](const float4& pj, const float4& vh, float dx, float dy, float dz, float d2) {
      float r = sqrtf(d2);
      float w = w_c2(r, k);
      float rho_avg = 0.5f * (rho_i + vh.w);
      float factor = pj.w / fmaxf(rho_avg, 1.0f) * w;
      sx += factor * (vh.x - vx);
      sy += factor * (vh.y - vy);
      sz += factor * (vh.z - vz);
    };
    uint32_t cnt = nbr ? __ldg(&ncount[i]) : 0xffffffffu;
    if (cnt <= kNbrCap) {
      // one 32-byte record per neighbour, two neighbours in flight
      uint32_t c = 0;
      auto pair = [&](int s0, int s1) {
        float4 p0, h0, p1, h1;
        ld_record(rec + 2 * s0, p0, h0);
        ld_record(rec + 2 * s1, p1, h1);
        float ax = pi.x - p0.x, ay = pi.y - p0.y, az = pi.z - p0.z;
        term(p0, h0, ax, ay, az, ax * ax + ay * ay + az * az);
        float bx = pi.x - p1.x, by = pi.y - p1.y, bz = pi.z - p1.z;
        term(p1, h1, bx, by, bz, bx * bx + by * by + bz * bz);
      };
      const uint32_t* e = nbr + i;  // entry c at e[c n]
      // the next four entries are loaded a round ahead, so that a round's
      // record gathers do not wait for its list loads (XSPH -2 %; in k_forces,
      // which holds more live registers, the same is slower)
      int n0 = 0, n1 = 0, n2 = 0, n3 = 0;
      if (cnt >= 4) {
        n0 = (int)__ldg(e);
        n1 = (int)__ldg(e + n);
        n2 = (int)__ldg(e + 2 * (size_t)n);
        n3 = (int)__ldg(e + 3 * (size_t)n);
      }
      for (; c + 3 < cnt; c += 4) {
        const int s0 = n0, s1 = n1, s2 = n2, s3 = n3;
        e += 4 * (size_t)n;
        if (c + 7 < cnt) {
          n0 = (int)__ldg(e);
          n1 = (int)__ldg(e + n);
          n2 = (int)__ldg(e + 2 * (size_t)n);
          n3 = (int)__ldg(e + 3 * (size_t)n);
        }
        pair(s0, s1);
        pair(s2, s3);
      }
      for (; c + 1 < cnt; c += 2) {
        const int s0 = (int)__ldg(e), s1 = (int)__ldg(e + n);
        e += 2 * (size_t)n;
        pair(s0, s1);
      }
      if (c < cnt) {
        int s = (int)__ldg(e);
        float4 pj, vh;
        ld_record(rec + 2 * s, pj, vh);
        float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        term(pj, vh, dx, dy, dz, dx * dx + dy * dy + dz * dz);
      }
    } else {
      for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                        [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
                          term(pj, __ldg(&rec[2 * s + 1]), dx, dy, dz, d2);
                        });
    }
  }
  float dvx = 0.5f * sx, dvy = 0.5f * sy, dvz = 0.5f * sz;
  float x = pi.x + (vx + dvx) * dt;
  float y = pi.y + (vy + dvy) * dt;
  float z = pi.z + (vz + dvz) * dt;
  if (k.flags & kFlagClamp) {
    const float rest = -0.2f;
    if (x < k.dmin[0]) { x = k.dmin[0]; if (vx < 0.0f) vx = rest * vx; }
    if (x > k.dmax[0]) { x = k.dmax[0]; if (vx > 0.0f) vx = rest * vx; }
    if (y < k.dmin[1]) { y = k.dmin[1]; if (vy < 0.0f) vy = rest * vy; }
    if (y > k.dmax[1]) { y = k.dmax[1]; if (vy > 0.0f) vy = rest * vy; }
    if (z < k.dmin[2]) { z = k.dmin[2]; if (vz < 0.0f) vz = rest * vz; }
    if (z > k.dmax[2]) { z = k.dmax[2]; if (vz > 0.0f) vz = rest * vz; }
  }
  posU[i] = make_float4(x, y, z, pi.w);
  velU[i] = make_float4(vx, vy, vz, vi.w);
  idU[i] = id[i];
  int lin = cell_hash(axis_cell(x, k.gmin[0], k.cell, k.dims[0]),
                      axis_cell(y, k.gmin[1], k.cell, k.dims[1]),
                      axis_cell(z, k.gmin[2], k.cell, k.dims[2]), k);
  uint32_t r = __ldg(&rank_of_lin[k.coff + lin]);
  keyU[i] = r;
  atomicAdd(&hist[r], 1u);
}

// Binning of an unsorted state (creation, bootstrap) without moving it.
template <class KP>
__global__ void k_bin(KP kp, int n, const float4* __restrict__ posU,
                      const uint32_t* __restrict__ rank_of_lin, uint32_t* __restrict__ keyU,
                      uint32_t* __restrict__ hist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SimConst& k = kp.at(i);
  float4 p = posU[i];
  int lin = cell_hash(axis_cell(p.x, k.gmin[0], k.cell, k.dims[0]),
                      axis_cell(p.y, k.gmin[1], k.cell, k.dims[1]),
                      axis_cell(p.z, k.gmin[2], k.cell, k.dims[2]), k);
  uint32_t r = __ldg(&rank_of_lin[k.coff + lin]);
  keyU[i] = r;
  atomicAdd(&hist[r], 1u);
}

// ---- exclusive scan of the rank histogram (neighbor.rs:103-110) -----------
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[kScanThreads / 32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < kScanThreads / 32 ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t before = wid > 0 ? warp_sums[wid - 1] : 0u;
  *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const uint32_t* __restrict__ hist, int C, uint32_t* __restrict__ bsum) {
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j)
    if (base + j < C) s += hist[base + j];
  uint32_t total;
  block_excl_scan(s, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// One block: in-place exclusive scan of the tile sums, any count.
__global__ void __launch_bounds__(kScanThreads) k_scan_bsum(uint32_t* __restrict__ bsum, int nb) {
  uint32_t carry = 0;
  for (int base = 0; base < nb; base += kScanThreads) {
    int i = base + threadIdx.x;
    uint32_t v = i < nb ? bsum[i] : 0u;
    uint32_t total;
    uint32_t ex = block_excl_scan(v, &total);
    if (i < nb) bsum[i] = carry + ex;
    carry += total;
  }
}

// Per rank: start, count, cursor; per linear cell: (start, count). Clears
// the histogram for the next binning.
__global__ void __launch_bounds__(kScanThreads)
k_scan_apply(uint32_t* __restrict__ hist, int C, const uint32_t* __restrict__ bsum,
             const uint32_t* __restrict__ lin_of_rank, uint32_t* __restrict__ cstart,
             uint32_t* __restrict__ ccount, uint32_t* __restrict__ cursor, uint2* __restrict__ ctab) {
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = base + j < C ? hist[base + j] : 0u;
    s += v[j];
  }
  uint32_t total;
  uint32_t run = block_excl_scan(s, &total) + bsum[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    int r = base + j;
    if (r < C) {
      cstart[r] = run;
      ccount[r] = v[j];
      cursor[r] = run;
      ctab[lin_of_rank[r]] = make_uint2(run, v[j]);
      hist[r] = 0u;
    }
    run += v[j];
  }
}

// Unordered bucket fill (rank within cell fixed by k_reorder).
__global__ void k_fill(int n, const uint32_t* __restrict__ keyU, const uint32_t* __restrict__ idU,
                       uint32_t* __restrict__ cursor, uint32_t* __restrict__ tmp,
                       uint32_t* __restrict__ tmpid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t slot = atomicAdd(&cursor[keyU[i]], 1u);
  tmp[slot] = (uint32_t)i;
  tmpid[slot] = idU[i];
}

// Final slot = cell start + number of cell members with a smaller original
// id: the stable scatter of neighbor.rs:112-121 in any cell order. Moves the
// particle into the sorted arrays; V = m / rho_old for delta-SPH (sph.rs:199).
__global__ void __launch_bounds__(256)
k_reorder(int n, const uint32_t* __restrict__ tmp, const uint32_t* __restrict__ tmpid,
          const uint32_t* __restrict__ keyU, const uint32_t* __restrict__ cstart,
          const uint32_t* __restrict__ ccount, const float4* __restrict__ posU,
          const float4* __restrict__ velU, float4* __restrict__ pos, float4* __restrict__ vel,
          float2* __restrict__ rv, uint32_t* __restrict__ id, uint32_t* __restrict__ err,
          const float4* __restrict__ accU, float4* __restrict__ acc,
          const float* __restrict__ prU, float* __restrict__ pr, float4* __restrict__ velout, Planes pl) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = tmp[s];
  uint32_t r = keyU[i];
  uint32_t st = cstart[r], cnt = ccount[r];
  uint32_t myid = tmpid[s];
  uint32_t me = myid & kIdMask;
  uint32_t rank = 0;
  if (cnt <= (uint32_t)kCellCap) {
    for (uint32_t q = st; q < st + cnt; ++q) rank += ((__ldg(&tmpid[q]) & kIdMask) < me) ? 1u : 0u;
  } else {
    atomicOr(err, kErrCellCap);
    rank = (uint32_t)s - st;
  }
  uint32_t d = st + rank;
  float4 p = posU[i];
  float4 v = velU[i];
  pos[d] = p;
  pl.xyz[d] = p.x;
  pl.xyz[pl.stride + d] = p.y;
  pl.xyz[2 * pl.stride + d] = p.z;
  vel[d] = v;
  rv[d] = make_float2(v.w, p.w / v.w);
  id[d] = myid;
  if (acc) {  // creation: also place the initial a, p and v
    acc[d] = accU[i];
    pr[d] = prU[i];
    velout[d] = v;
  }
}

// Density summation + delta-SPH + Tait EOS (lib.rs:213-237; sph.rs:112-216,
// 295-312). One thread per sorted particle.
// Closure sample buffers of the density pass (particles within 2h of the
// geometry SDF): count, slot, 16 features, density before correction; and
// the per-particle acceleration correction consumed by k_forces.
struct ClosureBufs {
  uint32_t* count;
  uint32_t* slot;
  float* feat;
  float* rho;
  float4* corr;
  const float4* vel;
  const __nv_bfloat16* wb;  // closure network (mode 2): BF16 weights
  const float* wf;          // and FP32 master parameters (biases)
};

// The learned correction of one particle from the network output y[4]:
// density += y0 rho0 1e-4 (EOS re-evaluated), acceleration correction
// y1..3 |g| stored for k_forces. The outputs are clamped to
// SPH_CLOSURE_MAX_DRHO units (0.3 % of rho0) and SPH_CLOSURE_MAX_ACC_G times
// |g| per component, so a network queried outside its training data cannot
// inject an arbitrarily large correction.
constexpr float kClosureMaxDrho = SPH_CLOSURE_MAX_DRHO;
constexpr float kClosureDrhoUnit = SPH_CLOSURE_DRHO_UNIT;
constexpr float kClosureMaxAcc = SPH_CLOSURE_MAX_ACC_G;
__device__ __forceinline__ void closure_apply_one(const SimConst& k, int i, bool air, float rho_pre, const float* y,
                                                  float2* __restrict__ rf, float* __restrict__ pr,
                                                  float4* __restrict__ corr) {
  float rest = air ? kAirRho0 : kWaterRho0;
  float gm = sqrtf(k.grav[0] * k.grav[0] + k.grav[1] * k.grav[1] + k.grav[2] * k.grav[2]);
  float y0 = fminf(fmaxf(y[0], -kClosureMaxDrho), kClosureMaxDrho);
  float rho = rho_pre + y0 * (rest * kClosureDrhoUnit);
  float p = tait(rho, air, k);
  rf[i] = make_float2(rho, p / (rho * rho));
  pr[i] = p;
  float c1 = fminf(fmaxf(y[1], -kClosureMaxAcc), kClosureMaxAcc);
  float c2 = fminf(fmaxf(y[2], -kClosureMaxAcc), kClosureMaxAcc);
  float c3 = fminf(fmaxf(y[3], -kClosureMaxAcc), kClosureMaxAcc);
  corr[i] = make_float4(c1 * gm, c2 * gm, c3 * gm, 1.0f);
}

// CL = 0: plain step. CL = 1: the particles within 2h of the feature SDF
// record their 16 closure features (capture mode). CL = 2: they also run the
// network in the kernel's epilogue: each warp gathers its near-wall
// particles' features into 16-sample tiles in shared memory and evaluates
// the 16 -> 64 -> 64 -> 4 MLP on the tensor cores (register-resident
// activations), so the corrected density and its EOS are written before the
// kernel ends and no separate inference launch is needed. CL = 2 lifts the
// register cap for the network's fragments.
constexpr int kClTileWords = 16 * 16 / 2 + 16 * 4;  // BF16 x tile + FP32 y tile, in 32-bit words
template <class KP, int CL>
__global__ void __maxnreg__(CL == 2 ? 96 : SPH_MAXNREG_DENSITY)
k_density(KP kp, int n, const float* __restrict__ dtp, const float4* __restrict__ pos, Planes pl,
          const float2* __restrict__ rv, const uint32_t* __restrict__ id,
          const uint2* __restrict__ ctab, const uint32_t* __restrict__ bc_start,
          const uint32_t* __restrict__ bc_list, const float4* __restrict__ bpos,
          float2* __restrict__ rf, float* __restrict__ pr, const uint32_t* __restrict__ err,
          uint32_t* __restrict__ nbr, uint32_t* __restrict__ ncount, const float* __restrict__ sdf,
          const float2* __restrict__ wall_tab, ClosureBufs cb, int warp_scan) {
  // a warp wholly past the end leaves at once; every other lane takes part
  // in the warp scan (and, with CL = 2, in the network epilogue)
  if (blockIdx.x * blockDim.x + (threadIdx.x & ~31u) >= (unsigned)n) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n && !*err;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  // the lane's state (a lane past the end holds slot 0's, unused)
  const int iv = live ? i : 0;
  const SimConst& k = kp.at(iv);
  const float4 pi = pos[iv];
  const float rho_old_i = rv[iv].x;
  float rho = pi.w * k.norm_h3;
  float diff_sum = 0.0f;
  float ssum = 0.0f;  // closure: kernel sum
  const bool delta = (k.flags & kFlagDelta) != 0;
  // density and delta-SPH terms of one neighbour, in list order
  auto term_rv = [&](const float4& pj, const float2& rvj, float dx, float dy, float dz, float d2) {
    float r = sqrtf(d2);
    if (delta) {
      float gx, gy, gz;
      grad_c2(dx, dy, dz, r, k, gx, gy, gz);
      float r_dot_grad = dx * gx + dy * gy + dz * gz;
      float density_diff = rho_old_i - rvj.x;
      diff_sum += rvj.y * density_diff * 2.0f * r_dot_grad / (d2 + k.eta_sq);
    }
    float w = w_c2(r, k);
    rho += pj.w * w;
    if (CL) ssum += rvj.y * w;
  };
  auto term = [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
    term_rv(pj, __ldg(&rv[s]), dx, dy, dz, d2);
  };
  auto pair = [&](int s0, int s1) {  // both neighbours' gathers in flight before either term
    float4 p0 = __ldg(&pos[s0]), p1 = __ldg(&pos[s1]);
    float2 r0 = __ldg(&rv[s0]), r1 = __ldg(&rv[s1]);
    float ax = pi.x - p0.x, ay = pi.y - p0.y, az = pi.z - p0.z;
    term_rv(p0, r0, ax, ay, az, ax * ax + ay * ay + az * az);
    float bx = pi.x - p1.x, by = pi.y - p1.y, bz = pi.z - p1.z;
    term_rv(p1, r1, bx, by, bz, bx * bx + by * by + bz * bz);
  };
  auto single = [&](int s) {
    float4 pj = __ldg(&pos[s]);
    float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    term(s, pj, dx, dy, dz, dx * dx + dy * dy + dz * dz);
  };
  // Phase 1: the warp scan lists every lane's in-support slots in visit order
  // and feeds them to the terms as it lists them. A simulation too small to
  // fill the GPU with warps of 32 particles (warp_scan = 0) takes the
  // per-thread scan instead: more, shorter warps hide its latency better.
  bool fed = false;
  uint32_t listed = 0;
  if (warp_scan)
    listed = scan_warp(kp, i, live, pl, ctab, reinterpret_cast<ScanWarp*>(s_dyn)[threadIdx.x >> 5], nbr, n, pair,
                       single, fed);
  else if (live)
    listed = record_neighbors(pi.x, pi.y, pi.z, i, pl, ctab, ScanGeo(k), nbr, n);
  bool near_wall = false;
  float f[16];
  float rho_pre = 0.0f;
  if (CL != 2 && !live) return;
  if (live) {
    float dt = dtp[k.inst];
    float rho_wall = 0.0f;  // closure: wall density
    uint32_t nwall = 0;
    ncount[i] = listed;
    // Phase 2 (the per-thread scan, or a neighbourhood too large for the warp
    // scan's masks): the terms over the list just stored, or over the cells
    // past its capacity.
    if (!fed) {
      if (listed <= kNbrCap) {
        // the list was written above by this thread: plain (coherent) loads
        uint32_t c = 0;
        const uint32_t* e = nbr + i;  // entry c at e[c n]
        for (; c + 1 < listed; c += 2) {
          const int s0 = (int)e[0], s1 = (int)e[n];
          e += 2 * (size_t)n;
          pair(s0, s1);
        }
        if (c < listed) single((int)e[0]);
      } else {
        for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k, term);
      }
    }
    int lin = cell_hash(axis_cell(pi.x, k.gmin[0], k.cell, k.dims[0]),
                        axis_cell(pi.y, k.gmin[1], k.cell, k.dims[1]),
                        axis_cell(pi.z, k.gmin[2], k.cell, k.dims[2]), k);
    uint32_t b0 = __ldg(&bc_start[k.coff + lin]), b1 = __ldg(&bc_start[k.coff + lin + 1]);
    auto bterm = [&](const float4& bp) {
      float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
      float d2 = dx * dx + dy * dy + dz * dz;
      if (d2 <= k.sup_d2) {
        float wb = bp.w * w_c2(sqrtf(d2), k);
        rho += wb;
        if (CL) { rho_wall += wb; ++nwall; }
      }
    };
    uint32_t q = b0;
    for (; q + 1 < b1; q += 2) {  // two candidates' loads in flight, terms in order
      uint32_t i0 = __ldg(&bc_list[q]), i1 = __ldg(&bc_list[q + 1]);
      float4 bp0 = __ldg(&bpos[i0]), bp1 = __ldg(&bpos[i1]);
      bterm(bp0);
      bterm(bp1);
    }
    if (q < b1) bterm(__ldg(&bpos[__ldg(&bc_list[q])]));
    bool air = (id[i] & kAirBit) != 0;
    float wall_m = 0.0f;
    if (k.sdf_mode) {  // kernel mass of the walls: box faces and obstacle
      BoxFaces bf = box_faces(k, pi.x, pi.y, pi.z);
      float dgeo = k.has_geo ? sdf_sample_clamped(sdf, k, pi.x, pi.y, pi.z) : k.support;
      wall_m = sdf_wall_mass(k, wall_tab, bf, dgeo);
      rho += (air ? kAirRho0 : kWaterRho0) * k.wall_scale * wall_m;
    }
    if (delta) {
      float diffusion = k.delta_coef * diff_sum;
      rho += diffusion * dt;
    }
    float p = tait(rho, air, k);
    rf[i] = make_float2(rho, p / (rho * rho));
    pr[i] = p;
    if (CL) {
      cb.corr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      // feature SDF: the given geometry SDF, or in SDF wall mode the distance
      // to the nearest wall (box face or obstacle)
      auto fsdf = [&](float x, float y, float z) {
        return k.sdf_mode ? wall_distance(k, sdf, x, y, z) : sdf_sample_clamped(sdf, k, x, y, z);
      };
      float d = k.feat_sdf ? fsdf(pi.x, pi.y, pi.z) : k.support;
      if (k.feat_sdf && d < k.support) {
        // Geometry and kinematics only: the particle's own density is not a
        // feature, so the correction cannot soften the equation of state.
        float nx, ny, nz;
        if (k.sdf_mode)
          wall_normal(k, sdf, pi.x, pi.y, pi.z, nx, ny, nz);
        else
          sdf_gradient_clamped(sdf, k, pi.x, pi.y, pi.z, nx, ny, nz);
        float4 v = cb.vel[i];
        float rest = air ? kAirRho0 : kWaterRho0;
        float gm = sqrtf(k.grav[0] * k.grav[0] + k.grav[1] * k.grav[1] + k.grav[2] * k.grav[2]);
        // h * Laplacian of the SDF (sum of the principal curvatures) by second
        // differences at step h; the trilinear field is piecewise linear, so a
        // step of one SDF cell would only see its kinks.
        float lap = fsdf(pi.x + k.h, pi.y, pi.z) + fsdf(pi.x - k.h, pi.y, pi.z) + fsdf(pi.x, pi.y + k.h, pi.z) +
                    fsdf(pi.x, pi.y - k.h, pi.z) + fsdf(pi.x, pi.y, pi.z + k.h) + fsdf(pi.x, pi.y, pi.z - k.h) -
                    6.0f * d;
        f[0] = d / k.h;
        f[1] = nx; f[2] = ny; f[3] = nz;
        f[4] = 1.0f - (rv[i].y * k.norm_h3 + ssum);
        f[5] = (float)listed / 73.0f;
        f[6] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) / k.c;
        f[7] = dt * k.c / k.h;
        f[8] = fminf(fmaxf(lap / k.h, -4.0f), 4.0f);
        f[9] = k.sdf_mode ? k.wall_scale * wall_m : rho_wall / rest;
        f[10] = gm > 0.0f ? (k.grav[0] * nx + k.grav[1] * ny + k.grav[2] * nz) / gm : 0.0f;
        f[11] = f[0] * f[0];
        f[12] = f[8] * f[0];
        f[13] = f[10] * f[0];
        f[14] = (float)nwall / 30.0f;
        f[15] = 1.0f;
        uint32_t q = atomicAdd(cb.count, 1u);
        cb.slot[q] = (uint32_t)i;
        cb.rho[q] = rho;
#pragma unroll
        for (int a = 0; a < 16; ++a) cb.feat[(size_t)q * 16 + a] = f[a];
        near_wall = true;
        rho_pre = rho;
      }
    }
  }  // live
  if (CL == 2) {
    // network epilogue: up to 16 of the warp's near-wall particles per tile
    const int lane = threadIdx.x & 31;
    uint32_t* tile = reinterpret_cast<uint32_t*>(s_dyn + (warp_scan ? (blockDim.x >> 5) * sizeof(ScanWarp) : 0)) +
                     (threadIdx.x >> 5) * kClTileWords;
    __nv_bfloat16* xt = reinterpret_cast<__nv_bfloat16*>(tile);
    float* yt = reinterpret_cast<float*>(tile + 16 * 16 / 2);
    unsigned pending = __ballot_sync(0xffffffffu, near_wall);
    while (pending) {
      unsigned rest = pending;  // the lowest 16 pending lanes form this tile
      for (int q = 0; q < 16 && rest; ++q) rest &= rest - 1u;
      unsigned take = pending & ~rest;
      pending = rest;
      const bool mine = (take >> lane) & 1u;
      const int row = __popc(take & ((1u << lane) - 1u));
      const int cnt = __popc(take);
      if (mine) {
#pragma unroll
        for (int a = 0; a < 16; ++a) xt[row * 16 + a] = __float2bfloat16_rn(f[a]);
      }
      for (int q = lane; q < 256; q += 32)
        if ((q >> 4) >= cnt) xt[q] = __float2bfloat16_rn(0.0f);
      __syncwarp();
      sphmlp::forward_tile_regs(xt, cb.wb, cb.wf, yt, lane);
      __syncwarp();
      if (mine) {
        const SimConst& k = kp.at(i);
        closure_apply_one(k, i, (id[i] & kAirBit) != 0, rho_pre, yt + row * 4, rf, pr, cb.corr);
      }
      __syncwarp();
    }
  }
}

// Adami boundary pressure (boundary.rs:87-131). One warp per boundary
// particle: the lanes evaluate the in-support fluid terms of a widened cell
// range, a warp bitonic sort orders them by fluid index, and lane 0 sums
// them in that order.
constexpr int kAdamiWarps = 4;
// Marks the boundary particles that an occupied fluid cell lists as
// candidates (bc_start/bc_list: every boundary particle whose support can
// reach a particle of the cell). A boundary particle with a fluid particle in
// support is marked; an unmarked one has no terms, and its Adami pressure is
// the empty sum's 0.
// One warp per cell with a non-empty list (`cells`, ncl of them), the lanes
// taking the cell's list entries in turn.
__global__ void k_adami_mark(int ncl, const uint32_t* __restrict__ cells, const uint2* __restrict__ ctab,
                             const uint32_t* __restrict__ bc_start, const uint32_t* __restrict__ bc_list,
                             uint8_t* __restrict__ act) {
  int w = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= ncl) return;
  uint32_t c = __ldg(&cells[w]);
  if (__ldg(&ctab[c]).y == 0u) return;
  uint32_t q1 = __ldg(&bc_start[c + 1]);
  for (uint32_t q = __ldg(&bc_start[c]) + lane; q < q1; q += 32) act[__ldg(&bc_list[q])] = 1;
}

// One boundary particle's in-support fluid term (boundary.rs:100-115): its
// kernel weight w, the weighted extrapolated pressure w p_ext and the fluid
// particle's original index (the order of the reference's sum).
template <class KC>
__device__ __forceinline__ bool adami_term(const KC& k, const float4& bp, int s, const float4* __restrict__ pos,
                                           const float2* __restrict__ rf, const float* __restrict__ pr,
                                           const uint32_t* __restrict__ id, float& w, float& wp, uint32_t& fid) {
  float4 pf = __ldg(&pos[s]);
  float dx = bp.x - pf.x, dy = bp.y - pf.y, dz = bp.z - pf.z;
  float d2 = dx * dx + dy * dy + dz * dz;
  if (!(d2 <= k.sup_d2)) return false;
  w = w_c2(sqrtf(d2), k);
  float g_dot_dr = k.grav[0] * dx + k.grav[1] * dy + k.grav[2] * dz;
  float p_ext = __ldg(&pr[s]) + __ldg(&rf[s]).x * g_dot_dr;
  wp = w * p_ext;
  fid = __ldg(&id[s]) & kIdMask;
  return true;
}

// The in-support fluid terms of boundary particle bp (one warp): the cells of
// a widened range around it are looked up 32 at a time, and their candidates
// taken 32 at a time across cells; the terms go to sid / sw / swp (up to
// kAdamiCap) in candidate order. Returns the term count; `overflow` is set
// on every lane when it exceeds kAdamiCap.
__device__ __forceinline__ int adami_search(const SimConst& k, const float4& bp, const float4* __restrict__ pos,
                                            const float2* __restrict__ rf, const float* __restrict__ pr,
                                            const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
                                            uint32_t* sid, float* sw, float* swp, bool& overflow) {
  const int lane = threadIdx.x & 31;
  int lo[3], hi[3];
  float bc[3] = {bp.x, bp.y, bp.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = axis_cell(bc[a] - k.reach, k.gmin[a], k.cell, k.dims[a]);
    hi[a] = axis_cell(bc[a] + k.reach, k.gmin[a], k.cell, k.dims[a]);
  }
  int count = 0;
  overflow = false;
  // Lanes look up the (at most 4x4x4) cells of the range in parallel; only
  // occupied cells whose box comes within 2h are then scanned (the box is
  // widened by a margin far above the rounding of the binning, edge cells
  // unbounded outward, as particles outside the domain are binned there),
  // their candidates taken 32 at a time across cells. The terms are sorted
  // by fluid index below, so the order of the candidates does not matter.
  int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
  int ncell = nx * ny * nz;
  const float margin = 1.0e-5f * k.cell + 1.0e-6f;
  for (int cbase = 0; cbase < ncell; cbase += 32) {
    int q = cbase + lane;
    uint2 mine = make_uint2(0u, 0u);
    if (q < ncell) {
      int c3[3] = {lo[0] + q % nx, lo[1] + (q / nx) % ny, lo[2] + q / (nx * ny)};
      float gap2 = 0.0f;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float face = k.gmin[a] + (float)c3[a] * k.cell;
        float below = c3[a] > 0 ? face - margin - bc[a] : 0.0f;
        float above = c3[a] < k.dims[a] - 1 ? bc[a] - (face + k.cell + margin) : 0.0f;
        float g = fmaxf(fmaxf(below, above), 0.0f);
        gap2 += g * g;
      }
      if (gap2 <= k.radius_sq) mine = __ldg(&ctab[k.coff + cell_hash(c3[0], c3[1], c3[2], k)]);
    }
    // the candidates of this round's cells as one stream, 32 at a time: lane
    // l takes candidate t = base + l, which lies in the cell whose prefix range
    // [excl, incl) holds it (the last lane with excl <= t, by bisection)
    uint32_t incl = mine.y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    uint32_t excl = incl - mine.y;
    uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
      uint32_t t = base + lane;
      int src = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        uint32_t e = __shfl_sync(0xffffffffu, excl, src + step);
        if (e <= t) src += step;
      }
      uint32_t st = __shfl_sync(0xffffffffu, mine.x, src);
      uint32_t s = st + (t - __shfl_sync(0xffffffffu, excl, src));
      {
        float w = 0.0f, wp = 0.0f;
        uint32_t fid = 0;
        const bool inr = t < total && adami_term(k, bp, (int)s, pos, rf, pr, id, w, wp, fid);
        unsigned m = __ballot_sync(0xffffffffu, inr);
        int off = count + __popc(m & ((1u << lane) - 1u));
        if (inr) {
          if (off < kAdamiCap) {
            sid[off] = fid;
            sw[off] = w;
            swp[off] = wp;
          } else {
            overflow = true;
          }
        }
        count += __popc(m);
      }
    }
  }
  overflow = __any_sync(0xffffffffu, overflow);
  return count;
}

// The Adami pressure of one boundary particle from its `count` terms in
// sid / sw / swp (one warp): the terms are ordered by fluid index (bitonic,
// in registers up to 32 terms, else in shared memory) and summed in that
// order, as the reference sums over the fluid particles in index order
// (boundary.rs:100-123); lane 0 writes *out.
__device__ __forceinline__ void adami_sum(int count, bool overflow, uint32_t* sid, float* sw, float* swp,
                                          float* __restrict__ out, uint32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  if (overflow || count > kAdamiCap) {
    if (lane == 0) atomicOr(err, kErrAdamiCap);
    return;
  }
  // lane 0 sums the ordered terms, in order (four at a time per 16-byte load
  // where the arrays allow it; the additions are the same)
  auto ordered_sum = [&]() {
    float weighted_pressure = 0.0f, weight_sum = 0.0f;
    int q = 0;
    if ((reinterpret_cast<uintptr_t>(sw) & 15u) == 0 && (reinterpret_cast<uintptr_t>(swp) & 15u) == 0)
      for (; q + 3 < count; q += 4) {
        const float4 a = *reinterpret_cast<const float4*>(swp + q), c = *reinterpret_cast<const float4*>(sw + q);
        weighted_pressure += a.x;
        weighted_pressure += a.y;
        weighted_pressure += a.z;
        weighted_pressure += a.w;
        weight_sum += c.x;
        weight_sum += c.y;
        weight_sum += c.z;
        weight_sum += c.w;
      }
    for (; q < count; ++q) {
      weighted_pressure += swp[q];
      weight_sum += sw[q];
    }
    *out = weight_sum > 1.0e-12f ? fmaxf(weighted_pressure / weight_sum, 0.0f) : 0.0f;
  };
  if (count <= 32) {
    // up to 32 terms, one per lane: each lane's rank is the number of smaller
    // fluid indices (they are distinct), and the terms are stored at their
    // ranks, i.e. in fluid-index order
    __syncwarp();
    const uint32_t key = lane < count ? sid[lane] : 0xffffffffu;
    const float w = lane < count ? sw[lane] : 0.0f;
    const float wp = lane < count ? swp[lane] : 0.0f;
    int rank = 0;
    for (int q = 0; q < count; ++q) rank += __shfl_sync(0xffffffffu, key, q) < key ? 1 : 0;
    __syncwarp();
    if (lane < count) {
      sw[rank] = w;
      swp[rank] = wp;
    }
    __syncwarp();
    if (lane == 0) ordered_sum();
    return;
  }
  int m2 = 1;
  while (m2 < count) m2 <<= 1;
  for (int q = count + lane; q < m2; q += 32) sid[q] = 0xffffffffu;
  __syncwarp();
  for (int kk = 2; kk <= m2; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < m2; q += 32) {
        int pq = q ^ j;
        if (pq > q) {
          bool up = (q & kk) == 0;
          uint32_t a = sid[q], c = sid[pq];
          if ((a > c) == up) {
            sid[q] = c; sid[pq] = a;
            float t = sw[q]; sw[q] = sw[pq]; sw[pq] = t;
            t = swp[q]; swp[q] = swp[pq]; swp[pq] = t;
          }
        }
      }
      __syncwarp();
    }
  }
  if (lane == 0) ordered_sum();
}

template <class KP>
__global__ void __launch_bounds__(kAdamiWarps * 32)
k_adami(KP kp, int nb, const float4* __restrict__ bpos, float* __restrict__ bpress,
        const float4* __restrict__ pos, const float2* __restrict__ rf, const float* __restrict__ pr,
        const uint32_t* __restrict__ id, const uint2* __restrict__ ctab, uint32_t* __restrict__ err,
        const uint8_t* __restrict__ act) {
  __shared__ uint32_t s_id[kAdamiWarps][kAdamiCap];
  __shared__ float s_w[kAdamiWarps][kAdamiCap];
  __shared__ float s_wp[kAdamiWarps][kAdamiCap];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int b = blockIdx.x * kAdamiWarps + warp;
  if (b >= nb || *err) return;
  if (!act[b]) {  // no fluid particle can be in support (k_adami_mark)
    if (lane == 0) bpress[b] = 0.0f;
    return;
  }
  bool overflow;
  const int count = adami_search(kp.at(b), bpos[b], pos, rf, pr, id, ctab, s_id[warp], s_w[warp], s_wp[warp],
                                 overflow);
  adami_sum(count, overflow, s_id[warp], s_w[warp], s_wp[warp], bpress + b, err);
}

// Adami boundary pressure with the boundary particles taken cell by cell (the
// row cell order, where a row's cells are consecutive). The boundary
// particles are visited in `border`, sorted once by the cell that holds them
// (they do not move), so that a warp's 32 entries fall into few cells. The
// active particles of one cell run (a "segment") share one candidate
// sequence: the (y, z) rows of the union of their widened ranges, each row
// the union's x-cells as one slot range, less the rows whose (y, z) box lies
// farther than 2h from the segment's bounding box (with adami_search's margin
// and unbounded edge cells). Every cell that adami_search scans for one of
// them lies in it, so no in-support fluid particle is missed. The lanes load
// 32 candidates of the sequence at a time and test them against four of the
// segment's particles at a time (two f32x2 chains, rounded as the scalar
// expression), one ballot mask per particle. Each particle's in-support
// candidates are then gathered, their terms evaluated one per lane
// (adami_term), and summed by adami_sum in fluid-index order. A segment whose
// sequence passes the masks' capacity takes adami_search per particle.
constexpr int kAdamiRows = 25;   // (y, z) rows per segment: at most 5 x 5
constexpr int kAdamiWords = 32;  // mask words per particle: up to 1024 candidates
struct __align__(16) AdamiWarp {
  float px[36], py[36], pz[36];          // the segment's particles, padded to quads with NaN
  uint32_t mask[kAdamiWords * 32];       // [word][particle]
  uint32_t sid[kAdamiCap];               // a particle's candidates (sequence index), then its terms' fluid ids
  float sw[kAdamiCap], swp[kAdamiCap];
  uint32_t vstart[kAdamiRows + 1];       // sequence index of each row's first candidate; [R] = total
  uint32_t sstart[kAdamiRows];           // slot of each row's first candidate
};
static_assert(offsetof(AdamiWarp, py) % 16 == 0 && offsetof(AdamiWarp, pz) % 16 == 0 &&
                  offsetof(AdamiWarp, mask) % 16 == 0 && offsetof(AdamiWarp, sw) % 16 == 0 &&
                  offsetof(AdamiWarp, swp) % 16 == 0 && sizeof(AdamiWarp) % 16 == 0,
              "quad loads and stores");

template <class KP>
__global__ void __launch_bounds__(kAdamiWarps * 32)
k_adami_cells(KP kp, int nb, const uint32_t* __restrict__ border, const float4* __restrict__ bpos,
              float* __restrict__ bpress, const float4* __restrict__ pos, Planes pl,
              const float2* __restrict__ rf, const float* __restrict__ pr, const uint32_t* __restrict__ id,
              const uint2* __restrict__ ctab, uint32_t* __restrict__ err, const uint8_t* __restrict__ act) {
  __shared__ AdamiWarp s_aw[kAdamiWarps];
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  AdamiWarp& S = s_aw[threadIdx.x >> 5];
  const int e0 = (blockIdx.x * kAdamiWarps + (threadIdx.x >> 5)) * 32;
  if (e0 >= nb || *err) return;  // whole warps
  const int e = e0 + lane;
  const bool valid = e < nb;
  const int b = valid ? (int)__ldg(&border[e]) : (int)__ldg(&border[e0]);
  const bool live = valid && act[b];
  if (valid && !live) bpress[b] = 0.0f;  // no fluid particle can be in support (k_adami_mark)
  const uint32_t livemask = __ballot_sync(kAll, live);
  if (!livemask) return;
  const float* xs = pl.xyz;
  const float* ys = xs + pl.stride;
  const float* zs = ys + pl.stride;
  const float nan = __int_as_float(0x7fc00000);
  const float4 bp = __ldg(&bpos[b]);
  uint32_t key = 0xffffffffu;
  if (live) {
    const SimConst& k = kp.at(b);
    key = (uint32_t)(k.coff + cell_hash(axis_cell(bp.x, k.gmin[0], k.cell, k.dims[0]),
                                        axis_cell(bp.y, k.gmin[1], k.cell, k.dims[1]),
                                        axis_cell(bp.z, k.gmin[2], k.cell, k.dims[2]), k));
  }
  const uint32_t prev = __shfl_up_sync(kAll, key, 1);
  const uint32_t heads = __ballot_sync(kAll, live && (lane == 0 || prev != key));
  for (uint32_t hh = heads; hh; hh &= hh - 1u) {
    const int hl = __ffs(hh) - 1;
    const uint32_t after = heads & ~(hl == 31 ? kAll : (2u << hl) - 1u);
    const int he = after ? __ffs(after) - 1 : 32;
    const uint32_t segmask = (he == 32 ? kAll : (1u << he) - 1u) & ~((1u << hl) - 1u);
    const uint32_t members = livemask & segmask;  // the segment's active particles
    const int m = __popc(members);
    const bool mine = (members >> lane) & 1u;
    const SimConst& k = kp.at(__shfl_sync(kAll, b, hl));
    // bounding box of the members, and the union of their widened ranges
    float lo3[3] = {mine ? bp.x : INFINITY, mine ? bp.y : INFINITY, mine ? bp.z : INFINITY};
    float hi3[3] = {mine ? bp.x : -INFINITY, mine ? bp.y : -INFINITY, mine ? bp.z : -INFINITY};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo3[a] = fminf(lo3[a], __shfl_xor_sync(kAll, lo3[a], o));
        hi3[a] = fmaxf(hi3[a], __shfl_xor_sync(kAll, hi3[a], o));
      }
    int clo[3], chi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      clo[a] = axis_cell(lo3[a] - k.reach, k.gmin[a], k.cell, k.dims[a]);
      chi[a] = axis_cell(hi3[a] + k.reach, k.gmin[a], k.cell, k.dims[a]);
    }
    const int ny = chi[1] - clo[1] + 1, nz = chi[2] - clo[2] + 1, R = ny * nz;
    uint32_t len = 0, st = 0;
    if (lane < R && R <= kAdamiRows) {
      const int cy = clo[1] + lane % ny, cz = clo[2] + lane / ny;
      const float margin = 1.0e-5f * k.cell + 1.0e-6f;  // as adami_search
      float gap2 = 0.0f;
      const int c2[2] = {cy, cz};
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int a = q + 1;
        const float face = k.gmin[a] + (float)c2[q] * k.cell;
        const float below = c2[q] > 0 ? face - margin - hi3[a] : 0.0f;
        const float above = c2[q] < k.dims[a] - 1 ? lo3[a] - (face + k.cell + margin) : 0.0f;
        const float g = fmaxf(fmaxf(below, above), 0.0f);
        gap2 += g * g;
      }
      if (gap2 <= k.radius_sq) {
        const int row = k.coff + (cy + cz * k.dims[1]) * k.dims[0];
        const uint2 sa = __ldg(&ctab[row + clo[0]]), sb = __ldg(&ctab[row + chi[0]]);
        st = sa.x;
        len = sb.x + sb.y - sa.x;
      }
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(kAll, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(kAll, incl, 31);
    const int nw = (int)((total + 31u) / 32u);
    const int q4 = (m + 3) & ~3;
    const bool fits = R <= kAdamiRows && nw <= kAdamiWords;
    __syncwarp();  // the previous segment's last reads of the tables are done
    if (lane < R && R <= kAdamiRows) {
      S.vstart[lane] = incl - len;
      S.sstart[lane] = st;
    }
    if (lane == 0 && R <= kAdamiRows) S.vstart[R] = total;
    const int mp = __popc(members & ((1u << lane) - 1u));  // this lane's index among the members
    if (mine) {
      S.px[mp] = bp.x;
      S.py[mp] = bp.y;
      S.pz[mp] = bp.z;
    }
    if (lane >= m && lane < q4) {
      S.px[lane] = nan;
      S.py[lane] = nan;
      S.pz[lane] = nan;
    }
    __syncwarp();
    // the row holding sequence index v (< total): the last row starting at or before it
    auto row_of = [&](uint32_t v) {
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1)
        if (r + step < R && S.vstart[r + step] <= v) r += step;
      return r;
    };
    if (fits) {
      const float r2 = k.sup_d2;
      float nxv = nan, nyv = nan, nzv = nan;
      auto fetch = [&](int w) {  // candidate 32 w + lane (NaN past the end: in no particle's support)
        const uint32_t v = (uint32_t)(w * 32 + lane);
        nxv = nan;
        nyv = nan;
        nzv = nan;
        if (v < total) {
          const int r = row_of(v);
          const uint32_t slot = S.sstart[r] + (v - S.vstart[r]);
          nxv = __ldg(&xs[slot]);
          nyv = __ldg(&ys[slot]);
          nzv = __ldg(&zs[slot]);
        }
      };
      fetch(0);
      for (int w = 0; w < nw; ++w) {
        const unsigned long long CX = f2_pack(nxv, nxv), CY = f2_pack(nyv, nyv), CZ = f2_pack(nzv, nzv);
        if (w + 1 < nw) fetch(w + 1);
        uint32_t* const row = S.mask + w * q4;
        for (int p = 0; p < m; p += 4) {  // boundary minus fluid, as adami_term
          const float4 ax = *reinterpret_cast<const float4*>(&S.px[p]);
          const float4 ay = *reinterpret_cast<const float4*>(&S.py[p]);
          const float4 az = *reinterpret_cast<const float4*>(&S.pz[p]);
          const unsigned long long dx0 = f2_sub(f2_pack(ax.x, ax.y), CX), dx1 = f2_sub(f2_pack(ax.z, ax.w), CX);
          const unsigned long long dy0 = f2_sub(f2_pack(ay.x, ay.y), CY), dy1 = f2_sub(f2_pack(ay.z, ay.w), CY);
          const unsigned long long dz0 = f2_sub(f2_pack(az.x, az.y), CZ), dz1 = f2_sub(f2_pack(az.z, az.w), CZ);
          float d0, d1, d2, d3;
          f2_unpack(f2_add(f2_add(f2_mul(dx0, dx0), f2_mul(dy0, dy0)), f2_mul(dz0, dz0)), d0, d1);
          f2_unpack(f2_add(f2_add(f2_mul(dx1, dx1), f2_mul(dy1, dy1)), f2_mul(dz1, dz1)), d2, d3);
          const uint32_t M0 = __ballot_sync(kAll, d0 <= r2), M1 = __ballot_sync(kAll, d1 <= r2);
          const uint32_t M2 = __ballot_sync(kAll, d2 <= r2), M3 = __ballot_sync(kAll, d3 <= r2);
          if (lane == 0) *reinterpret_cast<uint4*>(row + p) = make_uint4(M0, M1, M2, M3);
        }
      }
    }
    __syncwarp();
    // Each member in turn: its terms, then their ordered sum. A member with
    // up to 32 terms leaves them ordered in sw / swp from `base`, and its sum
    // waits: the pending members are summed together, one per lane, each in
    // its own order (the same additions as adami_sum's), when the arrays
    // fill up, before a member that needs them whole, and at the end.
    int npend = 0, base = 0;
    int pend_b = 0, pend_base = 0, pend_count = 0;  // lane j: pending member j
    auto flush = [&]() {
      __syncwarp();
      if (lane < npend) {
        float weighted_pressure = 0.0f, weight_sum = 0.0f;
        for (int q = 0; q < pend_count; ++q) {
          weighted_pressure += S.swp[pend_base + q];
          weight_sum += S.sw[pend_base + q];
        }
        bpress[pend_b] = weight_sum > 1.0e-12f ? fmaxf(weighted_pressure / weight_sum, 0.0f) : 0.0f;
      }
      __syncwarp();
      npend = 0;
      base = 0;
    };
    for (uint32_t mm = members; mm; mm &= mm - 1u) {
      const int ml = __ffs(mm) - 1;
      const int p = __popc(members & ((1u << ml) - 1u));
      const int bm = __shfl_sync(kAll, b, ml);
      const float4 bpm = make_float4(__shfl_sync(kAll, bp.x, ml), __shfl_sync(kAll, bp.y, ml),
                                     __shfl_sync(kAll, bp.z, ml), 0.0f);
      int count = 0;
      bool overflow = false;
      if (fits) {
        for (int w = 0; w < nw; ++w) {  // the in-support candidates, in sequence order
          const uint32_t M = S.mask[w * q4 + p];
          if (M == 0u) continue;
          if ((M >> lane) & 1u) {
            const int at = count + __popc(M & ((1u << lane) - 1u));
            if (at < kAdamiCap) S.sid[at] = (uint32_t)(w * 32 + lane);
          }
          count += __popc(M);
        }
        overflow = count > kAdamiCap;
        __syncwarp();
        if (count <= 32) {
          // one term per lane, placed at its rank (the count of smaller fluid indices)
          float w = 0.0f, wp = 0.0f;
          uint32_t fid = 0xffffffffu;
          if (lane < count) {
            const uint32_t v = S.sid[lane];
            const int r = row_of(v);
            adami_term(k, bpm, (int)(S.sstart[r] + (v - S.vstart[r])), pos, rf, pr, id, w, wp, fid);
          }
          int rank = 0;
          for (int q = 0; q < count; ++q) rank += __shfl_sync(kAll, fid, q) < fid ? 1 : 0;
          if (base + count > kAdamiCap || npend == 32) flush();
          if (lane < count) {
            S.sw[base + rank] = w;
            S.swp[base + rank] = wp;
          }
          if (lane == npend) {
            pend_b = bm;
            pend_base = base;
            pend_count = count;
          }
          ++npend;
          base += count;
          __syncwarp();
          continue;
        }
        flush();  // the arrays are needed whole
        const int nt = count < kAdamiCap ? count : kAdamiCap;
        for (int t = lane; t < nt; t += 32) {
          const uint32_t v = S.sid[t];
          const int r = row_of(v);
          float w = 0.0f, wp = 0.0f;
          uint32_t fid = 0;
          adami_term(k, bpm, (int)(S.sstart[r] + (v - S.vstart[r])), pos, rf, pr, id, w, wp, fid);
          S.sid[t] = fid;
          S.sw[t] = w;
          S.swp[t] = wp;
        }
        __syncwarp();
      } else {
        flush();
        count = adami_search(k, bpm, pos, rf, pr, id, ctab, S.sid, S.sw, S.swp, overflow);
      }
      adami_sum(count, overflow, S.sid, S.sw, S.swp, bpress + bm, err);
      __syncwarp();
    }
    flush();
  }
}

// Pressure force + Monaghan viscosity + gravity + boundary pressure force +
// repulsion (lib.rs:247-282; sph.rs:322-508; boundary.rs:143-181), then
// kick 2 (lib.rs:330-334) and the dt reduction inputs (sph.rs:597-616).
template <class KP, int CL>
__global__ void __maxnreg__(SPH_MAXNREG_FORCES)
k_forces(KP kp, int n, const float* __restrict__ dtp, float hdt_scale,
         const float4* __restrict__ pos, const float4* __restrict__ vel,
         const float2* __restrict__ rf, const float* __restrict__ pr,
         const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
         const uint32_t* __restrict__ bc_start, const uint32_t* __restrict__ bc_list,
         const float4* __restrict__ bpos, const float* __restrict__ bpress,
         float4* __restrict__ acc, float4* __restrict__ velout, float* __restrict__ red,
         const uint32_t* __restrict__ err, const uint32_t* __restrict__ nbr,
         const uint32_t* __restrict__ ncount, const float* __restrict__ sdf,
         const float2* __restrict__ wall_tab, const float4* __restrict__ corr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float sig = 0.0f, amag = 0.0f;
  int inst = -1;
  if (i < n && !*err) {
    const SimConst& k = kp.at(i);
    inst = k.inst;
    float hdt = (0.5f * dtp[k.inst]) * hdt_scale;
    float4 pi = pos[i];
    float4 vi = vel[i];
    float2 rfi = rf[i];
    float rho_i = rfi.x;
    float fpx = 0.0f, fpy = 0.0f, fpz = 0.0f;
    float fvx = 0.0f, fvy = 0.0f, fvz = 0.0f;
    float neg_mi = -pi.w;
    // one neighbour's terms, its position, velocity and (rho, p / rho^2) given
    auto term = [&](const float4& pj, const float4& vj, const float2& rfj, float dx, float dy, float dz,
                    float d2) {
      float r = sqrtf(d2);
      float gx, gy, gz;
      grad_c2(dx, dy, dz, r, k, gx, gy, gz);
      float factor = neg_mi * pj.w * (rfi.y + rfj.y);
      fpx += factor * gx;
      fpy += factor * gy;
      fpz += factor * gz;
      float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
      float vr_dot = dvx * dx + dvy * dy + dvz * dz;
      // every pair evaluates the viscous term (no divergent branch, -2.4 %
      // forces); a receding pair (v.r >= 0, sph.rs:460) adds a signed zero,
      // which leaves the sums unchanged: they start at +0 and a sum that
      // rounds to zero is +0, so they never hold -0
      float r_sq = r * r;
      float mu = k.h * vr_dot / (r_sq + k.eta_sq);
      float rho_avg = 0.5f * (rho_i + rfj.x);
      float pi_ij = (k.neg_alpha_c * mu + k.beta * mu * mu) / rho_avg;
      float fv = vr_dot < 0.0f ? -pj.w * pi_ij : 0.0f;
      fvx += fv * gx;
      fvy += fv * gy;
      fvz += fv * gz;
    };
    uint32_t cnt = nbr ? __ldg(&ncount[i]) : 0xffffffffu;
    if (cnt <= kNbrCap) {
      // both neighbours' gathers (position, velocity, density) issued before either term
      auto pair = [&](int s0, int s1) {
        float4 p0 = __ldg(&pos[s0]), p1 = __ldg(&pos[s1]);
        float4 v0 = __ldg(&vel[s0]), v1 = __ldg(&vel[s1]);
        float2 f0 = __ldg(&rf[s0]), f1 = __ldg(&rf[s1]);
        float ax = pi.x - p0.x, ay = pi.y - p0.y, az = pi.z - p0.z;
        term(p0, v0, f0, ax, ay, az, ax * ax + ay * ay + az * az);
        float bx = pi.x - p1.x, by = pi.y - p1.y, bz = pi.z - p1.z;
        term(p1, v1, f1, bx, by, bz, bx * bx + by * by + bz * bz);
      };
      uint32_t c = 0;
      const uint32_t* e = nbr + i;  // entry c at e[c n]
      for (; c + 3 < cnt; c += 4) {
        const int s0 = (int)__ldg(e), s1 = (int)__ldg(e + n), s2 = (int)__ldg(e + 2 * (size_t)n),
                  s3 = (int)__ldg(e + 3 * (size_t)n);
        e += 4 * (size_t)n;
        pair(s0, s1);
        pair(s2, s3);
      }
      for (; c + 1 < cnt; c += 2) {
        const int s0 = (int)__ldg(e), s1 = (int)__ldg(e + n);
        e += 2 * (size_t)n;
        pair(s0, s1);
      }
      if (c < cnt) {
        int s = (int)__ldg(e);
        float4 pj = __ldg(&pos[s]);
        float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        term(pj, __ldg(&vel[s]), __ldg(&rf[s]), dx, dy, dz, dx * dx + dy * dy + dz * dz);
      }
    } else {
      for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                        [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
                          term(pj, __ldg(&vel[s]), __ldg(&rf[s]), dx, dy, dz, d2);
                        });
    }
    int lin = cell_hash(axis_cell(pi.x, k.gmin[0], k.cell, k.dims[0]),
                        axis_cell(pi.y, k.gmin[1], k.cell, k.dims[1]),
                        axis_cell(pi.z, k.gmin[2], k.cell, k.dims[2]), k);
    uint32_t b0 = __ldg(&bc_start[k.coff + lin]), b1 = __ldg(&bc_start[k.coff + lin + 1]);
    bool air = (id[i] & kAirBit) != 0;
    if (b1 > b0) {
      float pic = fmaxf(pr[i], 0.0f);
      float pic_over = pic / (rho_i * rho_i);
      float brho = air ? kAirRho0 : kWaterRho0;
      float brho2 = brho * brho;
      auto bterm = [&](uint32_t bi, const float4& bp) {
        float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
        float d2 = dx * dx + dy * dy + dz * dz;
        if (d2 <= k.sup_d2) {
          float r = sqrtf(d2);
          float gx, gy, gz;
          grad_c2(dx, dy, dz, r, k, gx, gy, gz);
          float pb_over = __ldg(&bpress[bi]) / brho2;
          float factor = neg_mi * bp.w * (pic_over + pb_over);
          fpx += factor * gx;
          fpy += factor * gy;
          fpz += factor * gz;
        }
      };
      uint32_t q = b0;
      for (; q + 1 < b1; q += 2) {  // two candidates' loads in flight, terms in order
        uint32_t i0 = __ldg(&bc_list[q]), i1 = __ldg(&bc_list[q + 1]);
        float4 bp0 = __ldg(&bpos[i0]), bp1 = __ldg(&bpos[i1]);
        bterm(i0, bp0);
        bterm(i1, bp1);
      }
      if (q < b1) {
        uint32_t bi = __ldg(&bc_list[q]);
        bterm(bi, __ldg(&bpos[bi]));
      }
    }
    float ax = 0.0f + fpx / pi.w, ay = 0.0f + fpy / pi.w, az = 0.0f + fpz / pi.w;
    ax += fvx; ay += fvy; az += fvz;
    ax += k.grav[0]; ay += k.grav[1]; az += k.grav[2];
    if (k.sdf_mode) {
      // pressure force of the homogenised wall layers: the energy-consistent
      // counterpart of their kernel mass in rho_i (the gradient of
      // E = sum m e(rho) gives a_i += (p_i / rho_i^2) rho0 s grad(phi) per
      // wall term, the particle's own pressure only). Box faces per axis
      // (singles - edges + corner, then each face's repulsion), then the
      // obstacle along its SDF normal.
      float rest = air ? kAirRho0 : kWaterRho0;
      float pic = fmaxf(pr[i], 0.0f);
      float pic_over = pic / (rho_i * rho_i);
      float cw = rest * k.wall_scale;
      float base = pic_over * cw;
      BoxFaces bf = box_faces(k, pi.x, pi.y, pi.z);
      float wa[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (bf.on[a]) wa[a] += base * wall_lookup(wall_tab, k.wall_inv_step, bf.d[a]).y * bf.s[a];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = a + 1; c < 3; ++c)
          if (bf.on[a] && bf.on[c]) {
            wa[a] -= base * wall_lookup2(wall_tab, k.wall_inv2, bf.d[a], bf.d[c]).y * bf.s[a];
            wa[c] -= base * wall_lookup2(wall_tab, k.wall_inv2, bf.d[c], bf.d[a]).y * bf.s[c];
          }
      if (bf.on[0] && bf.on[1] && bf.on[2]) {
        wa[0] += base * wall_lookup3(wall_tab, k.wall_inv3, bf.d[0], bf.d[1], bf.d[2]).y * bf.s[0];
        wa[1] += base * wall_lookup3(wall_tab, k.wall_inv3, bf.d[1], bf.d[0], bf.d[2]).y * bf.s[1];
        wa[2] += base * wall_lookup3(wall_tab, k.wall_inv3, bf.d[2], bf.d[0], bf.d[1]).y * bf.s[2];
      }
      if (k.flags & kFlagRepulsion) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (bf.d[a] < k.r0) {
            float s = 1.0f - fmaxf(bf.d[a], 0.0f) / k.r0;
            float fm = k.sdf_coef * s * s / k.r0;
            wa[a] += fm * bf.s[a];
          }
      }
      ax += wa[0];
      ay += wa[1];
      az += wa[2];
      float d = k.has_geo ? sdf_sample_clamped(sdf, k, pi.x, pi.y, pi.z) : k.support;
      if (d < k.support) {
        float nx, ny, nz;
        sdf_gradient_clamped(sdf, k, pi.x, pi.y, pi.z, nx, ny, nz);
        float coef = base * wall_lookup(wall_tab, k.wall_inv_step, d).y;
        ax += coef * nx;
        ay += coef * ny;
        az += coef * nz;
        if ((k.flags & kFlagRepulsion) && d < k.r0) {
          float s = 1.0f - fmaxf(d, 0.0f) / k.r0;
          float fm = k.sdf_coef * s * s / k.r0;
          ax += fm * nx;
          ay += fm * ny;
          az += fm * nz;
        }
      }
    }
    if ((k.flags & kFlagRepulsion) && b1 > b0) {
      auto rterm = [&](const float4& bp) {
        float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
        float d2 = dx * dx + dy * dy + dz * dz;
        if (d2 <= k.r0_d2 && d2 > k.tiny_d2) {
          float r = sqrtf(d2);
          float s = 1.0f - r / k.r0;
          float force_mag = k.rep_d * s * s / k.r0;
          float inv_r = 1.0f / r;
          ax += force_mag * dx * inv_r;
          ay += force_mag * dy * inv_r;
          az += force_mag * dz * inv_r;
        }
      };
      uint32_t q = b0;
      for (; q + 1 < b1; q += 2) {
        uint32_t i0 = __ldg(&bc_list[q]), i1 = __ldg(&bc_list[q + 1]);
        float4 bp0 = __ldg(&bpos[i0]), bp1 = __ldg(&bpos[i1]);
        rterm(bp0);
        rterm(bp1);
      }
      if (q < b1) rterm(__ldg(&bpos[__ldg(&bc_list[q])]));
    }
    if (CL) {  // learned near-wall correction (the density kernel's network epilogue)
      float4 cr = corr[i];
      if (cr.w != 0.0f) { ax += cr.x; ay += cr.y; az += cr.z; }
    }
    float vx = vi.x + ax * hdt, vy = vi.y + ay * hdt, vz = vi.z + az * hdt;
    acc[i] = make_float4(ax, ay, az, 0.0f);
    velout[i] = make_float4(vx, vy, vz, rho_i);
    float v = sqrtf(vx * vx + vy * vy + vz * vz);
    sig = v + k.c;
    amag = sqrtf(ax * ax + ay * ay + az * az);
    if (!(sig >= 0.0f)) sig = 0.0f;    // NaN never wins (sph.rs:606)
    if (!(amag >= 0.0f)) amag = 0.0f;  // (sph.rs:613)
  }
  // per-instance maxima: a warp whose lanes share one instance reduces with
  // shuffles and issues one atomic pair; a mixed warp issues per lane
  int inst0 = __shfl_sync(0xffffffffu, inst, 0);
  bool uniform = __all_sync(0xffffffffu, inst == inst0 || inst < 0);
  if (uniform) {
    for (int o = 16; o > 0; o >>= 1) {
      sig = fmaxf(sig, __shfl_xor_sync(0xffffffffu, sig, o));
      amag = fmaxf(amag, __shfl_xor_sync(0xffffffffu, amag, o));
    }
    if ((threadIdx.x & 31) == 0 && inst0 >= 0) {
      atomic_max_pos(&red[2 * inst0], sig);
      atomic_max_pos(&red[2 * inst0 + 1], amag);
    }
  } else if (inst >= 0) {
    atomic_max_pos(&red[2 * inst], sig);
    atomic_max_pos(&red[2 * inst + 1], amag);
  }
}

// dt reduction over an arbitrary state (creation, restore): same maxima as
// the k_forces epilogue.
template <class KP>
__global__ void k_timestep_reduce(KP kp, int n, const float4* __restrict__ velout,
                                  const float4* __restrict__ acc, float* __restrict__ red) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SimConst& k = kp.at(i);
  float4 v = velout[i];
  float4 a = acc[i];
  float sig = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) + k.c;
  float amag = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
  if (sig >= 0.0f) atomic_max_pos(&red[2 * k.inst], sig);
  if (amag >= 0.0f) atomic_max_pos(&red[2 * k.inst + 1], amag);
}

// sph.rs:591-628 from the reduced maxima.
// Per instance (h, c, cfl in hcc[q]): dt = compute_timestep from its maxima.
__global__ void k_dt_finalize(int ninst, const float4* __restrict__ hcc, const float* __restrict__ red,
                              float* __restrict__ dt_out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ninst; q += gridDim.x * blockDim.x) {
    float4 p = hcc[q];
    float h = p.x, c = p.y, cfl = p.z;
    float max_signal = fmaxf(c, red[2 * q]);
    float max_accel = red[2 * q + 1];
    float dt_cfl = cfl * h / max_signal;
    float dt_force = max_accel > 1.0e-12f ? 0.25f * sqrtf(h / max_accel) : 0.01f;
    float dt = fminf(dt_cfl, dt_force);
    dt_out[q] = fminf(fmaxf(dt, 1.0e-8f), 0.01f);
  }
}

// ---- readback / metrics / checkpoint -------------------------------------

// Scatter the sorted state back to original order into 13 planar arrays
// (x..az, density, pressure, mass) + fluid type.
__global__ void k_unsort(int n, const float4* __restrict__ pos, const float4* __restrict__ velout,
                         const float4* __restrict__ acc, const float* __restrict__ pr,
                         const uint32_t* __restrict__ id, float* __restrict__ out,
                         uint8_t* __restrict__ ftype) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t raw = id[s];
  uint32_t o = raw & kIdMask;
  float4 p = pos[s], v = velout[s], a = acc[s];
  size_t N = (size_t)n;
  out[o] = p.x; out[N + o] = p.y; out[2 * N + o] = p.z;
  out[3 * N + o] = v.x; out[4 * N + o] = v.y; out[5 * N + o] = v.z;
  out[6 * N + o] = a.x; out[7 * N + o] = a.y; out[8 * N + o] = a.z;
  out[9 * N + o] = v.w; out[10 * N + o] = pr[s]; out[11 * N + o] = p.w;
  ftype[o] = (raw & kAirBit) ? 1 : 0;
}

// Per-block FP64 partial sums (lib.rs:177-194, 341-370): mass, energy, and
// the f32 maximum density variation.
constexpr int kMetricThreads = 256;
__global__ void __launch_bounds__(kMetricThreads)
k_metrics_partial(SimConst k, int n, const float4* __restrict__ pos, const float4* __restrict__ velout,
                  const uint32_t* __restrict__ id, double* __restrict__ part_m,
                  double* __restrict__ part_e, float* __restrict__ part_var) {
  __shared__ double sm[kMetricThreads], se[kMetricThreads];
  __shared__ float sv[kMetricThreads];
  double m_acc = 0.0, e_acc = 0.0;
  float var_max = 0.0f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = pos[i], v = velout[i];
    double m = (double)p.w;
    double vx = v.x, vy = v.y, vz = v.z;
    e_acc += 0.5 * m * (vx * vx + vy * vy + vz * vz);
    double x = p.x, y = p.y, z = p.z;
    e_acc -= m * ((double)k.grav[0] * x + (double)k.grav[1] * y + (double)k.grav[2] * z);
    m_acc += m;
    float rest = (id[i] & kAirBit) ? kAirRho0 : kWaterRho0;
    float var = fabsf(v.w - rest) / rest;
    if (var > var_max) var_max = var;
  }
  sm[threadIdx.x] = m_acc; se[threadIdx.x] = e_acc; sv[threadIdx.x] = var_max;
  __syncthreads();
  for (int o = kMetricThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sm[threadIdx.x] += sm[threadIdx.x + o];
      se[threadIdx.x] += se[threadIdx.x + o];
      sv[threadIdx.x] = fmaxf(sv[threadIdx.x], sv[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part_m[blockIdx.x] = sm[0]; part_e[blockIdx.x] = se[0]; part_var[blockIdx.x] = sv[0];
  }
}

__global__ void k_metrics_final(int nparts, const double* __restrict__ part_m,
                                const double* __restrict__ part_e, const float* __restrict__ part_var,
                                double* __restrict__ out_me, float* __restrict__ out_var) {
  // one warp: lane l sums partials l, l + 32, ... in order, then a fixed
  // butterfly combines the lanes, so the result does not vary between runs
  int lane = threadIdx.x & 31;
  double m = 0.0, e = 0.0;
  float v = 0.0f;
  for (int b = lane; b < nparts; b += 32) {
    m += part_m[b];
    e += part_e[b];
    v = fmaxf(v, part_var[b]);
  }
  for (int off = 16; off > 0; off >>= 1) {
    m += __shfl_xor_sync(0xffffffffu, m, off);
    e += __shfl_xor_sync(0xffffffffu, e, off);
    v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
  }
  if (lane == 0) {
    out_me[0] = m;
    out_me[1] = e;
    *out_var = v;
  }
}

// Particle records of the viewer's Frame message (server ws.rs:233-290):
// particle o = k * stride (original order, k < count) becomes 20 bytes at
// out + 20 k: x, y, z, temperature (f32), fluid type (u8), density ratio
// (u16, (rho / rho0) * 1000 clamped to [0, 65535] and truncated; NaN gives
// 0 like Rust's saturating cast), a zero byte; little endian, written as
// five aligned words.
__global__ void k_pack_frame(int n, const float4* __restrict__ pos, const float4* __restrict__ velout,
                             const uint32_t* __restrict__ id, const float* __restrict__ temp,
                             uint32_t stride, uint32_t count, uint32_t* __restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t raw = id[s];
  uint32_t o = raw & kIdMask;
  if (o % stride != 0u) return;
  uint32_t q = o / stride;
  if (q >= count) return;
  float4 p = pos[s];
  bool air = (raw & kAirBit) != 0;
  float r = (velout[s].w / (air ? kAirRho0 : kWaterRho0)) * 1000.0f;
  uint32_t ratio = (uint32_t)fminf(fmaxf(r, 0.0f), 65535.0f);
  uint32_t* w = out + (size_t)q * 5;
  w[0] = __float_as_uint(p.x);
  w[1] = __float_as_uint(p.y);
  w[2] = __float_as_uint(p.z);
  w[3] = __float_as_uint(temp[o]);
  w[4] = (air ? 1u : 0u) | (ratio << 8);
}

// ---- optimistic time stepping (orchestrator runner.rs:189-240) ------------
// Per step: dt_safe from the CFL maxima; outside a cooldown try
// dt_safe * alpha with a checkpoint, and if the step left a maximum density
// variation above the limit, restore and redo it with dt_safe, then skip
// the optimism for `cooldown` steps. One graph per step: these kernels keep
// the runner's state on the device and k_opt_decide selects the retry branch
// (a conditional graph node) without a host round trip.
struct RunState {
  double sim_time;
  unsigned long long steps, accepted, rejected;
  float dt_safe, dt_used;
  uint32_t cooldown, reject;
};

__global__ void k_opt_begin(RunState* run, const float* __restrict__ dt_safe, float* __restrict__ dt, float alpha) {
  float ds = *dt_safe;
  float try_dt = run->cooldown > 0u ? ds : ds * alpha;
  run->dt_safe = ds;
  run->dt_used = try_dt;
  *dt = try_dt;
}

__global__ void k_opt_decide(RunState* run, const float* __restrict__ var, float limit, uint32_t cooldown,
                             cudaGraphConditionalHandle retry) {
  uint32_t reject = 0u;
  if (run->cooldown > 0u) {
    run->cooldown -= 1u;
  } else if (*var > limit) {
    reject = 1u;
    run->cooldown = cooldown;
    run->rejected += 1ull;
  } else {
    run->accepted += 1ull;
  }
  if (!reject) run->sim_time += (double)run->dt_used;
  run->steps += 1ull;
  run->reject = reject;
  cudaGraphSetConditional(retry, reject);
}

__global__ void k_opt_retry(RunState* run, float* __restrict__ dt) {
  run->dt_used = run->dt_safe;
  *dt = run->dt_safe;
}

__global__ void k_opt_commit(RunState* run) { run->sim_time += (double)run->dt_used; }

// velocity *= factor (the end-of-step velocity the next step starts from)
__global__ void k_scale_velocities(int n, float4* __restrict__ velout, float factor) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = velout[i];
  velout[i] = make_float4(v.x * factor, v.y * factor, v.z * factor, v.w);
}

// Count of particles with a non-finite position, velocity or density.
__global__ void k_health(int n, const float4* __restrict__ pos, const float4* __restrict__ velout,
                         unsigned long long* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = pos[i], v = velout[i];
  bool ok = isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(v.x) && isfinite(v.y) &&
            isfinite(v.z) && isfinite(v.w);
  if (!ok) atomicAdd(bad, 1ull);
}

// Checkpoint: slot of each original id in the saved copy.
__global__ void k_index_ids(int n, const uint32_t* __restrict__ id, uint32_t* __restrict__ slot_of_id) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) slot_of_id[id[s] & kIdMask] = (uint32_t)s;
}

// Restore into the current slot order (the grid stays the one of the last
// force computation, as the reference keeps its NeighborGrid on restore).
__global__ void k_restore(int n, const uint32_t* __restrict__ id, const uint32_t* __restrict__ ck_slot,
                          const float4* __restrict__ ck_pos, const float4* __restrict__ ck_velout,
                          const float4* __restrict__ ck_acc, const float* __restrict__ ck_pr,
                          float4* __restrict__ pos, float4* __restrict__ velout,
                          float4* __restrict__ acc, float* __restrict__ pr, Planes pl) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t c = ck_slot[id[s] & kIdMask];
  float4 p = ck_pos[c];
  pos[s] = p;
  pl.xyz[s] = p.x;
  pl.xyz[pl.stride + s] = p.y;
  pl.xyz[2 * pl.stride + s] = p.z;
  velout[s] = ck_velout[c];
  acc[s] = ck_acc[c];
  pr[s] = ck_pr[c];
}

// ---- grid diagnostics ---------------------------------------------------

__global__ void k_grid_keys(SimConst k, int n, const float4* __restrict__ pos,
                            const uint32_t* __restrict__ id, uint32_t* __restrict__ lin_out,
                            uint32_t* __restrict__ morton_out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float4 p = pos[s];
  int cx = axis_cell(p.x, k.gmin[0], k.cell, k.dims[0]);
  int cy = axis_cell(p.y, k.gmin[1], k.cell, k.dims[1]);
  int cz = axis_cell(p.z, k.gmin[2], k.cell, k.dims[2]);
  uint32_t o = id[s] & kIdMask;
  lin_out[o] = (uint32_t)cell_hash(cx, cy, cz, k);
  morton_out[o] = morton30((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}

__global__ void k_find_slot(int n, const uint32_t* __restrict__ id, uint32_t want,
                            uint32_t* __restrict__ slot) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && (id[s] & kIdMask) == want) *slot = (uint32_t)s;
}

__global__ void k_list_neighbors(SimConst k, const float4* __restrict__ pos,
                                 const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
                                 const uint32_t* __restrict__ slot, uint32_t* __restrict__ out,
                                 uint32_t cap, uint32_t* __restrict__ count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int i = (int)*slot;
  float4 pi = pos[i];
  uint32_t c = 0;
  for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                    [&](int s, const float4&, float, float, float, float) {
                      if (c < cap) out[c] = id[s] & kIdMask;
                      ++c;
                    });
  *count = c;
}

}  // namespace sph

namespace sph {

// ---- force extraction (orchestrator force.rs:39-129) and body reaction ----

// One warp per surface node: Shepard-averaged fluid pressure (terms sorted by
// particle index, force.rs:88-100), then -p n dA and r x F in f32 as the
// reference computes them (force.rs:103-119). out[node] = (Fx, Fy, Fz, Mx, My,
// Mz) or zeros when no fluid particle is in support.
constexpr int kSurfWarps = 4;
__global__ void __launch_bounds__(kSurfWarps * 32)
k_surface_nodes(SimConst k, int nnodes, const float4* __restrict__ node_pos,
                const float4* __restrict__ node_nrm, float d_area, const float4* __restrict__ pos,
                const float* __restrict__ pr, const uint32_t* __restrict__ id,
                const uint2* __restrict__ ctab, float* __restrict__ out, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_id[kSurfWarps][kAdamiCap];
  __shared__ float s_w[kSurfWarps][kAdamiCap];
  __shared__ float s_wp[kSurfWarps][kAdamiCap];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int nd = blockIdx.x * kSurfWarps + warp;
  if (nd >= nnodes) return;
  float4 np4 = node_pos[nd];
  float c[3] = {np4.x, np4.y, np4.z};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = axis_cell(c[a] - k.reach, k.gmin[a], k.cell, k.dims[a]);
    hi[a] = axis_cell(c[a] + k.reach, k.gmin[a], k.cell, k.dims[a]);
  }
  int count = 0;
  bool overflow = false;
  int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
  int ncell = nx * ny * nz;
  for (int cbase = 0; cbase < ncell; cbase += 32) {
    int q = cbase + lane;
    uint2 mine = make_uint2(0u, 0u);
    if (q < ncell) {
      int qx = q % nx, qy = (q / nx) % ny, qz = q / (nx * ny);
      mine = __ldg(&ctab[cell_hash(lo[0] + qx, lo[1] + qy, lo[2] + qz, k)]);
    }
    unsigned occupied = __ballot_sync(0xffffffffu, mine.y > 0u);
    while (occupied) {
      int src = __ffs(occupied) - 1;
      occupied &= occupied - 1u;
      uint32_t st = __shfl_sync(0xffffffffu, mine.x, src);
      uint32_t cn = __shfl_sync(0xffffffffu, mine.y, src);
      for (uint32_t base = st; base < st + cn; base += 32) {
        uint32_t s = base + lane;
        bool inr = false;
        float w = 0.0f, wp = 0.0f;
        uint32_t fid = 0;
        if (s < st + cn) {
          float4 pf = __ldg(&pos[s]);
          float dx = pf.x - np4.x, dy = pf.y - np4.y, dz = pf.z - np4.z;
          float d2 = dx * dx + dy * dy + dz * dz;
          if (d2 <= k.sup_d2) {
            inr = true;
            w = w_c2(sqrtf(d2), k);
            wp = __ldg(&pr[s]) * w;
            fid = __ldg(&id[s]) & kIdMask;
          }
        }
        unsigned m = __ballot_sync(0xffffffffu, inr);
        int off = count + __popc(m & ((1u << lane) - 1u));
        if (inr) {
          if (off < kAdamiCap) { s_id[warp][off] = fid; s_w[warp][off] = w; s_wp[warp][off] = wp; }
          else overflow = true;
        }
        count += __popc(m);
      }
    }
  }
  if (__any_sync(0xffffffffu, overflow) || count > kAdamiCap) {
    if (lane == 0) atomicOr(err, kErrAdamiCap);
    return;
  }
  int m2 = 1;
  while (m2 < count) m2 <<= 1;
  for (int q = count + lane; q < m2; q += 32) s_id[warp][q] = 0xffffffffu;
  __syncwarp();
  for (int kk = 2; kk <= m2; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < m2; q += 32) {
        int pq = q ^ j;
        if (pq > q) {
          bool up = (q & kk) == 0;
          uint32_t a = s_id[warp][q], cc = s_id[warp][pq];
          if ((a > cc) == up) {
            s_id[warp][q] = cc; s_id[warp][pq] = a;
            float t = s_w[warp][q]; s_w[warp][q] = s_w[warp][pq]; s_w[warp][pq] = t;
            t = s_wp[warp][q]; s_wp[warp][q] = s_wp[warp][pq]; s_wp[warp][pq] = t;
          }
        }
      }
      __syncwarp();
    }
  if (lane == 0) {
    float lp = 0.0f, ws = 0.0f;
    for (int q = 0; q < count; ++q) { lp += s_wp[warp][q]; ws += s_w[warp][q]; }
    float f[6] = {0, 0, 0, 0, 0, 0};
    if (ws > 1e-12f) {
      lp = lp / ws;
      float4 n = node_nrm[nd];
      float fx = -lp * n.x * d_area, fy = -lp * n.y * d_area, fz = -lp * n.z * d_area;
      f[0] = fx; f[1] = fy; f[2] = fz;
      f[3] = np4.y * fz - np4.z * fy;
      f[4] = np4.z * fx - np4.x * fz;
      f[5] = np4.x * fy - np4.y * fx;
    }
    for (int a = 0; a < 6; ++a) out[(size_t)nd * 6 + a] = f[a];
  }
}

// Deterministic FP64 sum of `cols` interleaved columns of f32 rows (one
// block; fixed thread->row assignment and tree order).
__global__ void k_sum_rows_f64(int rows, int cols, const float* __restrict__ in, double* __restrict__ out) {
  __shared__ double sh[256];
  for (int c = 0; c < cols; ++c) {
    double acc = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += (double)in[(size_t)r * cols + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sh[0];
    __syncthreads();
  }
}

// Reaction of the fluid on the boundary particles [b_first, b_first+b_count)
// from the last force computation, per block in FP64: the boundary pressure
// force (sph.rs:391-408) and repulsion (boundary.rs:161-179) the fluid
// receives from them, negated; and the Monaghan viscous force with the body
// at rest (diagnostic; the reference has no wall viscosity). 18 columns:
// pressure F, M; repulsion F, M; viscous F, M (moments about the origin at
// the boundary particle's position).
constexpr int kBodyCols = 18;
__global__ void __launch_bounds__(256)
k_body_force(SimConst k, int n, uint32_t b_first, uint32_t b_count, const float4* __restrict__ pos,
             const float4* __restrict__ vel, const float2* __restrict__ rf, const float* __restrict__ pr,
             const uint32_t* __restrict__ id, const uint32_t* __restrict__ bc_start,
             const uint32_t* __restrict__ bc_list, const float4* __restrict__ bpos,
             const float* __restrict__ bpress, double* __restrict__ part) {
  double acc[kBodyCols];
#pragma unroll
  for (int c = 0; c < kBodyCols; ++c) acc[c] = 0.0;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    float4 pi = pos[i];
    int lin = cell_hash(axis_cell(pi.x, k.gmin[0], k.cell, k.dims[0]),
                        axis_cell(pi.y, k.gmin[1], k.cell, k.dims[1]),
                        axis_cell(pi.z, k.gmin[2], k.cell, k.dims[2]), k);
    uint32_t q0 = bc_start[lin], q1 = bc_start[lin + 1];
    if (q1 > q0) {
      float4 vi = vel[i];
      float2 rfi = rf[i];
      bool air = (id[i] & kAirBit) != 0;
      float rest = air ? kAirRho0 : kWaterRho0;
      float pic_over = fmaxf(pr[i], 0.0f) / (rfi.x * rfi.x);
      for (uint32_t q = q0; q < q1; ++q) {
        uint32_t b = bc_list[q];
        if (b < b_first || b >= b_first + b_count) continue;
        float4 bp = bpos[b];
        float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
        float d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 <= k.sup_d2)) continue;
        float r = sqrtf(d2);
        float gx, gy, gz;
        grad_c2(dx, dy, dz, r, k, gx, gy, gz);
        float factor = -pi.w * bp.w * (pic_over + bpress[b] / (rest * rest));
        double F[3] = {-(double)(factor * gx), -(double)(factor * gy), -(double)(factor * gz)};
        double R[3] = {0.0, 0.0, 0.0};
        if (d2 <= k.r0_d2 && d2 > k.tiny_d2) {
          float s = 1.0f - r / k.r0;
          float fm = k.rep_d * s * s / k.r0;
          float inv_r = 1.0f / r;
          R[0] = -(double)pi.w * (double)(fm * dx * inv_r);
          R[1] = -(double)pi.w * (double)(fm * dy * inv_r);
          R[2] = -(double)pi.w * (double)(fm * dz * inv_r);
        }
        double V[3] = {0.0, 0.0, 0.0};
        float vr = vi.x * dx + vi.y * dy + vi.z * dz;
        if (vr < 0.0f) {
          float mu = k.h * vr / (r * r + k.eta_sq);
          float pij = (k.neg_alpha_c * mu + k.beta * mu * mu) / (0.5f * (rfi.x + rest));
          float fv = -pi.w * bp.w * pij;
          V[0] = -(double)(fv * gx); V[1] = -(double)(fv * gy); V[2] = -(double)(fv * gz);
        }
        double X[3] = {bp.x, bp.y, bp.z};
        const double* G[3] = {F, R, V};
        for (int t = 0; t < 3; ++t) {
          acc[6 * t + 0] += G[t][0]; acc[6 * t + 1] += G[t][1]; acc[6 * t + 2] += G[t][2];
          acc[6 * t + 3] += X[1] * G[t][2] - X[2] * G[t][1];
          acc[6 * t + 4] += X[2] * G[t][0] - X[0] * G[t][2];
          acc[6 * t + 5] += X[0] * G[t][1] - X[1] * G[t][0];
        }
      }
    }
  }
  __shared__ double sh[256];
  for (int c = 0; c < kBodyCols; ++c) {
    sh[threadIdx.x] = acc[c];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * kBodyCols + c] = sh[0];
    __syncthreads();
  }
}

__global__ void k_sum_parts_f64(int parts, int cols, const double* __restrict__ in, double* __restrict__ out) {
  int c = threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int p = 0; p < parts; ++p) s += in[(size_t)p * cols + c];
  out[c] = s;
}

}  // namespace sph

namespace sph {

// Shepard interpolation of the fluid state at arbitrary points (a fine run
// sampled where coarse particles are): out[q] = (rho, p, ax, ay, az, wsum, n).
template <class KP>
__global__ void k_interpolate(KP kp, int npts, const float4* __restrict__ pts, const float4* __restrict__ pos,
                              const float2* __restrict__ rf, const float* __restrict__ pr,
                              const float4* __restrict__ acc, const uint2* __restrict__ ctab,
                              float* __restrict__ out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const SimConst& k = kp.at(0);
  float4 x = pts[q];
  float c3[3] = {x.x, x.y, x.z};
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = axis_cell(c3[a] - k.reach, k.gmin[a], k.cell, k.dims[a]);
    hi[a] = axis_cell(c3[a] + k.reach, k.gmin[a], k.cell, k.dims[a]);
  }
  double ws = 0.0, sr = 0.0, sp = 0.0, sa[3] = {0.0, 0.0, 0.0};
  int cnt = 0;
  for (int cz = lo[2]; cz <= hi[2]; ++cz)
    for (int cy = lo[1]; cy <= hi[1]; ++cy)
      for (int cx = lo[0]; cx <= hi[0]; ++cx) {
        uint2 se = ctab[k.coff + cell_hash(cx, cy, cz, k)];
        for (uint32_t s = se.x; s < se.x + se.y; ++s) {
          float4 pj = pos[s];
          float dx = x.x - pj.x, dy = x.y - pj.y, dz = x.z - pj.z;
          float d2 = dx * dx + dy * dy + dz * dz;
          if (!(d2 <= k.sup_d2)) continue;
          double w = (double)w_c2(sqrtf(d2), k);
          float4 a = acc[s];
          ws += w; sr += w * rf[s].x; sp += w * pr[s];
          sa[0] += w * a.x; sa[1] += w * a.y; sa[2] += w * a.z;
          ++cnt;
        }
      }
  float* o = out + (size_t)q * 7;
  double iw = ws > 0.0 ? 1.0 / ws : 0.0;
  o[0] = (float)(sr * iw); o[1] = (float)(sp * iw);
  o[2] = (float)(sa[0] * iw); o[3] = (float)(sa[1] * iw); o[4] = (float)(sa[2] * iw);
  o[5] = (float)ws; o[6] = (float)cnt;
}

}  // namespace sph
