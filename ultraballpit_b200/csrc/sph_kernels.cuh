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
#include <cstdint>
#include <cuda_runtime.h>

namespace sph {

constexpr uint32_t kIdMask = 0x7fffffffu;
constexpr uint32_t kAirBit = 0x80000000u;
constexpr float kWaterRho0 = 1000.0f;  // eos.rs:7
constexpr float kAirRho0 = 1.204f;     // eos.rs:10
constexpr int kAdamiCap = 256;         // fluid terms per boundary particle
constexpr int kCellCap = 4096;         // particles per cell for the id ranking

enum : uint32_t { kFlagDelta = 1, kFlagXsph = 2, kFlagRepulsion = 4, kFlagClamp = 8 };
enum : uint32_t { kErrCellCap = 1, kErrAdamiCap = 2 };

// Step constants, each rounded in f32 exactly as the reference evaluates it.
struct SimConst {
  float h, support, radius_sq, cell;
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

// sph.rs:35-46 with NORM/h^3 precomputed (same rounding).
__device__ __forceinline__ float w_c2(float r, const SimConst& k) {
  float q = r / k.h;
  if (q >= 2.0f) return 0.0f;
  float omq = 1.0f - 0.5f * q;
  float t = omq * omq;
  float t4 = t * t;
  return k.norm_h3 * t4 * (1.0f + 2.0f * q);
}

// sph.rs:68-85
__device__ __forceinline__ void grad_c2(float dx, float dy, float dz, float r, const SimConst& k,
                                        float& gx, float& gy, float& gz) {
  float q = r / k.h;
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
  for (int dz = -1; dz <= 1; ++dz) {
    int nz = cz + dz;
    if (nz < 0 || nz >= k.dims[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      int ny = cy + dy;
      if (ny < 0 || ny >= k.dims[1]) continue;
      int row = (ny + nz * k.dims[1]) * k.dims[0];
      for (int dx = -1; dx <= 1; ++dx) {
        int nx = cx + dx;
        if (nx < 0 || nx >= k.dims[0]) continue;
        uint2 se = __ldg(&ctab[row + nx]);
        int end = (int)(se.x + se.y);
        for (int s = (int)se.x; s < end; ++s) {
          if (s == self) continue;
          float4 pj = __ldg(&pos[s]);
          float ddx = px - pj.x, ddy = py - pj.y, ddz = pz - pj.z;
          float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (d2 <= k.radius_sq) f(s, pj, ddx, ddy, ddz, d2);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

__global__ void k_set_dt(float* dt, float value) { *dt = value; }

// Kick 1 (lib.rs:301-305) + XSPH (sph.rs:236-280) + drift (lib.rs:313-317)
// + domain clamp (boundary.rs:239-291) + binning of the new position
// (neighbor.rs:89-101) into a rank-indexed histogram. Reads the sorted state,
// writes the unsorted "U" arrays in the same slot order.
__global__ void __launch_bounds__(256)
k_xsph_drift(SimConst k, int n, const float* __restrict__ dtp, const float4* __restrict__ pos,
             const float4* __restrict__ velout, const float4* __restrict__ acc,
             const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
             const uint32_t* __restrict__ rank_of_lin, float4* __restrict__ posU,
             float4* __restrict__ velU, uint32_t* __restrict__ idU, uint32_t* __restrict__ keyU,
             uint32_t* __restrict__ hist, const uint32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || *err) return;
  float dt = *dtp;
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
    for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                      [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
                        float r = sqrtf(d2);
                        float w = w_c2(r, k);
                        float4 vj = __ldg(&velout[s]);
                        float4 aj = __ldg(&acc[s]);
                        float vjx = vj.x + aj.x * hdt;
                        float vjy = vj.y + aj.y * hdt;
                        float vjz = vj.z + aj.z * hdt;
                        float rho_avg = 0.5f * (rho_i + vj.w);
                        float factor = pj.w / fmaxf(rho_avg, 1.0f) * w;
                        sx += factor * (vjx - vx);
                        sy += factor * (vjy - vy);
                        sz += factor * (vjz - vz);
                      });
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
  uint32_t r = __ldg(&rank_of_lin[lin]);
  keyU[i] = r;
  atomicAdd(&hist[r], 1u);
}

// Binning of an unsorted state (creation, bootstrap) without moving it.
__global__ void k_bin(SimConst k, int n, const float4* __restrict__ posU,
                      const uint32_t* __restrict__ rank_of_lin, uint32_t* __restrict__ keyU,
                      uint32_t* __restrict__ hist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = posU[i];
  int lin = cell_hash(axis_cell(p.x, k.gmin[0], k.cell, k.dims[0]),
                      axis_cell(p.y, k.gmin[1], k.cell, k.dims[1]),
                      axis_cell(p.z, k.gmin[2], k.cell, k.dims[2]), k);
  uint32_t r = __ldg(&rank_of_lin[lin]);
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
          const float* __restrict__ prU, float* __restrict__ pr, float4* __restrict__ velout) {
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
__global__ void __launch_bounds__(256)
k_density(SimConst k, int n, const float* __restrict__ dtp, const float4* __restrict__ pos,
          const float2* __restrict__ rv, const uint32_t* __restrict__ id,
          const uint2* __restrict__ ctab, const uint32_t* __restrict__ bc_start,
          const uint32_t* __restrict__ bc_list, const float4* __restrict__ bpos,
          float2* __restrict__ rf, float* __restrict__ pr, const uint32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || *err) return;
  float dt = *dtp;
  float4 pi = pos[i];
  float rho_old_i = rv[i].x;
  float rho = pi.w * k.norm_h3;
  float diff_sum = 0.0f;
  bool delta = (k.flags & kFlagDelta) != 0;
  for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                    [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
                      float r = sqrtf(d2);
                      if (delta) {
                        float gx, gy, gz;
                        grad_c2(dx, dy, dz, r, k, gx, gy, gz);
                        float2 rvj = __ldg(&rv[s]);
                        float r_dot_grad = dx * gx + dy * gy + dz * gz;
                        float density_diff = rho_old_i - rvj.x;
                        diff_sum += rvj.y * density_diff * 2.0f * r_dot_grad / (d2 + k.eta_sq);
                      }
                      rho += pj.w * w_c2(r, k);
                    });
  int lin = cell_hash(axis_cell(pi.x, k.gmin[0], k.cell, k.dims[0]),
                      axis_cell(pi.y, k.gmin[1], k.cell, k.dims[1]),
                      axis_cell(pi.z, k.gmin[2], k.cell, k.dims[2]), k);
  uint32_t b0 = __ldg(&bc_start[lin]), b1 = __ldg(&bc_start[lin + 1]);
  for (uint32_t q = b0; q < b1; ++q) {
    float4 bp = __ldg(&bpos[__ldg(&bc_list[q])]);
    float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
    float r = sqrtf(dx * dx + dy * dy + dz * dz);
    if (r < k.support) rho += bp.w * w_c2(r, k);
  }
  if (delta) {
    float diffusion = k.delta_coef * diff_sum;
    rho += diffusion * dt;
  }
  bool air = (id[i] & kAirBit) != 0;
  float p = tait(rho, air, k);
  rf[i] = make_float2(rho, p / (rho * rho));
  pr[i] = p;
}

// Adami boundary pressure (boundary.rs:87-131). One warp per boundary
// particle: the lanes evaluate the in-support fluid terms of a widened cell
// range, a warp bitonic sort orders them by fluid index, and lane 0 sums
// them in that order.
constexpr int kAdamiWarps = 4;
__global__ void __launch_bounds__(kAdamiWarps * 32)
k_adami(SimConst k, int nb, const float4* __restrict__ bpos, float* __restrict__ bpress,
        const float4* __restrict__ pos, const float2* __restrict__ rf, const float* __restrict__ pr,
        const uint32_t* __restrict__ id, const uint2* __restrict__ ctab, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_id[kAdamiWarps][kAdamiCap];
  __shared__ float s_w[kAdamiWarps][kAdamiCap];
  __shared__ float s_wp[kAdamiWarps][kAdamiCap];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int b = blockIdx.x * kAdamiWarps + warp;
  if (b >= nb || *err) return;
  float4 bp = bpos[b];
  int lo[3], hi[3];
  float bc[3] = {bp.x, bp.y, bp.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = axis_cell(bc[a] - k.reach, k.gmin[a], k.cell, k.dims[a]);
    hi[a] = axis_cell(bc[a] + k.reach, k.gmin[a], k.cell, k.dims[a]);
  }
  int count = 0;
  bool overflow = false;
  for (int cz = lo[2]; cz <= hi[2]; ++cz)
    for (int cy = lo[1]; cy <= hi[1]; ++cy)
      for (int cx = lo[0]; cx <= hi[0]; ++cx) {
        uint2 se = __ldg(&ctab[cell_hash(cx, cy, cz, k)]);
        for (uint32_t base = se.x; base < se.x + se.y; base += 32) {
          uint32_t s = base + lane;
          bool inr = false;
          float w = 0.0f, wp = 0.0f;
          uint32_t fid = 0;
          if (s < se.x + se.y) {
            float4 pf = __ldg(&pos[s]);
            float dx = bp.x - pf.x, dy = bp.y - pf.y, dz = bp.z - pf.z;
            float r = sqrtf(dx * dx + dy * dy + dz * dz);
            if (r < k.support) {
              inr = true;
              w = w_c2(r, k);
              float g_dot_dr = k.grav[0] * dx + k.grav[1] * dy + k.grav[2] * dz;
              float p_ext = __ldg(&pr[s]) + __ldg(&rf[s]).x * g_dot_dr;
              wp = w * p_ext;
              fid = __ldg(&id[s]) & kIdMask;
            }
          }
          unsigned m = __ballot_sync(0xffffffffu, inr);
          int off = count + __popc(m & ((1u << lane) - 1u));
          if (inr) {
            if (off < kAdamiCap) {
              s_id[warp][off] = fid;
              s_w[warp][off] = w;
              s_wp[warp][off] = wp;
            } else {
              overflow = true;
            }
          }
          count += __popc(m);
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
  for (int kk = 2; kk <= m2; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < m2; q += 32) {
        int pq = q ^ j;
        if (pq > q) {
          bool up = (q & kk) == 0;
          uint32_t a = s_id[warp][q], c = s_id[warp][pq];
          if ((a > c) == up) {
            s_id[warp][q] = c; s_id[warp][pq] = a;
            float t = s_w[warp][q]; s_w[warp][q] = s_w[warp][pq]; s_w[warp][pq] = t;
            t = s_wp[warp][q]; s_wp[warp][q] = s_wp[warp][pq]; s_wp[warp][pq] = t;
          }
        }
      }
      __syncwarp();
    }
  }
  if (lane == 0) {
    float weighted_pressure = 0.0f, weight_sum = 0.0f;
    for (int q = 0; q < count; ++q) {
      weighted_pressure += s_wp[warp][q];
      weight_sum += s_w[warp][q];
    }
    bpress[b] = weight_sum > 1.0e-12f ? fmaxf(weighted_pressure / weight_sum, 0.0f) : 0.0f;
  }
}

// Pressure force + Monaghan viscosity + gravity + boundary pressure force +
// repulsion (lib.rs:247-282; sph.rs:322-508; boundary.rs:143-181), then
// kick 2 (lib.rs:330-334) and the dt reduction inputs (sph.rs:597-616).
__global__ void __launch_bounds__(256)
k_forces(SimConst k, int n, const float* __restrict__ dtp, float hdt_scale,
         const float4* __restrict__ pos, const float4* __restrict__ vel,
         const float2* __restrict__ rf, const float* __restrict__ pr,
         const uint32_t* __restrict__ id, const uint2* __restrict__ ctab,
         const uint32_t* __restrict__ bc_start, const uint32_t* __restrict__ bc_list,
         const float4* __restrict__ bpos, const float* __restrict__ bpress,
         float4* __restrict__ acc, float4* __restrict__ velout, float* __restrict__ red,
         const uint32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float sig = 0.0f, amag = 0.0f;
  if (i < n && !*err) {
    float hdt = (0.5f * *dtp) * hdt_scale;
    float4 pi = pos[i];
    float4 vi = vel[i];
    float2 rfi = rf[i];
    float rho_i = rfi.x;
    float fpx = 0.0f, fpy = 0.0f, fpz = 0.0f;
    float fvx = 0.0f, fvy = 0.0f, fvz = 0.0f;
    float neg_mi = -pi.w;
    for_each_neighbor(pi.x, pi.y, pi.z, i, pos, ctab, k,
                      [&](int s, const float4& pj, float dx, float dy, float dz, float d2) {
                        float r = sqrtf(d2);
                        float gx, gy, gz;
                        grad_c2(dx, dy, dz, r, k, gx, gy, gz);
                        float2 rfj = __ldg(&rf[s]);
                        float factor = neg_mi * pj.w * (rfi.y + rfj.y);
                        fpx += factor * gx;
                        fpy += factor * gy;
                        fpz += factor * gz;
                        float4 vj = __ldg(&vel[s]);
                        float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
                        float vr_dot = dvx * dx + dvy * dy + dvz * dz;
                        if (vr_dot < 0.0f) {
                          float r_sq = r * r;
                          float mu = k.h * vr_dot / (r_sq + k.eta_sq);
                          float rho_avg = 0.5f * (rho_i + rfj.x);
                          float pi_ij = (k.neg_alpha_c * mu + k.beta * mu * mu) / rho_avg;
                          float fv = -pj.w * pi_ij;
                          fvx += fv * gx;
                          fvy += fv * gy;
                          fvz += fv * gz;
                        }
                      });
    int lin = cell_hash(axis_cell(pi.x, k.gmin[0], k.cell, k.dims[0]),
                        axis_cell(pi.y, k.gmin[1], k.cell, k.dims[1]),
                        axis_cell(pi.z, k.gmin[2], k.cell, k.dims[2]), k);
    uint32_t b0 = __ldg(&bc_start[lin]), b1 = __ldg(&bc_start[lin + 1]);
    bool air = (id[i] & kAirBit) != 0;
    if (b1 > b0) {
      float pic = fmaxf(pr[i], 0.0f);
      float pic_over = pic / (rho_i * rho_i);
      float brho = air ? kAirRho0 : kWaterRho0;
      float brho2 = brho * brho;
      for (uint32_t q = b0; q < b1; ++q) {
        uint32_t bi = __ldg(&bc_list[q]);
        float4 bp = __ldg(&bpos[bi]);
        float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < k.support) {
          float gx, gy, gz;
          grad_c2(dx, dy, dz, r, k, gx, gy, gz);
          float pb_over = __ldg(&bpress[bi]) / brho2;
          float factor = neg_mi * bp.w * (pic_over + pb_over);
          fpx += factor * gx;
          fpy += factor * gy;
          fpz += factor * gz;
        }
      }
    }
    float ax = 0.0f + fpx / pi.w, ay = 0.0f + fpy / pi.w, az = 0.0f + fpz / pi.w;
    ax += fvx; ay += fvy; az += fvz;
    ax += k.grav[0]; ay += k.grav[1]; az += k.grav[2];
    if ((k.flags & kFlagRepulsion) && b1 > b0) {
      for (uint32_t q = b0; q < b1; ++q) {
        float4 bp = __ldg(&bpos[__ldg(&bc_list[q])]);
        float dx = pi.x - bp.x, dy = pi.y - bp.y, dz = pi.z - bp.z;
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < k.r0 && r > 1.0e-12f) {
          float s = 1.0f - r / k.r0;
          float force_mag = k.rep_d * s * s / k.r0;
          float inv_r = 1.0f / r;
          ax += force_mag * dx * inv_r;
          ay += force_mag * dy * inv_r;
          az += force_mag * dz * inv_r;
        }
      }
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
  // block max, one atomic per block
  for (int o = 16; o > 0; o >>= 1) {
    sig = fmaxf(sig, __shfl_xor_sync(0xffffffffu, sig, o));
    amag = fmaxf(amag, __shfl_xor_sync(0xffffffffu, amag, o));
  }
  __shared__ float s_sig[8], s_a[8];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_sig[wid] = sig; s_a[wid] = amag; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = s_sig[0], b = s_a[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { a = fmaxf(a, s_sig[w]); b = fmaxf(b, s_a[w]); }
    atomic_max_pos(&red[0], a);
    atomic_max_pos(&red[1], b);
  }
}

// dt reduction over an arbitrary state (creation, restore): same maxima as
// the k_forces epilogue.
__global__ void k_timestep_reduce(SimConst k, int n, const float4* __restrict__ velout,
                                  const float4* __restrict__ acc, float* __restrict__ red) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float sig = 0.0f, amag = 0.0f;
  if (i < n) {
    float4 v = velout[i];
    float4 a = acc[i];
    sig = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) + k.c;
    amag = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    if (!(sig >= 0.0f)) sig = 0.0f;
    if (!(amag >= 0.0f)) amag = 0.0f;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sig = fmaxf(sig, __shfl_xor_sync(0xffffffffu, sig, o));
    amag = fmaxf(amag, __shfl_xor_sync(0xffffffffu, amag, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&red[0], sig);
    atomic_max_pos(&red[1], amag);
  }
}

// sph.rs:591-628 from the reduced maxima.
__global__ void k_dt_finalize(float h, float c, float cfl, const float* __restrict__ red,
                              float* __restrict__ dt_out) {
  float max_signal = fmaxf(c, red[0]);
  float max_accel = red[1];
  float dt_cfl = cfl * h / max_signal;
  float dt_force = max_accel > 1.0e-12f ? 0.25f * sqrtf(h / max_accel) : 0.01f;
  float dt = fminf(dt_cfl, dt_force);
  *dt_out = fminf(fmaxf(dt, 1.0e-8f), 0.01f);
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
  if (threadIdx.x != 0) return;
  double m = 0.0, e = 0.0;
  float v = 0.0f;
  for (int b = 0; b < nparts; ++b) {
    m += part_m[b]; e += part_e[b];
    if (part_var[b] > v) v = part_var[b];
  }
  out_me[0] = m; out_me[1] = e; *out_var = v;
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
                          float4* __restrict__ acc, float* __restrict__ pr) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t c = ck_slot[id[s] & kIdMask];
  pos[s] = ck_pos[c];
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
