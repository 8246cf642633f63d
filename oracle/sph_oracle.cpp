// CPU oracle for the WCSPH step: a restatement of the reference Rust CPU path
// (tim-ai-twin/ultraballpit, crate `kernel`).
//
// TEST INFRASTRUCTURE ONLY. The product (libsph_cuda.so) never links, loads or
// calls this file. It is used by tests/, by __graft_entry__.smoke() and by the
// cpu_baseline / reference legs of bench.py, and only as the checker or as the
// timed CPU baseline.
//
// Parity pin: the Rust reference cannot be compiled in this image (no cargo or
// rustc), so this restatement is pinned against the reference's own
// known-answer tests (sph.rs:634-722, eos.rs:70-94, neighbor.rs:185-269,
// tests/two_particle.rs, tests/kernel_normalization.rs, tests/hydrostatic.rs,
// orchestrator geometry.rs:188-250). tests/test_oracle_kat.py runs them.
//
// Build: -O2 -ffp-contract=off -fno-fast-math (no FMA contraction, IEEE f32
// arithmetic in source order, like rustc which never contracts a*b+c).
//
// Two tiers share every formula:
//   Tier L (literal): the boundary loops are the reference's O(N*N_b) scans.
//   Tier G (grid): the same sums, visiting boundary candidates in ascending
//     boundary index through static per-cell candidate lists, and the Adami
//     fluid candidates through the fluid grid sorted by fluid index. Each
//     candidate set is a provable superset of the in-support set, so the
//     sums are identical to Tier L term for term.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <atomic>
#include <thread>

namespace {

// Dynamic-schedule parallel loop over [0, n) on `threads` std::threads. Each
// index is processed by exactly one thread with the same arithmetic as a
// serial loop, so results do not depend on the thread count.
template <class F>
void parallel_for(size_t n, int threads, size_t chunk, F&& body) {
  if (threads <= 1 || n <= chunk) {
    for (size_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<size_t> next(0);
  auto worker = [&]() {
    for (;;) {
      size_t s = next.fetch_add(chunk);
      if (s >= n) break;
      size_t e = std::min(n, s + chunk);
      for (size_t i = s; i < e; ++i) body(i);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
}

// std::f32::consts::PI
constexpr float kPi = 3.14159265358979323846f;
// sph.rs:20  WENDLAND_C2_NORM_3D = 21 / (16 pi), evaluated in f32.
const float kNorm = 21.0f / (16.0f * kPi);
// sph.rs:93  DELTA_SPH; sph.rs:224 XSPH_EPSILON
constexpr float kDeltaSph = 0.1f;
constexpr float kXsphEps = 0.5f;
// eos.rs:7-22
constexpr float kWaterRho0 = 1000.0f;
constexpr float kAirRho0 = 1.204f;
constexpr float kWaterGamma = 7.0f;
constexpr float kAirGamma = 1.4f;
// sph.rs:579-581
constexpr float kMinDt = 1.0e-8f;
constexpr float kMaxDt = 0.01f;

// sph.rs:35-46
inline float wendland_c2(float r, float h) {
  float q = r / h;
  if (q >= 2.0f) return 0.0f;
  float h3 = h * h * h;
  float omq = 1.0f - 0.5f * q;
  float t = omq * omq;
  float t4 = t * t;
  return kNorm / h3 * t4 * (1.0f + 2.0f * q);
}

// sph.rs:68-85
inline void wendland_c2_gradient(float dx, float dy, float dz, float r, float h,
                                 float* gx, float* gy, float* gz) {
  float q = r / h;
  if (q >= 2.0f || r < 1.0e-12f) {
    *gx = 0.0f; *gy = 0.0f; *gz = 0.0f;
    return;
  }
  float h3 = h * h * h;
  float omq = 1.0f - 0.5f * q;
  float t3 = omq * omq * omq;
  float dw_dr = kNorm / (h3 * h) * (-5.0f * q) * t3;
  float inv_r = 1.0f / r;
  *gx = dw_dr * dx * inv_r;
  *gy = dw_dr * dy * inv_r;
  *gz = dw_dr * dz * inv_r;
}

// Power used by the Tait EOS. pow_mode 0 calls the platform libm powf, which
// is what f32::powf lowers to on Linux (glibc; not correctly rounded in about
// 0.07% of inputs near 1). pow_mode 1 returns the correctly rounded x^gamma:
// for gamma = 7 a double-precision product (exact to well inside half an f32
// ulp, checked exhaustively against long double on [0.5, 2]), otherwise the
// double pow rounded to f32. The CUDA step implements pow_mode 1.
inline float eos_pow(float x, float gamma, int pow_mode) {
  if (pow_mode == 0) return powf(x, gamma);
  if (gamma == 7.0f) {
    double r = x, r2 = r * r, r4 = r2 * r2, r6 = r4 * r2;
    return (float)(r6 * r);
  }
  return (float)pow((double)x, (double)gamma);
}

// eos.rs:39-47
inline float tait_eos(float density, float rest_density, float c, float gamma, int pow_mode = 0) {
  float b = rest_density * c * c / gamma;
  float ratio = density / rest_density;
  float p = b * (eos_pow(ratio, gamma, pow_mode) - 1.0f);
  return fmaxf(p, 0.0f);
}

struct Particles {  // particle.rs:22-58 (SoA)
  std::vector<float> x, y, z, vx, vy, vz, ax, ay, az, density, pressure, mass,
      temperature;
  std::vector<uint8_t> fluid_type;  // 0 = Water, 1 = Air
  size_t len() const { return x.size(); }
  std::vector<float>* field(int k) {
    std::vector<float>* f[13] = {&x, &y, &z, &vx, &vy, &vz, &ax, &ay, &az,
                                 &density, &pressure, &mass, &temperature};
    return f[k];
  }
};

// neighbor.rs:11-183
struct NeighborGrid {
  float cell_size;
  float grid_min[3];
  uint32_t dims[3];
  std::vector<uint32_t> cell_indices, sorted_indices, cell_offsets, cell_counts;

  NeighborGrid() = default;
  // neighbor.rs:29-46
  NeighborGrid(float cs, const float mn[3], const float mx[3]) : cell_size(cs) {
    for (int k = 0; k < 3; ++k) {
      grid_min[k] = mn[k];
      dims[k] = (uint32_t)fmaxf(ceilf((mx[k] - mn[k]) / cs), 1.0f);
    }
    cell_offsets.assign(total_cells(), 0);
    cell_counts.assign(total_cells(), 0);
  }
  size_t total_cells() const { return (size_t)dims[0] * dims[1] * dims[2]; }
  // neighbor.rs:57-71
  inline uint32_t axis_cell(float p, int k) const {
    float f = floorf((p - grid_min[k]) / cell_size);
    f = fmaxf(f, 0.0f);
    f = fminf(f, (float)(dims[k] - 1));
    return (uint32_t)f;
  }
  inline void pos_to_cell(float px, float py, float pz, uint32_t* cx, uint32_t* cy,
                          uint32_t* cz) const {
    *cx = axis_cell(px, 0);
    *cy = axis_cell(py, 1);
    *cz = axis_cell(pz, 2);
  }
  // neighbor.rs:75-77
  inline uint32_t cell_hash(uint32_t cx, uint32_t cy, uint32_t cz) const {
    return cx + cy * dims[0] + cz * dims[0] * dims[1];
  }
  // neighbor.rs:82-122: keys, count, exclusive scan, stable scatter.
  void update(const float* x, const float* y, const float* z, size_t n) {
    size_t tc = total_cells();
    cell_indices.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
      uint32_t cx, cy, cz;
      pos_to_cell(x[i], y[i], z[i], &cx, &cy, &cz);
      cell_indices[i] = cell_hash(cx, cy, cz);
    }
    cell_counts.assign(tc, 0);
    for (size_t i = 0; i < n; ++i) cell_counts[cell_indices[i]] += 1;
    cell_offsets.assign(tc, 0);
    uint32_t running = 0;
    for (size_t c = 0; c < tc; ++c) {
      cell_offsets[c] = running;
      running += cell_counts[c];
    }
    sorted_indices.assign(n, 0);
    std::vector<uint32_t> heads(cell_offsets);
    for (size_t i = 0; i < n; ++i) {
      uint32_t ci = cell_indices[i];
      sorted_indices[heads[ci]] = (uint32_t)i;
      heads[ci] += 1;
    }
  }
  // neighbor.rs:129-182: 27 cells, dz -> dy -> dx, skip self, dist_sq <= r^2.
  template <class F>
  inline void for_each_neighbor(size_t pi, const float* x, const float* y,
                                const float* z, float radius, F&& f) const {
    float px = x[pi], py = y[pi], pz = z[pi];
    uint32_t cx, cy, cz;
    pos_to_cell(px, py, pz, &cx, &cy, &cz);
    float radius_sq = radius * radius;
    for (int dz = -1; dz <= 1; ++dz) {
      int nz = (int)cz + dz;
      if (nz < 0 || nz >= (int)dims[2]) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int ny = (int)cy + dy;
        if (ny < 0 || ny >= (int)dims[1]) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          int nx = (int)cx + dx;
          if (nx < 0 || nx >= (int)dims[0]) continue;
          uint32_t cell = cell_hash((uint32_t)nx, (uint32_t)ny, (uint32_t)nz);
          uint32_t start = cell_offsets[cell], count = cell_counts[cell];
          for (uint32_t s = start; s < start + count; ++s) {
            uint32_t j = sorted_indices[s];
            if (j == pi) continue;
            float ddx = px - x[j], ddy = py - y[j], ddz = pz - z[j];
            float dist_sq = ddx * ddx + ddy * ddy + ddz * ddz;
            if (dist_sq <= radius_sq) f((size_t)j);
          }
        }
      }
    }
  }
};

struct Boundary {  // boundary.rs:20-37
  std::vector<float> x, y, z, mass, nx, ny, nz, pressure;
  size_t len() const { return x.size(); }
};

// Morton interleave of three 10-bit cell coordinates (x in bit 0).
inline uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
inline uint32_t morton30(uint32_t cx, uint32_t cy, uint32_t cz) {
  return spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
}

struct OrcParams {
  float h;
  float gravity[3];
  float speed_of_sound;
  float cfl_number;
  float viscosity;
  float domain_min[3];
  float domain_max[3];
  float alpha;  // sph.rs:440 hardcodes 1.0
  float beta;   // sph.rs:441 hardcodes 2.0
  int tier;      // 0 = literal, 1 = grid
  int threads;   // worker threads for Tier G loops (results do not depend on it)
  int pow_mode;  // 0 = libm powf (reference on Linux), 1 = correctly rounded
  int boundary_mode;      // 0 = boundary particles (reference), 1 = SDF wall (tier S)
  float sdf_wall_coef;    // SDF wall repulsion scale
  float sdf_origin[3];
  float sdf_cell;
  uint32_t sdf_dims[3];
  const float* sdf;       // node grid, i*ny*nz + j*nz + k (copied at creation)
  // stage switches, as SphFlags of the C ABI: 1 delta-SPH, 2 XSPH,
  // 4 repulsion, 8 domain clamp (0xF = every reference stage)
  uint32_t flags;
};
constexpr uint32_t kOrcDelta = 1, kOrcXsph = 2, kOrcRepulsion = 4, kOrcClamp = 8;

// ---- Tier S: SDF wall (no reference counterpart; project definition) ----
// The SDF wall stands in for the reference's 3 layers of wall particles
// (orchestrator domain.rs:162-348: depths (layer + 0.5) dx behind the surface,
// lattice spacing dx = h / 1.3, mass rho0 dx^3), homogenised along the wall:
// for a particle at distance d in front of a plane wall, phi(d) is the
// lattice sum of W * dx^3 over those layers and g(d) the sum of -dW/dn dx^3,
// both averaged over 8 x 8 lateral offsets of the lattice. Tabulated at
// kWallN + 1 points on [0, 2h] in double, rounded to f32, linearly
// interpolated in f32.
constexpr int kWallN = 512;
constexpr int kWallN2 = 64;
constexpr int kWallN3 = 24;
struct WallTable {
  float inv_step = 0.0f, inv2 = 0.0f, inv3 = 0.0f;
  std::vector<float> phi, grad;     // one slab, kWallN + 1 distances
  std::vector<float> phi2, grad2;   // edge column, (kWallN2 + 1)^2, gradient along the first face
  std::vector<float> phi3, grad3;   // corner cube, (kWallN3 + 1)^3, gradient along the first face
};

inline WallTable make_wall_table(float hf) {
  WallTable t;
  const double h = hf, dx = h / 1.3, sup = 2.0 * h;
  const double C0 = 21.0 / (16.0 * 3.14159265358979323846);
  const int M = (int)std::ceil(sup / dx) + 1;
  t.phi.assign(kWallN + 1, 0.0f);
  t.grad.assign(kWallN + 1, 0.0f);
  for (int k = 0; k <= kWallN; ++k) {
    double d = (double)k * (sup / kWallN);
    double sw = 0.0, sg = 0.0;
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        double ox = (a + 0.5) / 8.0 * dx, oy = (b + 0.5) / 8.0 * dx;
        for (int layer = 0; layer < 3; ++layer) {
          double z = d + (layer + 0.5) * dx;
          for (int ix = -M; ix <= M; ++ix)
            for (int iy = -M; iy <= M; ++iy) {
              double X = ix * dx + ox, Y = iy * dx + oy;
              double r = std::sqrt(X * X + Y * Y + z * z);
              if (r >= sup) continue;
              double q = r / h, om = 1.0 - 0.5 * q;
              sw += C0 / (h * h * h) * om * om * om * om * (1.0 + 2.0 * q);
              sg += C0 / (h * h * h * h) * 5.0 * q * om * om * om * (z / r);
            }
        }
      }
    double vol = dx * dx * dx / 64.0;
    t.phi[k] = (float)(sw * vol);
    t.grad[k] = (float)(sg * vol);
  }
  t.inv_step = (float)((double)kWallN / sup);
  // Edge column and corner cube of the box walls: the wall sites common to
  // two (three) face slabs, counted once per slab, so the box walls are
  // slabs - edges + corner. Edge averaged over 8 offsets along the edge.
  auto w_and_dw = [&](double r, double& w, double& dw) {
    double q = r / h, om = 1.0 - 0.5 * q;
    w = C0 / (h * h * h) * om * om * om * om * (1.0 + 2.0 * q);
    dw = C0 / (h * h * h * h) * 5.0 * q * om * om * om;
  };
  t.phi2.assign((kWallN2 + 1) * (kWallN2 + 1), 0.0f);
  t.grad2.assign((kWallN2 + 1) * (kWallN2 + 1), 0.0f);
  for (int i = 0; i <= kWallN2; ++i)
    for (int j = 0; j <= kWallN2; ++j) {
      double da = (double)i * (sup / kWallN2), db = (double)j * (sup / kWallN2);
      double sw = 0.0, sg = 0.0;
      for (int c = 0; c < 8; ++c) {
        double oc = (c + 0.5) / 8.0 * dx;
        for (int la = 0; la < 3; ++la)
          for (int lb = 0; lb < 3; ++lb) {
            double za = da + (la + 0.5) * dx, zb = db + (lb + 0.5) * dx;
            for (int it = -M; it <= M; ++it) {
              double T = it * dx + oc;
              double r = std::sqrt(za * za + zb * zb + T * T);
              if (r >= sup) continue;
              double w, dw;
              w_and_dw(r, w, dw);
              sw += w;
              sg += dw * (za / r);
            }
          }
      }
      double vol = dx * dx * dx / 8.0;
      t.phi2[i * (kWallN2 + 1) + j] = (float)(sw * vol);
      t.grad2[i * (kWallN2 + 1) + j] = (float)(sg * vol);
    }
  const int S = kWallN3 + 1;
  t.phi3.assign(S * S * S, 0.0f);
  t.grad3.assign(S * S * S, 0.0f);
  for (int i = 0; i <= kWallN3; ++i)
    for (int j = 0; j <= kWallN3; ++j)
      for (int l = 0; l <= kWallN3; ++l) {
        double da = (double)i * (sup / kWallN3), db = (double)j * (sup / kWallN3), dc = (double)l * (sup / kWallN3);
        double sw = 0.0, sg = 0.0;
        for (int la = 0; la < 3; ++la)
          for (int lb = 0; lb < 3; ++lb)
            for (int lc = 0; lc < 3; ++lc) {
              double za = da + (la + 0.5) * dx, zb = db + (lb + 0.5) * dx, zc = dc + (lc + 0.5) * dx;
              double r = std::sqrt(za * za + zb * zb + zc * zc);
              if (r >= sup) continue;
              double w, dw;
              w_and_dw(r, w, dw);
              sw += w;
              sg += dw * (za / r);
            }
        double vol = dx * dx * dx;
        t.phi3[(i * S + j) * S + l] = (float)(sw * vol);
        t.grad3[(i * S + j) * S + l] = (float)(sg * vol);
      }
  t.inv2 = (float)((double)kWallN2 / sup);
  t.inv3 = (float)((double)kWallN3 / sup);
  return t;
}

// Linear interpolation of a wall table at distance d (clamped to [0, 2h]).
inline float wall_lookup(const std::vector<float>& v, float inv_step, float d) {
  float u = fmaxf(d, 0.0f) * inv_step;
  if (!(u < (float)kWallN)) return 0.0f;
  int i = (int)u;
  float f = u - (float)i;
  return v[i] + f * (v[i + 1] - v[i]);
}

// Bilinear / trilinear interpolation of the edge / corner tables.
inline float wall_lookup2(const std::vector<float>& v, float inv, float da, float db) {
  float u = fmaxf(da, 0.0f) * inv, w = fmaxf(db, 0.0f) * inv;
  if (!(u < (float)kWallN2) || !(w < (float)kWallN2)) return 0.0f;
  int i = (int)u, j = (int)w;
  float fu = u - (float)i, fv = w - (float)j;
  const float* t = v.data() + i * (kWallN2 + 1) + j;
  float a = t[0], b = t[1], c = t[kWallN2 + 1], d = t[kWallN2 + 2];
  float x0 = a + fv * (b - a), x1 = c + fv * (d - c);
  return x0 + fu * (x1 - x0);
}
inline float wall_lookup3(const std::vector<float>& v, float inv, float da, float db, float dc) {
  float u = fmaxf(da, 0.0f) * inv, w = fmaxf(db, 0.0f) * inv, x = fmaxf(dc, 0.0f) * inv;
  if (!(u < (float)kWallN3) || !(w < (float)kWallN3) || !(x < (float)kWallN3)) return 0.0f;
  int i = (int)u, j = (int)w, l = (int)x;
  float fu = u - (float)i, fv = w - (float)j, fw = x - (float)l;
  const int S = kWallN3 + 1;
  const float* t = v.data() + (i * S + j) * S + l;
  float c000 = t[0], c001 = t[1], c010 = t[S], c011 = t[S + 1];
  float c100 = t[S * S], c101 = t[S * S + 1], c110 = t[S * S + S], c111 = t[S * S + S + 1];
  float x00 = c000 + fw * (c001 - c000), x01 = c010 + fw * (c011 - c010);
  float x10 = c100 + fw * (c101 - c100), x11 = c110 + fw * (c111 - c110);
  float x0 = x00 + fv * (x01 - x00), x1 = x10 + fv * (x11 - x10);
  return x0 + fu * (x1 - x0);
}

// GridSDF::sample (geometry.rs:99-150) with the grid coordinate clamped to
// [0, dims-1-1e-3] so that points on or beyond the outer nodes still
// interpolate in the last cell instead of returning f32::MAX.
inline float sdf_sample_clamped(const float* d, const uint32_t dims[3], const float origin[3],
                                float cell, float px, float py, float pz) {
  float g[3] = {(px - origin[0]) / cell, (py - origin[1]) / cell, (pz - origin[2]) / cell};
  int i0[3];
  float fr[3];
  for (int a = 0; a < 3; ++a) {
    g[a] = fminf(fmaxf(g[a], 0.0f), (float)(dims[a] - 1) - 0.001f);
    i0[a] = (int)floorf(g[a]);
    fr[a] = g[a] - (float)i0[a];
  }
  uint32_t ny = dims[1], nz = dims[2];
  auto at = [&](int di, int dj, int dk) {
    return d[(uint64_t)(i0[0] + di) * ny * nz + (uint64_t)(i0[1] + dj) * nz + (uint64_t)(i0[2] + dk)];
  };
  float fx = fr[0], fy = fr[1], fz = fr[2];
  float c00 = at(0, 0, 0) * (1.0f - fz) + at(0, 0, 1) * fz;
  float c01 = at(0, 1, 0) * (1.0f - fz) + at(0, 1, 1) * fz;
  float c10 = at(1, 0, 0) * (1.0f - fz) + at(1, 0, 1) * fz;
  float c11 = at(1, 1, 0) * (1.0f - fz) + at(1, 1, 1) * fz;
  float c0 = c00 * (1.0f - fy) + c01 * fy;
  float c1 = c10 * (1.0f - fy) + c11 * fy;
  return c0 * (1.0f - fx) + c1 * fx;
}

// GridSDF::gradient (geometry.rs:153-175) on the clamped sampler.
inline void sdf_gradient_clamped(const float* d, const uint32_t dims[3], const float origin[3],
                                 float cell, float px, float py, float pz, float out[3]) {
  float h = cell * 0.5f;
  float gx = (sdf_sample_clamped(d, dims, origin, cell, px + h, py, pz) -
              sdf_sample_clamped(d, dims, origin, cell, px - h, py, pz)) / (2.0f * h);
  float gy = (sdf_sample_clamped(d, dims, origin, cell, px, py + h, pz) -
              sdf_sample_clamped(d, dims, origin, cell, px, py - h, pz)) / (2.0f * h);
  float gz = (sdf_sample_clamped(d, dims, origin, cell, px, py, pz + h) -
              sdf_sample_clamped(d, dims, origin, cell, px, py, pz - h)) / (2.0f * h);
  float mag = sqrtf(gx * gx + gy * gy + gz * gz);
  if (mag > 1e-8f) { out[0] = gx / mag; out[1] = gy / mag; out[2] = gz / mag; }
  else { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; }
}

class Kernel {
 public:
  Particles p;
  Boundary b;
  NeighborGrid grid;
  OrcParams prm;
  double initial_energy = 0.0, initial_mass = 0.0;
  bool needs_init = true;
  bool has_checkpoint = false;
  Particles checkpoint;
  // Tier G: static boundary candidate lists per fluid cell (ascending b).
  std::vector<uint32_t> bc_start, bc_list;
  std::vector<float> vx_used, vy_used, vz_used;  // velocities seen by the last compute_forces
  std::vector<float> sdf;  // tier S node grid
  WallTable wall;          // tier S wall table

  // lib.rs:138-174
  Kernel(const OrcParams& pr, Particles&& parts, Boundary&& bnd)
      : p(std::move(parts)), b(std::move(bnd)), prm(pr) {
    grid = NeighborGrid(2.0f * prm.h, prm.domain_min, prm.domain_max);
    double m = 0.0;
    for (size_t i = 0; i < p.len(); ++i) m += (double)p.mass[i];
    initial_mass = m;
    initial_energy = total_energy();
    if (prm.boundary_mode == 1) {
      if (prm.sdf) {
        sdf.assign(prm.sdf, prm.sdf + (size_t)prm.sdf_dims[0] * prm.sdf_dims[1] * prm.sdf_dims[2]);
        prm.sdf = sdf.data();
      }
      wall = make_wall_table(prm.h);
      wall_scale = wall_mass_scale();
    }
    if (prm.tier == 1 && prm.boundary_mode == 0) build_boundary_lists();
  }

  bool sdf_mode() const { return prm.boundary_mode == 1; }
  bool has_geo() const { return prm.sdf != nullptr; }
  // Tier S walls: the nearer face of the domain box on each axis (distance,
  // inward normal sign, within 2h) and the obstacle SDF.
  struct Faces {
    float d[3], s[3];
    bool on[3];
  };
  Faces box_faces(size_t i) const {
    Faces b;
    float pt[3] = {p.x[i], p.y[i], p.z[i]};
    for (int a = 0; a < 3; ++a) {
      float dl = pt[a] - prm.domain_min[a], dh = prm.domain_max[a] - pt[a];
      if (dl <= dh) {
        b.d[a] = dl;
        b.s[a] = 1.0f;
      } else {
        b.d[a] = dh;
        b.s[a] = -1.0f;
      }
      b.on[a] = b.d[a] < 2.0f * prm.h;
    }
    return b;
  }
  // Kernel mass of the walls: box faces (slabs - edges + corner), then the
  // obstacle at SDF distance dgeo.
  float sdf_wall_mass(const Faces& b, float dgeo) const {
    float m = 0.0f;
    for (int a = 0; a < 3; ++a)
      if (b.on[a]) m += wall_lookup(wall.phi, wall.inv_step, b.d[a]);
    for (int a = 0; a < 3; ++a)
      for (int c = a + 1; c < 3; ++c)
        if (b.on[a] && b.on[c]) m -= wall_lookup2(wall.phi2, wall.inv2, b.d[a], b.d[c]);
    if (b.on[0] && b.on[1] && b.on[2]) m += wall_lookup3(wall.phi3, wall.inv3, b.d[0], b.d[1], b.d[2]);
    if (has_geo() && dgeo < 2.0f * prm.h) m += wall_lookup(wall.phi, wall.inv_step, dgeo);
    return m;
  }
  // Wall layers carry the first water particle's mass (domain.rs:57-62),
  // relative to rho0 (h / 1.3)^3; exactly 1 within 1e-5 of 1.
  float wall_scale = 1.0f;
  float wall_mass_scale() const {
    size_t i = 0;
    while (i < p.len() && p.fluid_type[i] != 0) ++i;
    if (i == p.len()) return 1.0f;
    double dx = (double)prm.h / 1.3;
    double s = (double)p.mass[i] / (1000.0 * dx * dx * dx);
    return std::fabs(s - 1.0) < 1e-5 ? 1.0f : (float)s;
  }
  float wall_distance(size_t i) const {
    return sdf_sample_clamped(prm.sdf, prm.sdf_dims, prm.sdf_origin, prm.sdf_cell, p.x[i], p.y[i], p.z[i]);
  }

  // lib.rs:177-194
  double total_energy() const {
    double e = 0.0;
    const float* g = prm.gravity;
    for (size_t i = 0; i < p.len(); ++i) {
      double m = (double)p.mass[i];
      double vx = p.vx[i], vy = p.vy[i], vz = p.vz[i];
      e += 0.5 * m * (vx * vx + vy * vy + vz * vz);
      double x = p.x[i], y = p.y[i], z = p.z[i];
      e -= m * ((double)g[0] * x + (double)g[1] * y + (double)g[2] * z);
    }
    return e;
  }

  // Tier G: a boundary particle b is a candidate of fluid cell c when its
  // distance to the cell's box, widened by a relative margin that exceeds
  // the rounding of pos_to_cell and unbounded outward on clamped edge cells,
  // is below 2h (with margin). Lists are in ascending b.
  void build_boundary_lists() {
    size_t tc = grid.total_cells();
    double cs = grid.cell_size, margin = 1e-4 * cs;
    double reach = 2.0 * (double)prm.h * (1.0 + 1e-4) + margin;
    std::vector<std::vector<uint32_t>> per(tc);
    for (size_t bi = 0; bi < b.len(); ++bi) {
      double pos[3] = {b.x[bi], b.y[bi], b.z[bi]};
      int lo[3], hi[3];
      for (int k = 0; k < 3; ++k) {
        double u0 = (pos[k] - reach - grid.grid_min[k]) / cs;
        double u1 = (pos[k] + reach - grid.grid_min[k]) / cs;
        lo[k] = (int)std::max(0.0, std::min((double)grid.dims[k] - 1, std::floor(u0)));
        hi[k] = (int)std::max(0.0, std::min((double)grid.dims[k] - 1, std::floor(u1)));
      }
      for (int cz = lo[2]; cz <= hi[2]; ++cz)
        for (int cy = lo[1]; cy <= hi[1]; ++cy)
          for (int cx = lo[0]; cx <= hi[0]; ++cx) {
            int c3[3] = {cx, cy, cz};
            double d2 = 0.0;
            for (int k = 0; k < 3; ++k) {
              double blo = (c3[k] == 0) ? -1e300 : grid.grid_min[k] + c3[k] * cs - margin;
              double bhi = (c3[k] == (int)grid.dims[k] - 1) ? 1e300
                                                            : grid.grid_min[k] + (c3[k] + 1) * cs + margin;
              double d = 0.0;
              if (pos[k] < blo) d = blo - pos[k];
              else if (pos[k] > bhi) d = pos[k] - bhi;
              d2 += d * d;
            }
            if (d2 < reach * reach)
              per[grid.cell_hash(cx, cy, cz)].push_back((uint32_t)bi);
          }
    }
    bc_start.assign(tc + 1, 0);
    for (size_t c = 0; c < tc; ++c) bc_start[c + 1] = bc_start[c] + (uint32_t)per[c].size();
    bc_list.resize(bc_start[tc]);
    for (size_t c = 0; c < tc; ++c)
      std::copy(per[c].begin(), per[c].end(), bc_list.begin() + bc_start[c]);
  }

  // Visit boundary particles that may lie in support of fluid particle i, in
  // ascending boundary index (Tier L: all of them).
  template <class F>
  inline void for_each_boundary(size_t i, F&& f) const {
    if (sdf_mode()) return;
    if (prm.tier == 0) {
      for (size_t bi = 0; bi < b.len(); ++bi) f(bi);
    } else {
      uint32_t cx, cy, cz;
      grid.pos_to_cell(p.x[i], p.y[i], p.z[i], &cx, &cy, &cz);
      uint32_t c = grid.cell_hash(cx, cy, cz);
      for (uint32_t s = bc_start[c]; s < bc_start[c + 1]; ++s) f((size_t)bc_list[s]);
    }
  }

  int nthreads() const { return prm.tier == 1 ? std::max(1, prm.threads) : 1; }

  // sph.rs:169-216
  std::vector<float> density_diffusion() const {
    size_t n = p.len();
    float h = prm.h, c = prm.speed_of_sound;
    float support = 2.0f * h;
    float eta_sq = 0.01f * h * h;
    std::vector<float> diffusion(n, 0.0f);
    parallel_for(n, nthreads(), 256, [&](size_t i) {
      float diff_sum = 0.0f;
      grid.for_each_neighbor(i, p.x.data(), p.y.data(), p.z.data(), support, [&](size_t j) {
        float dx = p.x[i] - p.x[j], dy = p.y[i] - p.y[j], dz = p.z[i] - p.z[j];
        float dist_sq = dx * dx + dy * dy + dz * dz;
        float r = sqrtf(dist_sq);
        float gx, gy, gz;
        wendland_c2_gradient(dx, dy, dz, r, h, &gx, &gy, &gz);
        float v_j = p.mass[j] / p.density[j];
        float r_dot_grad = dx * gx + dy * gy + dz * gz;
        float density_diff = p.density[i] - p.density[j];
        diff_sum += v_j * density_diff * 2.0f * r_dot_grad / (dist_sq + eta_sq);
      });
      diffusion[i] = kDeltaSph * h * c * diff_sum;
    });
    return diffusion;
  }

  // sph.rs:112-160
  void compute_density() {
    size_t n = p.len();
    float h = prm.h;
    float support = 2.0f * h;
    std::vector<float> out(n);
    parallel_for(n, nthreads(), 256, [&](size_t i) {
      float rho = p.mass[i] * wendland_c2(0.0f, h);
      grid.for_each_neighbor(i, p.x.data(), p.y.data(), p.z.data(), support, [&](size_t j) {
        float dx = p.x[i] - p.x[j], dy = p.y[i] - p.y[j], dz = p.z[i] - p.z[j];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        rho += p.mass[j] * wendland_c2(r, h);
      });
      float px = p.x[i], py = p.y[i], pz = p.z[i];
      for_each_boundary(i, [&](size_t bi) {
        float dx = px - b.x[bi], dy = py - b.y[bi], dz = pz - b.z[bi];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < support) rho += b.mass[bi] * wendland_c2(r, h);
      });
      if (sdf_mode()) {  // tier S: kernel mass of the walls (box faces, obstacle)
        Faces bf = box_faces(i);
        float dgeo = has_geo() ? wall_distance(i) : support;
        float m = sdf_wall_mass(bf, dgeo);
        float rest = p.fluid_type[i] == 0 ? kWaterRho0 : kAirRho0;
        rho += rest * wall_scale * m;
      }
      out[i] = rho;
    });
    p.density.swap(out);
  }

  // sph.rs:295-312
  void compute_pressure() {
    float c = prm.speed_of_sound;
    for (size_t i = 0; i < p.len(); ++i)
      p.pressure[i] = p.fluid_type[i] == 0
                          ? tait_eos(p.density[i], kWaterRho0, c, kWaterGamma, prm.pow_mode)
                          : tait_eos(p.density[i], kAirRho0, c, kAirGamma, prm.pow_mode);
  }

  // boundary.rs:87-131 (Tier L: fluid index order 0..n; Tier G: the fluid
  // candidates of a widened cell range, sorted by fluid index, then summed).
  void update_boundary_pressures() {
    float h = prm.h, support = 2.0f * h;
    const float* g = prm.gravity;
    size_t nf = p.len();
    parallel_for(b.len(), nthreads(), 64, [&](size_t bi) {
      float bx = b.x[bi], by = b.y[bi], bz = b.z[bi];
      float weighted_pressure = 0.0f, weight_sum = 0.0f;
      auto term = [&](size_t f) {
        float dx = bx - p.x[f], dy = by - p.y[f], dz = bz - p.z[f];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < support) {
          float w = wendland_c2(r, h);
          float g_dot_dr = g[0] * dx + g[1] * dy + g[2] * dz;
          float p_ext = p.pressure[f] + p.density[f] * g_dot_dr;
          weighted_pressure += w * p_ext;
          weight_sum += w;
        }
      };
      if (prm.tier == 0) {
        for (size_t f = 0; f < nf; ++f) term(f);
      } else {
        std::vector<uint32_t> cand;
        double cs = grid.cell_size;
        double reach = 2.0 * (double)h * (1.0 + 1e-4) + 1e-4 * cs;
        double pos[3] = {bx, by, bz};
        int lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
          lo[k] = (int)grid.axis_cell((float)(pos[k] - reach), k);
          hi[k] = (int)grid.axis_cell((float)(pos[k] + reach), k);
        }
        for (int cz = lo[2]; cz <= hi[2]; ++cz)
          for (int cy = lo[1]; cy <= hi[1]; ++cy)
            for (int cx = lo[0]; cx <= hi[0]; ++cx) {
              uint32_t c = grid.cell_hash(cx, cy, cz);
              for (uint32_t s = grid.cell_offsets[c]; s < grid.cell_offsets[c] + grid.cell_counts[c]; ++s)
                cand.push_back(grid.sorted_indices[s]);
            }
        std::sort(cand.begin(), cand.end());
        for (uint32_t f : cand) term(f);
      }
      if (weight_sum > 1.0e-12f) b.pressure[bi] = fmaxf(weighted_pressure / weight_sum, 0.0f);
      else b.pressure[bi] = 0.0f;
    });
  }

  // sph.rs:322-417
  void compute_pressure_forces() {
    size_t n = p.len();
    float h = prm.h, support = 2.0f * h;
    std::vector<float> fx(n, 0.0f), fy(n, 0.0f), fz(n, 0.0f);
    parallel_for(n, nthreads(), 256, [&](size_t i) {
      float pi_over_rho2_i = p.pressure[i] / (p.density[i] * p.density[i]);
      grid.for_each_neighbor(i, p.x.data(), p.y.data(), p.z.data(), support, [&](size_t j) {
        float dx = p.x[i] - p.x[j], dy = p.y[i] - p.y[j], dz = p.z[i] - p.z[j];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        float gx, gy, gz;
        wendland_c2_gradient(dx, dy, dz, r, h, &gx, &gy, &gz);
        float pj_over_rho2_j = p.pressure[j] / (p.density[j] * p.density[j]);
        float factor = -p.mass[i] * p.mass[j] * (pi_over_rho2_i + pj_over_rho2_j);
        fx[i] += factor * gx;
        fy[i] += factor * gy;
        fz[i] += factor * gz;
      });
      float px = p.x[i], py = p.y[i], pz = p.z[i];
      float m_i = p.mass[i];
      float pi_clamped = fmaxf(p.pressure[i], 0.0f);
      float pi_clamped_over_rho2 = pi_clamped / (p.density[i] * p.density[i]);
      float boundary_rho = p.fluid_type[i] == 0 ? kWaterRho0 : kAirRho0;
      for_each_boundary(i, [&](size_t bi) {
        float dx = px - b.x[bi], dy = py - b.y[bi], dz = pz - b.z[bi];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < support) {
          float gx, gy, gz;
          wendland_c2_gradient(dx, dy, dz, r, h, &gx, &gy, &gz);
          float pb_over_rho2_b = b.pressure[bi] / (boundary_rho * boundary_rho);
          float factor = -m_i * b.mass[bi] * (pi_clamped_over_rho2 + pb_over_rho2_b);
          fx[i] += factor * gx;
          fy[i] += factor * gy;
          fz[i] += factor * gz;
        }
      });
    });
    for (size_t i = 0; i < n; ++i) {
      p.ax[i] += fx[i] / p.mass[i];
      p.ay[i] += fy[i] / p.mass[i];
      p.az[i] += fz[i] / p.mass[i];
    }
  }

  // sph.rs:432-492 (alpha, beta are parameters; the reference hardcodes 1, 2)
  void compute_viscous_forces() {
    size_t n = p.len();
    float h = prm.h, support = 2.0f * h, c = prm.speed_of_sound;
    float alpha = prm.alpha, beta = prm.beta;
    float eta_sq = 0.01f * h * h;
    std::vector<float> fx(n, 0.0f), fy(n, 0.0f), fz(n, 0.0f);
    parallel_for(n, nthreads(), 256, [&](size_t i) {
      grid.for_each_neighbor(i, p.x.data(), p.y.data(), p.z.data(), support, [&](size_t j) {
        float dx = p.x[i] - p.x[j], dy = p.y[i] - p.y[j], dz = p.z[i] - p.z[j];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        float dvx = p.vx[i] - p.vx[j], dvy = p.vy[i] - p.vy[j], dvz = p.vz[i] - p.vz[j];
        float vr_dot = dvx * dx + dvy * dy + dvz * dz;
        if (vr_dot < 0.0f) {
          float r_sq = r * r;
          float mu_ij = h * vr_dot / (r_sq + eta_sq);
          float rho_avg = 0.5f * (p.density[i] + p.density[j]);
          float pi_ij = (-alpha * c * mu_ij + beta * mu_ij * mu_ij) / rho_avg;
          float gx, gy, gz;
          wendland_c2_gradient(dx, dy, dz, r, h, &gx, &gy, &gz);
          float factor = -p.mass[j] * pi_ij;
          fx[i] += factor * gx;
          fy[i] += factor * gy;
          fz[i] += factor * gz;
        }
      });
    });
    for (size_t i = 0; i < n; ++i) {
      p.ax[i] += fx[i];
      p.ay[i] += fy[i];
      p.az[i] += fz[i];
    }
  }

  // boundary.rs:143-181
  void compute_repulsive_forces() {
    float h = prm.h;
    float r0 = 0.5f * h;
    float d = 10.0f * 9.81f * 0.01f;
    parallel_for(p.len(), nthreads(), 256, [&](size_t i) {
      float px = p.x[i], py = p.y[i], pz = p.z[i];
      for_each_boundary(i, [&](size_t bi) {
        float dx = px - b.x[bi], dy = py - b.y[bi], dz = pz - b.z[bi];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        if (r < r0 && r > 1.0e-12f) {
          float s = 1.0f - r / r0;
          float force_mag = d * s * s / r0;
          float inv_r = 1.0f / r;
          p.ax[i] += force_mag * dx * inv_r;
          p.ay[i] += force_mag * dy * inv_r;
          p.az[i] += force_mag * dz * inv_r;
        }
      });
    });
  }

  // lib.rs:203-283
  void compute_forces(float dt) {
    size_t n = p.len();
    vx_used = p.vx; vy_used = p.vy; vz_used = p.vz;
    grid.update(p.x.data(), p.y.data(), p.z.data(), n);
    if (prm.flags & kOrcDelta) {
      std::vector<float> diffusion = density_diffusion();
      compute_density();
      for (size_t i = 0; i < n; ++i) p.density[i] += diffusion[i] * dt;
    } else {
      compute_density();
    }
    compute_pressure();
    if (!sdf_mode()) update_boundary_pressures();
    for (size_t i = 0; i < n; ++i) { p.ax[i] = 0.0f; p.ay[i] = 0.0f; p.az[i] = 0.0f; }
    compute_pressure_forces();
    compute_viscous_forces();
    for (size_t i = 0; i < n; ++i) {  // sph.rs:502-508
      p.ax[i] += prm.gravity[0];
      p.ay[i] += prm.gravity[1];
      p.az[i] += prm.gravity[2];
    }
    if (sdf_mode()) compute_sdf_wall_forces();
    else if (prm.flags & kOrcRepulsion) compute_repulsive_forces();
  }

  // Tier S wall force, after gravity: the energy-consistent counterpart of the
  // walls' kernel mass in rho_i, (p_i / rho_i^2) rho0 s grad(phi) per wall
  // term (box faces per axis: slabs - edges + corner, then each face's
  // repulsion; then the obstacle along its SDF normal and its repulsion).
  void compute_sdf_wall_forces() {
    float h = prm.h, support = 2.0f * h, r0 = 0.5f * h;
    parallel_for(p.len(), nthreads(), 256, [&](size_t i) {
      float rest = p.fluid_type[i] == 0 ? kWaterRho0 : kAirRho0;
      float rho_i = p.density[i];
      float pic = fmaxf(p.pressure[i], 0.0f);
      float pic_over = pic / (rho_i * rho_i);
      float cw = rest * wall_scale;
      float base = pic_over * cw;
      // box faces per axis: slabs - edges + corner, then each face's repulsion
      Faces bf = box_faces(i);
      float wa[3] = {0.0f, 0.0f, 0.0f};
      for (int a = 0; a < 3; ++a)
        if (bf.on[a]) wa[a] += base * wall_lookup(wall.grad, wall.inv_step, bf.d[a]) * bf.s[a];
      for (int a = 0; a < 3; ++a)
        for (int c = a + 1; c < 3; ++c)
          if (bf.on[a] && bf.on[c]) {
            wa[a] -= base * wall_lookup2(wall.grad2, wall.inv2, bf.d[a], bf.d[c]) * bf.s[a];
            wa[c] -= base * wall_lookup2(wall.grad2, wall.inv2, bf.d[c], bf.d[a]) * bf.s[c];
          }
      if (bf.on[0] && bf.on[1] && bf.on[2]) {
        wa[0] += base * wall_lookup3(wall.grad3, wall.inv3, bf.d[0], bf.d[1], bf.d[2]) * bf.s[0];
        wa[1] += base * wall_lookup3(wall.grad3, wall.inv3, bf.d[1], bf.d[0], bf.d[2]) * bf.s[1];
        wa[2] += base * wall_lookup3(wall.grad3, wall.inv3, bf.d[2], bf.d[0], bf.d[1]) * bf.s[2];
      }
      for (int a = 0; a < 3; ++a)
        if ((prm.flags & kOrcRepulsion) && bf.d[a] < r0) {
          float s = 1.0f - fmaxf(bf.d[a], 0.0f) / r0;
          float fm = prm.sdf_wall_coef * s * s / r0;
          wa[a] += fm * bf.s[a];
        }
      p.ax[i] += wa[0];
      p.ay[i] += wa[1];
      p.az[i] += wa[2];
      // the obstacle along its SDF normal
      float d = has_geo() ? wall_distance(i) : support;
      if (!(d < support)) return;
      float n[3];
      sdf_gradient_clamped(prm.sdf, prm.sdf_dims, prm.sdf_origin, prm.sdf_cell, p.x[i], p.y[i], p.z[i], n);
      float coef = base * wall_lookup(wall.grad, wall.inv_step, d);
      p.ax[i] += coef * n[0];
      p.ay[i] += coef * n[1];
      p.az[i] += coef * n[2];
      if ((prm.flags & kOrcRepulsion) && d < r0) {
        float s = 1.0f - fmaxf(d, 0.0f) / r0;
        float fm = prm.sdf_wall_coef * s * s / r0;
        p.ax[i] += fm * n[0];
        p.ay[i] += fm * n[1];
        p.az[i] += fm * n[2];
      }
    });
  }

  // sph.rs:236-280
  void xsph(std::vector<float>& dvx, std::vector<float>& dvy, std::vector<float>& dvz) const {
    size_t n = p.len();
    float h = prm.h, support = 2.0f * h;
    dvx.assign(n, 0.0f); dvy.assign(n, 0.0f); dvz.assign(n, 0.0f);
    parallel_for(n, nthreads(), 256, [&](size_t i) {
      float cx = 0.0f, cy = 0.0f, cz = 0.0f;
      grid.for_each_neighbor(i, p.x.data(), p.y.data(), p.z.data(), support, [&](size_t j) {
        float dx = p.x[i] - p.x[j], dy = p.y[i] - p.y[j], dz = p.z[i] - p.z[j];
        float r = sqrtf(dx * dx + dy * dy + dz * dz);
        float w = wendland_c2(r, h);
        float rho_avg = 0.5f * (p.density[i] + p.density[j]);
        float factor = p.mass[j] / fmaxf(rho_avg, 1.0f) * w;
        cx += factor * (p.vx[j] - p.vx[i]);
        cy += factor * (p.vy[j] - p.vy[i]);
        cz += factor * (p.vz[j] - p.vz[i]);
      });
      dvx[i] = kXsphEps * cx;
      dvy[i] = kXsphEps * cy;
      dvz[i] = kXsphEps * cz;
    });
  }

  // boundary.rs:239-291
  void enforce_no_penetration_domain() {
    const float restitution = 0.2f;
    const float* mn = prm.domain_min;
    const float* mx = prm.domain_max;
    for (size_t i = 0; i < p.len(); ++i) {
      if (p.x[i] < mn[0]) { p.x[i] = mn[0]; if (p.vx[i] < 0.0f) p.vx[i] = -restitution * p.vx[i]; }
      if (p.x[i] > mx[0]) { p.x[i] = mx[0]; if (p.vx[i] > 0.0f) p.vx[i] = -restitution * p.vx[i]; }
      if (p.y[i] < mn[1]) { p.y[i] = mn[1]; if (p.vy[i] < 0.0f) p.vy[i] = -restitution * p.vy[i]; }
      if (p.y[i] > mx[1]) { p.y[i] = mx[1]; if (p.vy[i] > 0.0f) p.vy[i] = -restitution * p.vy[i]; }
      if (p.z[i] < mn[2]) { p.z[i] = mn[2]; if (p.vz[i] < 0.0f) p.vz[i] = -restitution * p.vz[i]; }
      if (p.z[i] > mx[2]) { p.z[i] = mx[2]; if (p.vz[i] > 0.0f) p.vz[i] = -restitution * p.vz[i]; }
    }
  }

  // lib.rs:287-335
  void step(float dt) {
    size_t n = p.len();
    float half_dt = 0.5f * dt;
    if (needs_init) {
      compute_forces(dt);
      needs_init = false;
    }
    for (size_t i = 0; i < n; ++i) {
      p.vx[i] += p.ax[i] * half_dt;
      p.vy[i] += p.ay[i] * half_dt;
      p.vz[i] += p.az[i] * half_dt;
    }
    std::vector<float> dvx, dvy, dvz;
    if (prm.flags & kOrcXsph) {
      xsph(dvx, dvy, dvz);
    } else {  // the drift adds a zero correction, as the CUDA step does
      dvx.assign(n, 0.0f); dvy.assign(n, 0.0f); dvz.assign(n, 0.0f);
    }
    for (size_t i = 0; i < n; ++i) {
      p.x[i] += (p.vx[i] + dvx[i]) * dt;
      p.y[i] += (p.vy[i] + dvy[i]) * dt;
      p.z[i] += (p.vz[i] + dvz[i]) * dt;
    }
    if (prm.flags & kOrcClamp) enforce_no_penetration_domain();
    compute_forces(dt);
    for (size_t i = 0; i < n; ++i) {
      p.vx[i] += p.ax[i] * half_dt;
      p.vy[i] += p.ay[i] * half_dt;
      p.vz[i] += p.az[i] * half_dt;
    }
  }

  // lib.rs:341-377
  void error_metrics(float out[3]) const {
    float max_var = 0.0f;
    for (size_t i = 0; i < p.len(); ++i) {
      float rest = p.fluid_type[i] == 0 ? kWaterRho0 : kAirRho0;
      float var = fabsf(p.density[i] - rest) / rest;
      if (var > max_var) max_var = var;
    }
    double e = total_energy();
    float ed = fabs(initial_energy) > 1.0e-12 ? (float)fabs((e - initial_energy) / initial_energy)
                                               : (float)fabs(e - initial_energy);
    double m = 0.0;
    for (size_t i = 0; i < p.len(); ++i) m += (double)p.mass[i];
    float md = fabs(initial_mass) > 1.0e-12 ? (float)fabs((m - initial_mass) / initial_mass)
                                             : (float)fabs(m - initial_mass);
    out[0] = max_var; out[1] = ed; out[2] = md;
  }
};

// sph.rs:591-628
float compute_timestep(const Particles& p, float h, float c, float cfl) {
  float max_signal = c, max_accel = 0.0f;
  for (size_t i = 0; i < p.len(); ++i) {
    float v = sqrtf(p.vx[i] * p.vx[i] + p.vy[i] * p.vy[i] + p.vz[i] * p.vz[i]);
    float signal = v + c;
    if (signal > max_signal) max_signal = signal;
    float a = sqrtf(p.ax[i] * p.ax[i] + p.ay[i] * p.ay[i] + p.az[i] * p.az[i]);
    if (a > max_accel) max_accel = a;
  }
  float dt_cfl = cfl * h / max_signal;
  float dt_force = max_accel > 1.0e-12f ? 0.25f * sqrtf(h / max_accel) : kMaxDt;
  float dt = fminf(dt_cfl, dt_force);
  return fminf(fmaxf(dt, kMinDt), kMaxDt);
}

Particles make_particles(size_t n, float* const* fields, const uint8_t* ft) {
  Particles p;
  for (int k = 0; k < 13; ++k) p.field(k)->assign(fields[k], fields[k] + n);
  p.fluid_type.assign(ft, ft + n);
  return p;
}

// orchestrator geometry.rs:178-181
inline float sdf_get(const float* d, const uint32_t dims[3], uint32_t i, uint32_t j, uint32_t k) {
  uint64_t idx = (uint64_t)(i * dims[1] * dims[2] + j * dims[2] + k);
  uint64_t total = (uint64_t)dims[0] * dims[1] * dims[2];
  return idx < total ? d[idx] : 3.40282347e38f;
}

// orchestrator geometry.rs:99-150
float sdf_sample(const float* d, const uint32_t dims[3], const float origin[3], float cell,
                 const float pt[3]) {
  float gx = (pt[0] - origin[0]) / cell;
  float gy = (pt[1] - origin[1]) / cell;
  float gz = (pt[2] - origin[2]) / cell;
  int i0 = (int)floorf(gx), j0 = (int)floorf(gy), k0 = (int)floorf(gz);
  const float FMAX = 3.40282347e38f;
  if (i0 < 0 || j0 < 0 || k0 < 0) return FMAX;
  int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  if (i1 >= (int)dims[0] || j1 >= (int)dims[1] || k1 >= (int)dims[2]) return FMAX;
  float fx = gx - (float)i0, fy = gy - (float)j0, fz = gz - (float)k0;
  float c000 = sdf_get(d, dims, i0, j0, k0), c001 = sdf_get(d, dims, i0, j0, k1);
  float c010 = sdf_get(d, dims, i0, j1, k0), c011 = sdf_get(d, dims, i0, j1, k1);
  float c100 = sdf_get(d, dims, i1, j0, k0), c101 = sdf_get(d, dims, i1, j0, k1);
  float c110 = sdf_get(d, dims, i1, j1, k0), c111 = sdf_get(d, dims, i1, j1, k1);
  float c00 = c000 * (1.0f - fz) + c001 * fz;
  float c01 = c010 * (1.0f - fz) + c011 * fz;
  float c10 = c100 * (1.0f - fz) + c101 * fz;
  float c11 = c110 * (1.0f - fz) + c111 * fz;
  float c0 = c00 * (1.0f - fy) + c01 * fy;
  float c1 = c10 * (1.0f - fy) + c11 * fy;
  return c0 * (1.0f - fx) + c1 * fx;
}

// orchestrator geometry.rs:153-175
void sdf_gradient(const float* d, const uint32_t dims[3], const float origin[3], float cell,
                  const float pt[3], float out[3]) {
  float h = cell * 0.5f;
  float a[3], bb[3];
  float g[3];
  for (int k = 0; k < 3; ++k) {
    for (int m = 0; m < 3; ++m) { a[m] = pt[m]; bb[m] = pt[m]; }
    a[k] = pt[k] + h;
    bb[k] = pt[k] - h;
    g[k] = (sdf_sample(d, dims, origin, cell, a) - sdf_sample(d, dims, origin, cell, bb)) / (2.0f * h);
  }
  float mag = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if (mag > 1e-8f) { out[0] = g[0] / mag; out[1] = g[1] / mag; out[2] = g[2] / mag; }
  else { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; }
}

}  // namespace

extern "C" {

// ---- scalar known-answer functions -------------------------------------
float orc_wendland(float r, float h) { return wendland_c2(r, h); }
void orc_wendland_gradient(float dx, float dy, float dz, float r, float h, float* out3) {
  wendland_c2_gradient(dx, dy, dz, r, h, &out3[0], &out3[1], &out3[2]);
}
float orc_tait(float rho, float rho0, float c, float gamma, int pow_mode) {
  return tait_eos(rho, rho0, c, gamma, pow_mode);
}
float orc_norm() { return kNorm; }

// ---- neighbour grid -----------------------------------------------------
void orc_grid_dims(float cell, const float* mn, const float* mx, uint32_t* dims_out) {
  NeighborGrid g(cell, mn, mx);
  for (int k = 0; k < 3; ++k) dims_out[k] = g.dims[k];
}

// NeighborGrid::update restated; plus per-particle (cx,cy,cz), the 30-bit
// Morton key of the cell, and the Morton-ordered layout: cells ranked by
// Morton code, particles stably sorted by (cell rank, index).
// counts/offsets/morton_offsets have total_cells entries.
void orc_grid_build(size_t n, const float* x, const float* y, const float* z, float cell,
                    const float* mn, const float* mx, uint32_t* cell_idx, uint32_t* counts,
                    uint32_t* offsets, uint32_t* sorted, uint32_t* morton_key,
                    uint32_t* morton_offsets, uint32_t* morton_perm) {
  NeighborGrid g(cell, mn, mx);
  g.update(x, y, z, n);
  size_t tc = g.total_cells();
  std::memcpy(cell_idx, g.cell_indices.data(), n * 4);
  std::memcpy(counts, g.cell_counts.data(), tc * 4);
  std::memcpy(offsets, g.cell_offsets.data(), tc * 4);
  std::memcpy(sorted, g.sorted_indices.data(), n * 4);
  for (size_t i = 0; i < n; ++i) {
    uint32_t cx, cy, cz;
    g.pos_to_cell(x[i], y[i], z[i], &cx, &cy, &cz);
    morton_key[i] = morton30(cx, cy, cz);
  }
  // Cells in Morton order (dims <= 1024 per axis so codes are unique).
  std::vector<std::pair<uint32_t, uint32_t>> cells(tc);
  for (uint32_t cz = 0; cz < g.dims[2]; ++cz)
    for (uint32_t cy = 0; cy < g.dims[1]; ++cy)
      for (uint32_t cx = 0; cx < g.dims[0]; ++cx) {
        uint32_t lin = g.cell_hash(cx, cy, cz);
        cells[lin] = {morton30(cx, cy, cz), lin};
      }
  std::sort(cells.begin(), cells.end());
  uint32_t running = 0;
  for (size_t r = 0; r < tc; ++r) {
    uint32_t lin = cells[r].second;
    morton_offsets[lin] = running;
    running += g.cell_counts[lin];
  }
  std::vector<uint32_t> heads(morton_offsets, morton_offsets + tc);
  for (size_t i = 0; i < n; ++i) {
    uint32_t ci = g.cell_indices[i];
    morton_perm[heads[ci]++] = (uint32_t)i;
  }
}

// Neighbour list of particle i in the reference visit order.
size_t orc_neighbors(size_t n, const float* x, const float* y, const float* z, float h,
                     const float* mn, const float* mx, size_t i, uint32_t* out, size_t cap) {
  NeighborGrid g(2.0f * h, mn, mx);
  g.update(x, y, z, n);
  size_t k = 0;
  g.for_each_neighbor(i, x, y, z, 2.0f * h, [&](size_t j) {
    if (k < cap) out[k] = (uint32_t)j;
    ++k;
  });
  return k;
}

// ---- kernel -------------------------------------------------------------
void* orc_create(const OrcParams* prm, size_t n, float* const* fields, const uint8_t* ft,
                 size_t nb, float* const* bfields) {
  Particles p = make_particles(n, fields, ft);
  Boundary b;
  std::vector<float>* bf[7] = {&b.x, &b.y, &b.z, &b.mass, &b.nx, &b.ny, &b.nz};
  for (int k = 0; k < 7; ++k) bf[k]->assign(bfields[k], bfields[k] + nb);
  b.pressure.assign(nb, 0.0f);
  return new Kernel(*prm, std::move(p), std::move(b));
}
void orc_destroy(void* k) { delete static_cast<Kernel*>(k); }
void orc_step(void* k, float dt) { static_cast<Kernel*>(k)->step(dt); }
void orc_compute_forces(void* k, float dt) { static_cast<Kernel*>(k)->compute_forces(dt); }
size_t orc_particle_count(void* k) { return static_cast<Kernel*>(k)->p.len(); }
void orc_get(void* kp, float* const* fields, uint8_t* ft) {
  Kernel* k = static_cast<Kernel*>(kp);
  size_t n = k->p.len();
  for (int f = 0; f < 13; ++f) std::memcpy(fields[f], k->p.field(f)->data(), n * 4);
  if (ft) std::memcpy(ft, k->p.fluid_type.data(), n);
}
void orc_get_boundary_pressure(void* kp, float* out) {
  Kernel* k = static_cast<Kernel*>(kp);
  std::memcpy(out, k->b.pressure.data(), k->b.len() * 4);
}
void orc_error_metrics(void* k, float* out3) { static_cast<Kernel*>(k)->error_metrics(out3); }
float orc_compute_timestep(void* kp, float cfl) {
  Kernel* k = static_cast<Kernel*>(kp);
  return compute_timestep(k->p, k->prm.h, k->prm.speed_of_sound, cfl);
}
// lib.rs:383-395: the checkpoint holds the particle arrays only.
int orc_save_checkpoint(void* kp) {
  Kernel* k = static_cast<Kernel*>(kp);
  k->checkpoint = k->p;
  k->has_checkpoint = true;
  return 1;
}
int orc_restore_checkpoint(void* kp) {
  Kernel* k = static_cast<Kernel*>(kp);
  if (!k->has_checkpoint) return 0;
  k->p = std::move(k->checkpoint);
  k->checkpoint = Particles();
  k->has_checkpoint = false;
  return 1;
}
// Number of (cell, boundary) candidate pairs of Tier G (0 for Tier L).
size_t orc_boundary_list_size(void* kp) { return static_cast<Kernel*>(kp)->bc_list.size(); }

float orc_compute_timestep_arrays(size_t n, const float* vx, const float* vy, const float* vz,
                                  const float* ax, const float* ay, const float* az, float h,
                                  float c, float cfl) {
  Particles p;
  p.vx.assign(vx, vx + n); p.vy.assign(vy, vy + n); p.vz.assign(vz, vz + n);
  p.ax.assign(ax, ax + n); p.ay.assign(ay, ay + n); p.az.assign(az, az + n);
  p.x.resize(n);
  return compute_timestep(p, h, c, cfl);
}

// ---- force extraction ---------------------------------------------------
// orchestrator force.rs:39-129, literal: f32 sums over nodes in (i,j,k)
// order with brute-force particle loops; out_f32[6] = force, moment. Also
// the same per-node contributions summed in FP64 (out_f64[6]).
void orc_surface_forces(void* kp, const float* d, const uint32_t* dims, const float* origin, float cell,
                        float* out_f32, double* out_f64, uint32_t* nodes) {
  Kernel* k = static_cast<Kernel*>(kp);
  const Particles& p = k->p;
  float h = k->prm.h;
  float surface_threshold = 2.0f * h;
  float d_area = cell * cell;
  float nf[3] = {0, 0, 0}, nm[3] = {0, 0, 0};
  double df[3] = {0, 0, 0}, dm[3] = {0, 0, 0};
  uint32_t cnt = 0;
  for (uint32_t i = 0; i < dims[0]; ++i)
    for (uint32_t j = 0; j < dims[1]; ++j)
      for (uint32_t kk = 0; kk < dims[2]; ++kk) {
        float pt[3] = {origin[0] + (float)i * cell, origin[1] + (float)j * cell, origin[2] + (float)kk * cell};
        float dist = sdf_sample(d, dims, origin, cell, pt);
        if (fabsf(dist) > surface_threshold || dist > 0.0f) continue;
        float n[3];
        sdf_gradient(d, dims, origin, cell, pt, n);
        float nmag = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nmag < 1e-8f) continue;
        ++cnt;
        float lp = 0.0f, ws = 0.0f;
        for (size_t q = 0; q < p.len(); ++q) {
          float dx = p.x[q] - pt[0], dy = p.y[q] - pt[1], dz = p.z[q] - pt[2];
          float r = sqrtf(dx * dx + dy * dy + dz * dz);
          if (r < 2.0f * h) {
            float w = wendland_c2(r, h);
            lp += p.pressure[q] * w;
            ws += w;
          }
        }
        if (ws > 1e-12f) {
          lp /= ws;
          float fx = -lp * n[0] * d_area, fy = -lp * n[1] * d_area, fz = -lp * n[2] * d_area;
          float mx = pt[1] * fz - pt[2] * fy, my = pt[2] * fx - pt[0] * fz, mz = pt[0] * fy - pt[1] * fx;
          nf[0] += fx; nf[1] += fy; nf[2] += fz;
          nm[0] += mx; nm[1] += my; nm[2] += mz;
          df[0] += fx; df[1] += fy; df[2] += fz;
          dm[0] += mx; dm[1] += my; dm[2] += mz;
        }
      }
  for (int a = 0; a < 3; ++a) {
    out_f32[a] = nf[a]; out_f32[3 + a] = nm[a];
    out_f64[a] = df[a]; out_f64[3 + a] = dm[a];
  }
  *nodes = cnt;
}

// Fluid reaction on boundary particles [first, first+count) from the last
// force computation (the negated terms of sph.rs:391-408 and
// boundary.rs:161-179; viscous: Monaghan with the body at rest). 18 doubles:
// pressure F, M; repulsion F, M; viscous F, M.
void orc_body_force(void* kp, uint32_t first, uint32_t count, double* out) {
  Kernel* k = static_cast<Kernel*>(kp);
  const float* vx_used = k->vx_used.data();
  const float* vy_used = k->vy_used.data();
  const float* vz_used = k->vz_used.data();
  const Particles& p = k->p;
  const Boundary& b = k->b;
  float h = k->prm.h, support = 2.0f * h, r0 = 0.5f * h, eta_sq = 0.01f * h * h;
  float dconst = 10.0f * 9.81f * 0.01f;
  float nac = -k->prm.alpha * k->prm.speed_of_sound;
  for (int c = 0; c < 18; ++c) out[c] = 0.0;
  for (size_t i = 0; i < p.len(); ++i) {
    float rest = p.fluid_type[i] == 0 ? kWaterRho0 : kAirRho0;
    float pic_over = fmaxf(p.pressure[i], 0.0f) / (p.density[i] * p.density[i]);
    for (uint32_t bi = first; bi < first + count; ++bi) {
      float dx = p.x[i] - b.x[bi], dy = p.y[i] - b.y[bi], dz = p.z[i] - b.z[bi];
      float r = sqrtf(dx * dx + dy * dy + dz * dz);
      if (!(r < support)) continue;
      float g[3];
      wendland_c2_gradient(dx, dy, dz, r, h, &g[0], &g[1], &g[2]);
      float factor = -p.mass[i] * b.mass[bi] * (pic_over + b.pressure[bi] / (rest * rest));
      double F[3] = {-(double)(factor * g[0]), -(double)(factor * g[1]), -(double)(factor * g[2])};
      double R[3] = {0, 0, 0};
      if (r < r0 && r > 1.0e-12f) {
        float s = 1.0f - r / r0;
        float fm = dconst * s * s / r0;
        float inv_r = 1.0f / r;
        R[0] = -(double)p.mass[i] * (double)(fm * dx * inv_r);
        R[1] = -(double)p.mass[i] * (double)(fm * dy * inv_r);
        R[2] = -(double)p.mass[i] * (double)(fm * dz * inv_r);
      }
      double V[3] = {0, 0, 0};
      float vr = vx_used[i] * dx + vy_used[i] * dy + vz_used[i] * dz;
      if (vr < 0.0f) {
        float mu = h * vr / (r * r + eta_sq);
        float pij = (nac * mu + k->prm.beta * mu * mu) / (0.5f * (p.density[i] + rest));
        float fv = -p.mass[i] * b.mass[bi] * pij;
        V[0] = -(double)(fv * g[0]); V[1] = -(double)(fv * g[1]); V[2] = -(double)(fv * g[2]);
      }
      double X[3] = {b.x[bi], b.y[bi], b.z[bi]};
      const double* G[3] = {F, R, V};
      for (int t = 0; t < 3; ++t) {
        out[6 * t + 0] += G[t][0]; out[6 * t + 1] += G[t][1]; out[6 * t + 2] += G[t][2];
        out[6 * t + 3] += X[1] * G[t][2] - X[2] * G[t][1];
        out[6 * t + 4] += X[2] * G[t][0] - X[0] * G[t][2];
        out[6 * t + 5] += X[0] * G[t][1] - X[1] * G[t][0];
      }
    }
  }
}

// ---- Tier S helpers -----------------------------------------------------
// Wall tables for smoothing length h: kWallN + 1 entries each.
int orc_wall_table(float h, float* phi, float* grad, float* inv_step) {
  WallTable t = make_wall_table(h);
  std::memcpy(phi, t.phi.data(), t.phi.size() * 4);
  std::memcpy(grad, t.grad.data(), t.grad.size() * 4);
  *inv_step = t.inv_step;
  return kWallN;
}
// Edge ((kWallN2 + 1)^2) and corner ((kWallN3 + 1)^3) tables; returns
// kWallN2 * 1000 + kWallN3.
int orc_wall_tables_box(float h, float* phi2, float* grad2, float* phi3, float* grad3, float* inv2, float* inv3) {
  WallTable t = make_wall_table(h);
  std::memcpy(phi2, t.phi2.data(), t.phi2.size() * 4);
  std::memcpy(grad2, t.grad2.data(), t.grad2.size() * 4);
  std::memcpy(phi3, t.phi3.data(), t.phi3.size() * 4);
  std::memcpy(grad3, t.grad3.data(), t.grad3.size() * 4);
  *inv2 = t.inv2;
  *inv3 = t.inv3;
  return kWallN2 * 1000 + kWallN3;
}
float orc_sdf_sample_clamped(const float* d, const uint32_t* dims, const float* origin, float cell,
                             const float* pt) {
  return sdf_sample_clamped(d, dims, origin, cell, pt[0], pt[1], pt[2]);
}
void orc_sdf_gradient_clamped(const float* d, const uint32_t* dims, const float* origin, float cell,
                              const float* pt, float* out3) {
  sdf_gradient_clamped(d, dims, origin, cell, pt[0], pt[1], pt[2], out3);
}

// ---- setup_domain (orchestrator domain.rs:36-402), literally ------------
// Loops, tests and f32 expressions as the reference writes them; results
// appended in its order. `counts` gets (fluid, boundary); the arrays (NULL to
// count only) must hold that many. fluid_type: 0 water, 1 air, 2 mixed;
// wall_faces bit f = face f (x_min, x_max, y_min, y_max, z_min, z_max) is a
// Wall. Fluid fields written: x, y, z, mass, density, type (the others are
// push_particle's zeros and the temperature); boundary: x, y, z, mass, n.
void orc_setup_domain(float spacing, const float* dmin, const float* dmax, int fluid_type, uint32_t wall_faces,
                      const float* d, const uint32_t* dims, const float* origin, float cell, uint64_t* counts,
                      float* fx, float* fy, float* fz, float* fmass, float* fdens, uint8_t* ftype, float* bx,
                      float* by, float* bz, float* bmass_out, float* bnx, float* bny, float* bnz) {
  const float volume = spacing * (spacing * spacing);  // powi(3) (domain.rs:43)
  const float water_mass = 1000.0f * volume, air_mass = 1.2f * volume;
  std::vector<float> F[5];
  std::vector<uint8_t> T;
  std::vector<float> B[7];
  auto axis = [&](int a) {
    float v = std::ceil((dmax[a] - dmin[a]) / spacing);
    return v > 0.0f ? (size_t)v : (size_t)0;
  };
  size_t nx = axis(0), ny = axis(1), nz = axis(2);
  // domain.rs:88-160
  float center_y = (dmin[1] + dmax[1]) * 0.5f;
  for (size_t i = 0; i < nx; ++i)
    for (size_t j = 0; j < ny; ++j)
      for (size_t k = 0; k < nz; ++k) {
        float x = dmin[0] + ((float)i + 0.5f) * spacing;
        float y = dmin[1] + ((float)j + 0.5f) * spacing;
        float z = dmin[2] + ((float)k + 0.5f) * spacing;
        if (x < dmin[0] || x > dmax[0] || y < dmin[1] || y > dmax[1] || z < dmin[2] || z > dmax[2]) continue;
        float pt[3] = {x, y, z};
        if (sdf_sample(d, dims, origin, cell, pt) < 0.0f) continue;
        bool water = fluid_type == 0 || (fluid_type == 2 && y < center_y);
        F[0].push_back(x);
        F[1].push_back(y);
        F[2].push_back(z);
        F[3].push_back(water ? water_mass : air_mass);
        F[4].push_back(water ? 1000.0f : 1.2f);
        T.push_back(water ? 0 : 1);
      }
  float mass = fluid_type == 1 ? air_mass : water_mass;  // domain.rs:60-66
  auto push = [&](float x, float y, float z, float a, float b, float c) {
    B[0].push_back(x); B[1].push_back(y); B[2].push_back(z); B[3].push_back(mass);
    B[4].push_back(a); B[5].push_back(b); B[6].push_back(c);
  };
  // domain.rs:189-347, face by face
  if (wall_faces & 1u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t j = 0; j < ny; ++j)
        for (size_t k = 0; k < nz; ++k)
          push(dmin[0] - ((float)l + 0.5f) * spacing, dmin[1] + ((float)j + 0.5f) * spacing,
               dmin[2] + ((float)k + 0.5f) * spacing, 1.0f, 0.0f, 0.0f);
  if (wall_faces & 2u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t j = 0; j < ny; ++j)
        for (size_t k = 0; k < nz; ++k)
          push(dmax[0] + ((float)l + 0.5f) * spacing, dmin[1] + ((float)j + 0.5f) * spacing,
               dmin[2] + ((float)k + 0.5f) * spacing, -1.0f, 0.0f, 0.0f);
  if (wall_faces & 4u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t i = 0; i < nx; ++i)
        for (size_t k = 0; k < nz; ++k)
          push(dmin[0] + ((float)i + 0.5f) * spacing, dmin[1] - ((float)l + 0.5f) * spacing,
               dmin[2] + ((float)k + 0.5f) * spacing, 0.0f, 1.0f, 0.0f);
  if (wall_faces & 8u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t i = 0; i < nx; ++i)
        for (size_t k = 0; k < nz; ++k)
          push(dmin[0] + ((float)i + 0.5f) * spacing, dmax[1] + ((float)l + 0.5f) * spacing,
               dmin[2] + ((float)k + 0.5f) * spacing, 0.0f, -1.0f, 0.0f);
  if (wall_faces & 16u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j)
          push(dmin[0] + ((float)i + 0.5f) * spacing, dmin[1] + ((float)j + 0.5f) * spacing,
               dmin[2] - ((float)l + 0.5f) * spacing, 0.0f, 0.0f, 1.0f);
  if (wall_faces & 32u)
    for (size_t l = 0; l < 3; ++l)
      for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j)
          push(dmin[0] + ((float)i + 0.5f) * spacing, dmin[1] + ((float)j + 0.5f) * spacing,
               dmax[2] + ((float)l + 0.5f) * spacing, 0.0f, 0.0f, -1.0f);
  // domain.rs:351-402
  float thr = spacing * 0.5f;
  for (size_t i = 0; i < nx; ++i)
    for (size_t j = 0; j < ny; ++j)
      for (size_t k = 0; k < nz; ++k) {
        float pt[3] = {dmin[0] + ((float)i + 0.5f) * spacing, dmin[1] + ((float)j + 0.5f) * spacing,
                       dmin[2] + ((float)k + 0.5f) * spacing};
        float dist = sdf_sample(d, dims, origin, cell, pt);
        if (dist > 0.0f && dist < thr) {
          float n[3];
          sdf_gradient(d, dims, origin, cell, pt, n);
          for (size_t l = 0; l < 3; ++l) {
            float off = ((float)l + 0.5f) * spacing;
            push(pt[0] - n[0] * off, pt[1] - n[1] * off, pt[2] - n[2] * off, n[0], n[1], n[2]);
          }
        }
      }
  counts[0] = T.size();
  counts[1] = B[0].size();
  float* fo[5] = {fx, fy, fz, fmass, fdens};
  for (int c = 0; c < 5; ++c)
    if (fo[c] && !F[c].empty()) std::memcpy(fo[c], F[c].data(), F[c].size() * 4);
  if (ftype && !T.empty()) std::memcpy(ftype, T.data(), T.size());
  float* bo[7] = {bx, by, bz, bmass_out, bnx, bny, bnz};
  for (int c = 0; c < 7; ++c)
    if (bo[c] && !B[c].empty()) std::memcpy(bo[c], B[c].data(), B[c].size() * 4);
}

// ---- GridSDF ------------------------------------------------------------
float orc_sdf_sample(const float* d, const uint32_t* dims, const float* origin, float cell,
                     const float* pt) {
  return sdf_sample(d, dims, origin, cell, pt);
}
void orc_sdf_gradient(const float* d, const uint32_t* dims, const float* origin, float cell,
                      const float* pt, float* out3) {
  sdf_gradient(d, dims, origin, cell, pt, out3);
}

}  // extern "C"
