// sph_domain.cu - the orchestrator's domain setup (orchestrator
// domain.rs:36-402) on the device.
//
// setup_domain walks the particle lattice of the domain box three times on
// the host: fluid placement (domain.rs:88-160, every lattice point inside the
// box and outside the geometry), wall layers (domain.rs:162-348, three
// layers behind each Wall face) and geometry layers (domain.rs:351-402,
// three layers along the inward SDF normal under every lattice point within
// half a spacing of the surface), sampling the GridSDF at every point. Here
// one thread takes one lattice point: a counting pass sums the fluid and
// surface points per block, one block scans the block sums, and an emit pass
// writes every kept point at its rank among the kept points, so the output
// order is the reference's loop order (x outermost, z innermost) without a
// sort. Wall layers have closed-form counts and are written directly. Every
// coordinate is the reference's f32 expression evaluated in the same order
// (the library is built without FMA contraction), so the particles are the
// reference's bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "sph_cuda.h"
#include "sph_sdf.cuh"

namespace {

constexpr int kThreads = 256;      // lattice points per block (count and emit passes)
constexpr int kScanThreads = 1024;  // the block-sum scan runs in one block

struct Lattice {
  float lo[3], hi[3], s;
  long long n[3];  // points per axis: ceil((hi - lo) / s) (domain.rs:105-107)
  long long total;
  float center_y;  // (lo.y + hi.y) * 0.5 (domain.rs:101)
  float thr;       // s * 0.5 (domain.rs:369)
  int fluid;       // SPH_FLUID_*
  float temperature;
  float water_mass, air_mass;
};

struct Grid {
  const float* d;
  float origin[3];
  float cell;
  int dims[3];
};

// lo + (i + 0.5) * s, the lattice coordinate (domain.rs:114-116)
__device__ __forceinline__ float coord(float lo, long long i, float s) { return lo + ((float)i + 0.5f) * s; }

struct Point {
  float p[3];
  float d;
  bool fluid, surface;
};

__device__ __forceinline__ Point classify(const Lattice& L, const Grid& g, long long t) {
  Point q;
  long long k = t % L.n[2], r = t / L.n[2];
  long long j = r % L.n[1], i = r / L.n[1];
  q.p[0] = coord(L.lo[0], i, L.s);
  q.p[1] = coord(L.lo[1], j, L.s);
  q.p[2] = coord(L.lo[2], k, L.s);
  q.d = sph::sdf_sample_exact(g.d, g.origin, g.cell, g.dims, q.p[0], q.p[1], q.p[2]);
  bool inside = !(q.p[0] < L.lo[0] || q.p[0] > L.hi[0] || q.p[1] < L.lo[1] || q.p[1] > L.hi[1] ||
                  q.p[2] < L.lo[2] || q.p[2] > L.hi[2]);
  q.fluid = inside && !(q.d < 0.0f);           // domain.rs:119-130
  q.surface = q.d > 0.0f && q.d < L.thr;       // domain.rs:383 (no box test there)
  return q;
}

__global__ void k_dom_count(Lattice L, Grid g, uint32_t* __restrict__ bf, uint32_t* __restrict__ bs) {
  long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
  bool f = false, s = false;
  if (t < L.total) {
    Point q = classify(L, g, t);
    f = q.fluid;
    s = q.surface;
  }
  int cf = __syncthreads_count(f);
  int cs = __syncthreads_count(s);
  if (threadIdx.x == 0) {
    bf[blockIdx.x] = (uint32_t)cf;
    bs[blockIdx.x] = (uint32_t)cs;
  }
}

// Exclusive scan of both block-count arrays in place, one block; totals in
// tot[0] (fluid) and tot[1] (surface points). Sums of counts of at most
// 2^31 lattice points fit 32 bits.
__global__ void k_dom_scan(int nb, uint32_t* __restrict__ bf, uint32_t* __restrict__ bs, uint32_t* __restrict__ tot) {
  __shared__ uint32_t sf[kScanThreads], ss[kScanThreads];
  int per = (nb + kScanThreads - 1) / kScanThreads;
  int a = threadIdx.x * per, b = min(a + per, nb);
  uint32_t f = 0, s = 0;
  for (int u = a; u < b; ++u) {
    f += bf[u];
    s += bs[u];
  }
  sf[threadIdx.x] = f;
  ss[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < kScanThreads; off <<= 1) {  // inclusive Hillis-Steele
    uint32_t xf = threadIdx.x >= off ? sf[threadIdx.x - off] : 0u;
    uint32_t xs = threadIdx.x >= off ? ss[threadIdx.x - off] : 0u;
    __syncthreads();
    sf[threadIdx.x] += xf;
    ss[threadIdx.x] += xs;
    __syncthreads();
  }
  uint32_t of = sf[threadIdx.x] - f, os = ss[threadIdx.x] - s;
  for (int u = a; u < b; ++u) {
    uint32_t cf = bf[u], cs = bs[u];
    bf[u] = of;
    bs[u] = os;
    of += cf;
    os += cs;
  }
  if (threadIdx.x == kScanThreads - 1) {
    tot[0] = sf[threadIdx.x];
    tot[1] = ss[threadIdx.x];
  }
}

struct FluidOut {
  float *x, *y, *z, *mass, *density;
  uint8_t* type;
};
struct WallOut {
  float *x, *y, *z, *mass, *nx, *ny, *nz;
};

__device__ __forceinline__ void put_wall(const WallOut& o, long long r, float x, float y, float z, float m, float nx,
                                         float ny, float nz) {
  o.x[r] = x;
  o.y[r] = y;
  o.z[r] = z;
  o.mass[r] = m;
  o.nx[r] = nx;
  o.ny[r] = ny;
  o.nz[r] = nz;
}

__global__ void k_dom_emit(Lattice L, Grid g, const uint32_t* __restrict__ bf, const uint32_t* __restrict__ bs,
                           long long surf_base, float bmass, FluidOut fo, WallOut wo) {
  __shared__ uint32_t wf[kThreads / 32], ws[kThreads / 32];
  long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
  Point q;
  q.fluid = q.surface = false;
  if (t < L.total) q = classify(L, g, t);
  unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  unsigned mf = __ballot_sync(0xffffffffu, q.fluid), ms = __ballot_sync(0xffffffffu, q.surface);
  if (lane == 0) {
    wf[w] = __popc(mf);
    ws[w] = __popc(ms);
  }
  __syncthreads();
  uint32_t rf = bf[blockIdx.x], rs = bs[blockIdx.x];
  for (unsigned u = 0; u < w; ++u) {
    rf += wf[u];
    rs += ws[u];
  }
  unsigned below = (1u << lane) - 1u;
  if (q.fluid) {  // domain.rs:133-157
    uint32_t r = rf + __popc(mf & below);
    bool water = L.fluid == SPH_FLUID_WATER || (L.fluid == SPH_FLUID_MIXED && q.p[1] < L.center_y);
    fo.x[r] = q.p[0];
    fo.y[r] = q.p[1];
    fo.z[r] = q.p[2];
    fo.mass[r] = water ? L.water_mass : L.air_mass;
    fo.density[r] = water ? 1000.0f : 1.2f;
    fo.type[r] = water ? 0 : 1;
  }
  if (q.surface) {  // domain.rs:384-398
    long long r = surf_base + 3ll * (long long)(rs + __popc(ms & below));
    float n[3];
    sph::sdf_gradient_exact(g.d, g.origin, g.cell, g.dims, q.p[0], q.p[1], q.p[2], n);
    for (int layer = 0; layer < 3; ++layer) {
      float off = ((float)layer + 0.5f) * L.s;
      put_wall(wo, r + layer, q.p[0] - n[0] * off, q.p[1] - n[1] * off, q.p[2] - n[2] * off, bmass, n[0], n[1],
               n[2]);
    }
  }
}

// Three layers behind face `face` (0..5 = x_min, x_max, y_min, y_max, z_min,
// z_max; domain.rs:189-347): layer outermost, then the face's first and
// second in-plane axes, as the reference's loops run.
__global__ void k_dom_walls(Lattice L, int face, long long base, float bmass, WallOut wo) {
  int axis = face >> 1;
  bool upper = face & 1;
  int a0 = axis == 0 ? 1 : 0, a1 = axis == 2 ? 1 : 2;  // in-plane axes, outer then inner
  long long na = L.n[a0], nb = L.n[a1], per = na * nb;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * per) return;
  int layer = (int)(t / per);
  long long r = t % per, ia = r / nb, ib = r % nb;
  float off = ((float)layer + 0.5f) * L.s;
  float p[3], nrm[3] = {0.0f, 0.0f, 0.0f};
  p[a0] = coord(L.lo[a0], ia, L.s);
  p[a1] = coord(L.lo[a1], ib, L.s);
  p[axis] = upper ? L.hi[axis] + off : L.lo[axis] - off;
  nrm[axis] = upper ? -1.0f : 1.0f;
  put_wall(wo, base + t, p[0], p[1], p[2], bmass, nrm[0], nrm[1], nrm[2]);
}

__global__ void k_fill(float* __restrict__ p, long long n, float v) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return SPH_OK;
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
}

// ceil((hi - lo) / s) as usize (f32 arithmetic; negative or NaN -> 0)
long long axis_points(float lo, float hi, float s) {
  float v = std::ceil((hi - lo) / s);
  return v > 0.0f ? (long long)v : 0ll;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Constant fields of the output: a kernel for device memory, a loop for host
// memory (nothing crosses the bus for them).
cudaError_t fill(float* dst, size_t n, float v, cudaStream_t st) {
  if (!n) return cudaSuccess;
  if (is_device_ptr(dst)) {
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, (long long)n, v);
    return cudaGetLastError();
  }
  std::fill(dst, dst + n, v);
  return cudaSuccess;
}

struct Scratch {
  std::vector<void*> ptrs;
  cudaStream_t st = nullptr;
  template <class T>
  cudaError_t alloc(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return e;
  }
  ~Scratch() {
    if (st) cudaStreamSynchronize(st);
    for (void* p : ptrs) cudaFree(p);
    if (st) cudaStreamDestroy(st);
  }
};

}  // namespace

int sph_setup_domain(int device, const SphDomainSpec* spec, const SphSdfView* sdf, SphParticlesMut* fluid,
                     SphBoundaryMut* boundary, size_t* n_fluid, size_t* n_boundary) {
  if (!spec || !sdf || !sdf->distances || !n_fluid || !n_boundary) return SPH_ERR_INVALID_ARG;
  const SphDomainSpec& S = *spec;
  if (!(S.particle_spacing > 0.0f) || !std::isfinite(S.particle_spacing)) return SPH_ERR_INVALID_ARG;
  if (S.fluid_type < SPH_FLUID_WATER || S.fluid_type > SPH_FLUID_MIXED || (S.wall_faces & ~0x3fu))
    return SPH_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(S.domain_min[a]) || !std::isfinite(S.domain_max[a])) return SPH_ERR_INVALID_ARG;
  if (!(sdf->cell_size > 0.0f) || sdf->dims[0] < 1 || sdf->dims[1] < 1 || sdf->dims[2] < 1 ||
      sdf->dims[0] > 0x7fffffffu || sdf->dims[1] > 0x7fffffffu || sdf->dims[2] > 0x7fffffffu)
    return SPH_ERR_INVALID_ARG;
  if (fluid && (!fluid->x || !fluid->y || !fluid->z || !fluid->vx || !fluid->vy || !fluid->vz || !fluid->ax ||
                !fluid->ay || !fluid->az || !fluid->density || !fluid->pressure || !fluid->mass ||
                !fluid->temperature || !fluid->fluid_type))
    return SPH_ERR_INVALID_ARG;
  if (boundary && (!boundary->x || !boundary->y || !boundary->z || !boundary->mass || !boundary->nx ||
                   !boundary->ny || !boundary->nz))
    return SPH_ERR_INVALID_ARG;

  Lattice L;
  L.s = S.particle_spacing;
  for (int a = 0; a < 3; ++a) {
    L.lo[a] = S.domain_min[a];
    L.hi[a] = S.domain_max[a];
    L.n[a] = axis_points(L.lo[a], L.hi[a], L.s);
  }
  if (L.n[0] > 0x7fffffffll || L.n[1] > 0x7fffffffll || L.n[2] > 0x7fffffffll) return SPH_ERR_INVALID_ARG;
  L.total = L.n[0] * L.n[1] * L.n[2];
  if (L.total > 0x7fffffffll) return SPH_ERR_INVALID_ARG;
  L.center_y = (L.lo[1] + L.hi[1]) * 0.5f;
  L.thr = L.s * 0.5f;
  L.fluid = S.fluid_type;
  L.temperature = S.initial_temperature;
  float vol = L.s * (L.s * L.s);  // spacing.powi(3) (domain.rs:43)
  L.water_mass = 1000.0f * vol;
  L.air_mass = 1.2f * vol;
  float bmass = S.fluid_type == SPH_FLUID_AIR ? L.air_mass : L.water_mass;  // domain.rs:60-66

  long long wall_base[7] = {0};
  for (int f = 0; f < 6; ++f) {
    int axis = f >> 1;
    long long per = (S.wall_faces >> f) & 1u ? L.n[axis == 0 ? 1 : 0] * L.n[axis == 2 ? 1 : 2] : 0;
    wall_base[f + 1] = wall_base[f] + 3 * per;
  }

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess || major != 10) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return status_of(cudaErrorInvalidDevice);

  Scratch sc;
  cudaError_t e = cudaStreamCreateWithFlags(&sc.st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return status_of(e);
  Grid g;
  size_t nodes = (size_t)sdf->dims[0] * sdf->dims[1] * sdf->dims[2];
  float* dsdf = nullptr;
  int nb = (int)((L.total + kThreads - 1) / kThreads);
  uint32_t *bf = nullptr, *bs = nullptr, *tot = nullptr;
  if (e == cudaSuccess) e = sc.alloc(&dsdf, nodes);
  if (e == cudaSuccess) e = sc.alloc(&bf, nb);
  if (e == cudaSuccess) e = sc.alloc(&bs, nb);
  if (e == cudaSuccess) e = sc.alloc(&tot, 2);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dsdf, sdf->distances, nodes * sizeof(float), cudaMemcpyDefault, sc.st);
  if (e != cudaSuccess) return status_of(e);
  g.d = dsdf;
  g.cell = sdf->cell_size;
  for (int a = 0; a < 3; ++a) {
    g.origin[a] = sdf->origin[a];
    g.dims[a] = (int)sdf->dims[a];
  }

  uint32_t htot[2] = {0u, 0u};
  if (nb > 0) {
    k_dom_count<<<nb, kThreads, 0, sc.st>>>(L, g, bf, bs);
    k_dom_scan<<<1, kScanThreads, 0, sc.st>>>(nb, bf, bs, tot);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(htot, tot, sizeof(htot), cudaMemcpyDeviceToHost, sc.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc.st);
    if (e != cudaSuccess) return status_of(e);
  }
  size_t nf = htot[0];
  long long surf_base = wall_base[6];
  size_t nbt = (size_t)surf_base + 3ull * htot[1];
  *n_fluid = nf;
  *n_boundary = nbt;
  if (!fluid && !boundary) return SPH_OK;
  if ((fluid && fluid->n < nf) || (boundary && boundary->n < nbt)) return SPH_ERR_CAPACITY;

  FluidOut fo;
  WallOut wo;
  float* fbuf = nullptr;
  float* wbuf = nullptr;
  uint8_t* tbuf = nullptr;
  e = sc.alloc(&fbuf, 5 * nf);
  if (e == cudaSuccess) e = sc.alloc(&tbuf, nf);
  if (e == cudaSuccess) e = sc.alloc(&wbuf, 7 * nbt);
  if (e != cudaSuccess) return status_of(e);
  fo = {fbuf, fbuf + nf, fbuf + 2 * nf, fbuf + 3 * nf, fbuf + 4 * nf, tbuf};
  wo = {wbuf, wbuf + nbt, wbuf + 2 * nbt, wbuf + 3 * nbt, wbuf + 4 * nbt, wbuf + 5 * nbt, wbuf + 6 * nbt};
  for (int f = 0; f < 6; ++f) {
    long long cnt = wall_base[f + 1] - wall_base[f];
    if (cnt > 0)
      k_dom_walls<<<(unsigned)((cnt + 255) / 256), 256, 0, sc.st>>>(L, f, wall_base[f], bmass, wo);
  }
  if (nb > 0) k_dom_emit<<<nb, kThreads, 0, sc.st>>>(L, g, bf, bs, surf_base, bmass, fo, wo);
  e = cudaGetLastError();

  auto copy = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, sc.st);
  };
  if (fluid) {
    copy(fluid->x, fo.x, nf * 4);
    copy(fluid->y, fo.y, nf * 4);
    copy(fluid->z, fo.z, nf * 4);
    copy(fluid->mass, fo.mass, nf * 4);
    copy(fluid->density, fo.density, nf * 4);
    copy(fluid->fluid_type, fo.type, nf);
    // push_particle (kernel particle.rs:96-120): zero velocity, acceleration
    // and pressure, the configured temperature
    float* zeros[7] = {fluid->vx, fluid->vy, fluid->vz, fluid->ax, fluid->ay, fluid->az, fluid->pressure};
    for (float* z : zeros)
      if (e == cudaSuccess) e = fill(z, nf, 0.0f, sc.st);
    if (e == cudaSuccess) e = fill(fluid->temperature, nf, L.temperature, sc.st);
  }
  if (boundary) {
    float* dst[7] = {boundary->x, boundary->y, boundary->z, boundary->mass, boundary->nx, boundary->ny, boundary->nz};
    const float* src[7] = {wo.x, wo.y, wo.z, wo.mass, wo.nx, wo.ny, wo.nz};
    for (int c = 0; c < 7; ++c) copy(dst[c], src[c], nbt * 4);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(sc.st);
  return status_of(e);
}
