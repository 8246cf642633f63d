// sph_api.cu - host side of libsph_cuda.so: the C ABI of include/sph_cuda.h.
//
// One SphHandle = one simulation on one device: its own stream, device
// buffers and CUDA graphs. The step body (9 kernels) is captured once into a
// graph and replayed; dt lives in device memory so the graph never changes.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_bf16.h>

#include "sph_cuda.h"
#include "sph_kernels.cuh"

using sph::SimConst;

namespace {

constexpr float kPiF = 3.14159265358979323846f;

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

inline int grid_for(long long n, int block) { return (int)((n + block - 1) / block); }

}  // namespace

struct SphHandle {
  int dev = 0;
  cudaStream_t st = nullptr;
  SphParams prm{};
  SimConst k{};  // constants of instance 0 (the simulation, for a single one)
  int n = 0, nb = 0, C = 0;
  // batch: instances, their constants on the device, the instance of every
  // particle slot and boundary particle, (h, c, cfl) for the dt finalize
  int ninst = 1;
  std::vector<SimConst> ktab_h;
  SimConst* ktab = nullptr;
  uint16_t *inst_p = nullptr, *inst_b = nullptr;
  float4* hcc = nullptr;
  std::vector<size_t> poff, boff;
  std::vector<double> init_e, init_m;
  // launch shapes (threads per block of the neighbour kernels)
  // threads per block of the neighbour kernels (sph_set_launch / sph_autotune
  // change them): the fastest shapes measured on the 2M dam break
  int bs_xsph = 128, bs_density = 128, bs_forces = 128;
  std::vector<float> temperature;
  double init_energy = 0.0, init_mass = 0.0;
  bool needs_init = true;
  bool red_valid = false;
  bool has_ck = false;
  bool list_valid = false;  // nbr holds the in-support lists of the current grid/positions
  uint64_t launches = 0;
  int body_kernels = 0;
  uint64_t boundary_candidates = 0;
  std::string error;

  // sorted state
  float4 *pos = nullptr, *vel = nullptr, *velout = nullptr, *acc = nullptr;
  float2 *rv = nullptr, *rf = nullptr;
  float* pr = nullptr;
  uint32_t* id = nullptr;
  // unsorted (post-drift) state and sort scratch
  float4 *posU = nullptr, *velU = nullptr;
  uint32_t *idU = nullptr, *keyU = nullptr, *tmp = nullptr, *tmpid = nullptr;
  uint32_t *hist = nullptr, *cstart = nullptr, *ccount = nullptr, *cursor = nullptr, *bsum = nullptr;
  uint32_t *rank_of_lin = nullptr, *lin_of_rank = nullptr;
  uint2* ctab = nullptr;
  int nbsum = 0;
  // neighbour lists recorded by k_density (entry-major, sph::nbr_index), count per particle
  uint32_t *nbr = nullptr, *ncount = nullptr;
  // XSPH gather records: (x, y, z, m), (v + a dt/2, rho) per particle
  float4* xrec = nullptr;
  float* xyz = nullptr;     // sorted positions as x | y | z planes (the density scan's candidates)
  size_t xyz_stride = 0;
  // viewer frames (sph_pack_frame): temperature on the device (uploaded on
  // the first call) and the packed particle records
  float* temp_dev = nullptr;
  uint32_t* frame_dev = nullptr;
  size_t frame_cap = 0;
  // optimistic runner (sph_run_optimistic): state on the device, one graph
  // per parameter set, kernels per launch of its main part and retry branch
  sph::RunState* run = nullptr;
  float* dt_safe_dev = nullptr;
  cudaGraphExec_t g_opt = nullptr;
  float opt_alpha = 0.0f, opt_limit = 0.0f;
  uint32_t opt_cool = 0;
  int opt_kernels = 0, retry_kernels = 0;
  unsigned long long opt_rejected_counted = 0;
  // boundary
  float4* bpos = nullptr;
  float* bpress = nullptr;
  uint8_t* bact = nullptr;  // per boundary particle: an occupied cell lists it (k_adami_mark)
  uint32_t* bc_cells = nullptr;  // the linear cells whose boundary candidate list is not empty
  int nbc_cells = 0;
  // the boundary particles sorted by the (global) cell that holds them, for
  // k_adami_cells; used when every instance is in the row or linear order
  uint32_t* border = nullptr;
  bool adami_cells = false;
  int pool = -1;  // device arrays from the library's pool (1) or cudaMalloc (0); set by the first one
  // Below these sizes the per-particle forms of the density scan and of the
  // boundary pressure run instead of the warp-cooperative ones: a warp per 32
  // particles (or boundary particles) then leaves the SMs too few warps to
  // hide the longer per-warp chains. Set at creation from the SM count.
  int warp_scan_min = 0;
  size_t adami_cells_min = 0;
  uint32_t *bc_start = nullptr, *bc_list = nullptr;
  // SDF node grid and wall table (boundary_mode SPH_BOUNDARY_SDF), or the
  // geometry SDF(s) of the closure features
  float* sdf = nullptr;
  float2* wall_tab = nullptr;
  // learned closure: 0 off, 1 capture features, 2 capture and apply
  int cl_mode = 0;
  uint32_t *cl_count = nullptr, *cl_slot = nullptr;
  float *cl_feat = nullptr, *cl_rho = nullptr, *cl_wf = nullptr;
  float4* corr = nullptr;
  __nv_bfloat16* cl_wb = nullptr;
  // scalars
  float *dt = nullptr, *dt_query = nullptr, *red = nullptr;
  uint32_t* err = nullptr;
  // metrics
  int nparts = 0;
  double *part_m = nullptr, *part_e = nullptr, *me = nullptr;
  float *part_var = nullptr, *var = nullptr;
  unsigned long long* bad = nullptr;
  // checkpoint
  float4 *ck_pos = nullptr, *ck_velout = nullptr, *ck_acc = nullptr;
  float* ck_pr = nullptr;
  uint32_t* ck_slot = nullptr;
  // readback staging
  float* stage = nullptr;
  uint8_t* stage_ft = nullptr;
  // diagnostics scratch
  uint32_t* diag = nullptr;
  // geometry for force extraction
  float4 *geo_pos = nullptr, *geo_nrm = nullptr;
  float* geo_out = nullptr;
  double* geo_sum = nullptr;
  int geo_nodes = 0;
  float geo_area = 0.0f;
  double* body_part = nullptr;
  double* body_sum = nullptr;
  int body_parts = 0;
  // graphs
  cudaGraphExec_t g_step = nullptr;
  cudaGraphExec_t g_auto = nullptr;
  std::vector<void*> allocs;
};

namespace {

int set_err(SphHandle* h, int code, const std::string& msg) {
  if (h) h->error = msg;
  return code;
}

int cuda_status(SphHandle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SPH_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return set_err(h, SPH_ERR_OOM, m);
  return set_err(h, SPH_ERR_CUDA, m);
}

#define SPH_TRY(h, call)                                   \
  do {                                                     \
    cudaError_t _e = (call);                               \
    if (_e != cudaSuccess) return cuda_status(h, _e, #call); \
  } while (0)

// The handles' device arrays come from one memory pool per device, owned by
// this library, in stream order on the handle's stream. The pool keeps what
// a closed handle frees (release threshold: unlimited), so a process that
// creates simulations one after another reuses mapped memory instead of
// asking the driver to map it again each time; the memory stays reserved for
// this library until the process exits.
cudaMemPool_t device_pool(int dev) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = pool;
  return pool;
}

template <class T>
cudaError_t dalloc(SphHandle* h, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  if (h->pool < 0) h->pool = (h->st && device_pool(h->dev)) ? 1 : 0;  // fixed for the handle's life
  cudaError_t e = h->pool ? cudaMallocFromPoolAsync((void**)p, count * sizeof(T), device_pool(h->dev), h->st)
                          : cudaMalloc((void**)p, count * sizeof(T));
  if (e == cudaSuccess) h->allocs.push_back((void*)*p);
  return e;
}

uint64_t spread21(uint64_t v) {
  uint64_t r = 0;
  for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
  return r;
}
uint64_t spread2(uint64_t v) {  // 21 bits to every second bit
  uint64_t r = 0;
  for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (2 * b);
  return r;
}

// Largest float t with sqrtf(t) < s (sqrtf is correctly rounded on host and
// device, and monotone), so that sqrtf(d2) < s  <=>  d2 <= t.
float sqrt_below(float s) {
  float t = s * s;
  while (t > 0.0f && !(std::sqrt(t) < s)) t = std::nextafter(t, 0.0f);
  while (std::sqrt(std::nextafter(t, INFINITY)) < s) t = std::nextafter(t, INFINITY);
  return t;
}

// Largest float t with sqrtf(t) <= s, so that sqrtf(d2) > s  <=>  d2 > t.
float sqrt_at_most(float s) {
  float t = s * s;
  while (t > 0.0f && !(std::sqrt(t) <= s)) t = std::nextafter(t, 0.0f);
  while (std::sqrt(std::nextafter(t, INFINITY)) <= s) t = std::nextafter(t, INFINITY);
  return t;
}

// Step constants rounded in f32 as the reference evaluates them.
SimConst make_const(const SphParams& p, const uint32_t dims[3]) {
  SimConst k{};
  float h = p.h;
  k.h = h;
  volatile float one = 1.0f;
  k.inv_h = one / h;  // RN(1/h), the divisor's reciprocal for sph::div_h
  k.support = 2.0f * h;
  k.radius_sq = k.support * k.support;
  k.cell = 2.0f * h;
  for (int a = 0; a < 3; ++a) {
    k.gmin[a] = p.domain_min[a];
    k.dims[a] = (int)dims[a];
    k.grav[a] = p.gravity[a];
    k.dmin[a] = p.domain_min[a];
    k.dmax[a] = p.domain_max[a];
  }
  volatile float norm = 21.0f / (16.0f * kPiF);
  float h3 = h * h * h;
  k.norm_h3 = norm / h3;
  k.norm_h4 = norm / (h3 * h);
  k.eta_sq = 0.01f * h * h;
  k.delta_coef = 0.1f * h * p.speed_of_sound;
  k.neg_alpha_c = -p.alpha * p.speed_of_sound;
  k.beta = p.beta;
  k.b_water = 1000.0f * p.speed_of_sound * p.speed_of_sound / 7.0f;
  k.b_air = 1.204f * p.speed_of_sound * p.speed_of_sound / 1.4f;
  k.r0 = 0.5f * h;
  volatile float ten = 10.0f;
  k.rep_d = ten * 9.81f * 0.01f;
  k.c = p.speed_of_sound;
  k.reach = (float)(2.0 * (double)h * (1.0 + 1e-4) + 1e-4 * (double)k.cell);
  k.sdf_coef = p.sdf_wall_coef;
  k.flags = p.flags;
  k.sup_d2 = sqrt_below(k.support);
  k.r0_d2 = sqrt_below(k.r0);
  k.tiny_d2 = sqrt_at_most(1.0e-12f);
  return k;
}

// SDF wall table: for a particle at distance d in front of a plane wall, the
// sums over the reference's 3 wall layers (depths (layer + 0.5) dx, lattice
// spacing dx = h / 1.3, orchestrator domain.rs:162-348) of W dx^3 and of
// -dW/dn dx^3, averaged over 8 x 8 lateral lattice offsets, at kWallN + 1
// distances on [0, 2h]; evaluated in double and rounded to f32.
std::vector<float2> make_wall_table(float hf, float* inv_step) {
  const int N = sph::kWallN;
  std::vector<float2> t(N + 1);
  const double h = hf, dx = h / 1.3, sup = 2.0 * h;
  const double C0 = 21.0 / (16.0 * 3.14159265358979323846);
  const int M = (int)std::ceil(sup / dx) + 1;
  for (int k = 0; k <= N; ++k) {
    double d = (double)k * (sup / N);
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
    t[k] = make_float2((float)(sw * vol), (float)(sg * vol));
  }
  *inv_step = (float)((double)N / sup);
  return t;
}

// Edge and corner tables of the SDF wall (appended to the slab table at
// kWallOff2 and kWallOff3): where the 3-layer slabs of two (three) box faces
// meet, their common wall sites (depths (la + 0.5) dx, (lb + 0.5) dx
// [, (lc + 0.5) dx] beyond the faces) are counted once per slab, so the box
// walls are sum(slabs) - sum(edge columns) + corner cube. Edge: W and the
// gradient along the first face's normal, averaged over 8 offsets along the
// edge, at (d_a, d_b) on a (kWallN2 + 1)^2 grid of [0, 2h]^2. Corner: the 27
// sites, at (d_a, d_b, d_c) on a (kWallN3 + 1)^3 grid.
std::vector<float2> make_wall_tables(float hf, float* inv1, float* inv2, float* inv3) {
  std::vector<float2> t = make_wall_table(hf, inv1);
  t.resize(sph::kWallTabSize);
  const double h = hf, dx = h / 1.3, sup = 2.0 * h;
  const double C0 = 21.0 / (16.0 * 3.14159265358979323846);
  const int M = (int)std::ceil(sup / dx) + 1;
  auto w_and_dw = [&](double r, double& w, double& dw) {  // W and -dW/dr
    double q = r / h, om = 1.0 - 0.5 * q;
    w = C0 / (h * h * h) * om * om * om * om * (1.0 + 2.0 * q);
    dw = C0 / (h * h * h * h) * 5.0 * q * om * om * om;
  };
  const int N2 = sph::kWallN2, N3 = sph::kWallN3;
  for (int i = 0; i <= N2; ++i)
    for (int j = 0; j <= N2; ++j) {
      double da = (double)i * (sup / N2), db = (double)j * (sup / N2);
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
      t[sph::kWallOff2 + i * (N2 + 1) + j] = make_float2((float)(sw * vol), (float)(sg * vol));
    }
  for (int i = 0; i <= N3; ++i)
    for (int j = 0; j <= N3; ++j)
      for (int l = 0; l <= N3; ++l) {
        double da = (double)i * (sup / N3), db = (double)j * (sup / N3), dc = (double)l * (sup / N3);
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
        t[sph::kWallOff3 + (i * (N3 + 1) + j) * (N3 + 1) + l] = make_float2((float)(sw * vol), (float)(sg * vol));
      }
  *inv2 = (float)((double)N2 / sup);
  *inv3 = (float)((double)N3 / sup);
  return t;
}

// Mass of the homogenised wall layers relative to rho0 (h / 1.3)^3: the
// walls carry the mass of the first water particle (the reference gives wall
// particles the water particle mass, orchestrator/src/domain.rs:57-62).
// Within 1e-5 of 1 (mass rho0 dx^3 with h = 1.3 dx, up to f32 rounding) it
// is exactly 1.
float wall_mass_scale(float hf, const SphParticlesView* pv) {
  size_t i = 0;
  while (i < pv->n && pv->fluid_type && pv->fluid_type[i] != 0) ++i;
  if (i == pv->n || !pv->mass) return 1.0f;
  double dx = (double)hf / 1.3;
  double s = (double)pv->mass[i] / (1000.0 * dx * dx * dx);
  return std::fabs(s - 1.0) < 1e-5 ? 1.0f : (float)s;
}

// GridSDF::sample and ::gradient (orchestrator geometry.rs:99-181), f32.
float host_sdf_get(const SphSdfView& g, int i, int j, int k) {
  uint64_t idx = (uint64_t)((uint32_t)i * g.dims[1] * g.dims[2] + (uint32_t)j * g.dims[2] + (uint32_t)k);
  uint64_t total = (uint64_t)g.dims[0] * g.dims[1] * g.dims[2];
  return idx < total ? g.distances[idx] : 3.40282347e38f;
}
float host_sdf_sample(const SphSdfView& g, float px, float py, float pz) {
  float gx = (px - g.origin[0]) / g.cell_size, gy = (py - g.origin[1]) / g.cell_size;
  float gz = (pz - g.origin[2]) / g.cell_size;
  int i0 = (int)std::floor(gx), j0 = (int)std::floor(gy), k0 = (int)std::floor(gz);
  if (i0 < 0 || j0 < 0 || k0 < 0) return 3.40282347e38f;
  int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  if (i1 >= (int)g.dims[0] || j1 >= (int)g.dims[1] || k1 >= (int)g.dims[2]) return 3.40282347e38f;
  float fx = gx - (float)i0, fy = gy - (float)j0, fz = gz - (float)k0;
  float c00 = host_sdf_get(g, i0, j0, k0) * (1.0f - fz) + host_sdf_get(g, i0, j0, k1) * fz;
  float c01 = host_sdf_get(g, i0, j1, k0) * (1.0f - fz) + host_sdf_get(g, i0, j1, k1) * fz;
  float c10 = host_sdf_get(g, i1, j0, k0) * (1.0f - fz) + host_sdf_get(g, i1, j0, k1) * fz;
  float c11 = host_sdf_get(g, i1, j1, k0) * (1.0f - fz) + host_sdf_get(g, i1, j1, k1) * fz;
  float c0 = c00 * (1.0f - fy) + c01 * fy;
  float c1 = c10 * (1.0f - fy) + c11 * fy;
  return c0 * (1.0f - fx) + c1 * fx;
}
void host_sdf_gradient(const SphSdfView& g, float px, float py, float pz, float out[3]) {
  float h = g.cell_size * 0.5f;
  float dx = (host_sdf_sample(g, px + h, py, pz) - host_sdf_sample(g, px - h, py, pz)) / (2.0f * h);
  float dy = (host_sdf_sample(g, px, py + h, pz) - host_sdf_sample(g, px, py - h, pz)) / (2.0f * h);
  float dz = (host_sdf_sample(g, px, py, pz + h) - host_sdf_sample(g, px, py, pz - h)) / (2.0f * h);
  float mag = std::sqrt(dx * dx + dy * dy + dz * dz);
  if (mag > 1e-8f) { out[0] = dx / mag; out[1] = dy / mag; out[2] = dz / mag; }
  else { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; }
}

// Static per-cell candidate lists of boundary particles, ascending index. A
// boundary particle is listed for every cell whose box (widened by a margin
// above the rounding of pos_to_cell, unbounded outward on edge cells) comes
// within 2h (plus margin): a superset of the particles in support.
// f(t, begin, end) on up to `max_threads` host threads over [0, n) in
// contiguous chunks, chunk t on thread t; small ranges run inline.
template <class F>
void parallel_chunks(size_t n, unsigned max_threads, F&& f) {
  unsigned T = std::max(1u, std::min(max_threads, std::thread::hardware_concurrency()));
  if (n < 65536 || T == 1) {
    f(0u, (size_t)0, n);
    return;
  }
  size_t chunk = (n + T - 1) / T;
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < T; ++t) {
    size_t a = (size_t)t * chunk, e = std::min(n, a + chunk);
    if (a >= e) break;
    try {
      ts.emplace_back([&f, t, a, e] { f(t, a, e); });
    } catch (...) {  // no thread to be had: this chunk runs here
      f(t, a, e);
    }
  }
  for (std::thread& th : ts) th.join();
}
constexpr unsigned kHostThreads = 32;
// f(t) for t < T, one host thread each (inline when T == 1)
template <class F>
void run_threads(unsigned T, F&& f) {
  if (T <= 1) {
    if (T == 1) f(0u);
    return;
  }
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < T; ++t) {
    try {
      ts.emplace_back([&f, t] { f(t); });
    } catch (...) {  // no thread to be had: this part runs here
      f(t);
    }
  }
  for (std::thread& th : ts) th.join();
}

// Per linear cell, the boundary particles whose support can reach a particle
// in that cell, in ascending boundary index (CSR: start[C + 1], list). Host
// threads take contiguous ranges of boundary particles; each cell's entries
// are laid out thread by thread, so the order is ascending as with one thread.
void build_boundary_lists(const SimConst& k, const SphBoundaryView* b, int C,
                          std::vector<uint32_t>& start, std::vector<uint32_t>& list) {
  start.assign((size_t)C + 1, 0);
  list.clear();
  if (!b || b->n == 0) return;
  double cs = k.cell, margin = 1e-4 * cs;
  double reach = 2.0 * (double)k.h * (1.0 + 1e-4) + margin;
  // per-thread cell counts cost C words per thread: bound their memory
  unsigned T = (unsigned)std::max<size_t>(1, std::min<size_t>(kHostThreads, ((size_t)64 << 20) / ((size_t)C + 1)));
  std::vector<std::vector<uint64_t>> pairs(T);  // (cell << 32) | b, per thread
  unsigned used = 0;
  std::mutex mu;
  parallel_chunks(b->n, T, [&](unsigned t, size_t first, size_t last) {
    std::vector<uint64_t>& out = pairs[t];
    out.reserve((last - first) * 12);
    for (size_t bi = first; bi < last; ++bi) {
      double pos[3] = {b->x[bi], b->y[bi], b->z[bi]};
      int lo[3], hi[3];
      bool empty = false;
      for (int a = 0; a < 3; ++a) {
        double u0 = std::floor((pos[a] - reach - k.gmin[a]) / cs);
        double u1 = std::floor((pos[a] + reach - k.gmin[a]) / cs);
        lo[a] = (int)std::max(0.0, std::min((double)k.dims[a] - 1, u0));
        hi[a] = (int)std::max(0.0, std::min((double)k.dims[a] - 1, u1));
        if (!(pos[a] == pos[a])) empty = true;
      }
      if (empty) continue;
      // squared distance from the particle to each candidate cell's slab, per
      // axis (a cell's box is widened by `margin`, edge cells unbounded
      // outward); a cell's d2 is their sum, x + y + z in that order
      double e2[3][8];
      for (int a = 0; a < 3; ++a)
        for (int c = lo[a]; c <= hi[a] && c - lo[a] < 8; ++c) {
          double blo = c == 0 ? -1e300 : k.gmin[a] + c * cs - margin;
          double bhi = c == k.dims[a] - 1 ? 1e300 : k.gmin[a] + (c + 1) * cs + margin;
          double d = pos[a] < blo ? blo - pos[a] : (pos[a] > bhi ? pos[a] - bhi : 0.0);
          e2[a][c - lo[a]] = d * d;
        }
      for (int cz = lo[2]; cz <= hi[2]; ++cz)
        for (int cy = lo[1]; cy <= hi[1]; ++cy) {
          const double ezy = e2[1][cy - lo[1]];
          const uint64_t row = (uint64_t)cy * k.dims[0] + (uint64_t)cz * k.dims[0] * k.dims[1];
          for (int cx = lo[0]; cx <= hi[0]; ++cx) {
            const double d2 = (e2[0][cx - lo[0]] + ezy) + e2[2][cz - lo[2]];
            if (d2 < reach * reach) out.push_back(((row + (uint64_t)cx) << 32) | (uint64_t)bi);
          }
        }
    }
    std::lock_guard<std::mutex> lock(mu);
    used = std::max(used, t + 1);
  });
  // per-thread counts (each thread zeroes and fills its own array), per-cell
  // totals in parallel, one scan, then per-thread write offsets within each cell
  std::vector<std::vector<uint32_t>> at(used);
  run_threads(used, [&](unsigned t) {
    at[t].assign((size_t)C, 0u);
    for (uint64_t pr : pairs[t]) at[t][pr >> 32]++;
  });
  parallel_chunks((size_t)C, kHostThreads, [&](unsigned, size_t c0, size_t c1) {
    for (size_t c = c0; c < c1; ++c) {
      uint32_t run = 0;
      for (unsigned t = 0; t < used; ++t) run += at[t][c];
      start[c + 1] = run;
    }
  });
  for (int c = 0; c < C; ++c) start[(size_t)c + 1] += start[c];
  list.resize(start[C]);
  parallel_chunks((size_t)C, kHostThreads, [&](unsigned, size_t c0, size_t c1) {
    for (size_t c = c0; c < c1; ++c) {
      uint32_t off = start[c];
      for (unsigned t = 0; t < used; ++t) {
        uint32_t n = at[t][c];
        at[t][c] = off;
        off += n;
      }
    }
  });
  run_threads(used, [&](unsigned t) {
    for (uint64_t pr : pairs[t]) list[at[t][pr >> 32]++] = (uint32_t)(pr & 0xffffffffu);
  });
}

// Calls f with the constants provider of the handle: the by-value constants
// of a single simulation, or the per-instance table of a batch (indexed by
// particle slot, or by boundary particle when `boundary`).
template <class F>
void dispatch(SphHandle* h, bool boundary, F&& f) {
  if (h->ninst == 1) f(sph::OneSim{h->k});
  else f(sph::ManySim{h->ktab, boundary ? h->inst_b : h->inst_p});
}

sph::Planes planes(SphHandle* h) { return sph::Planes{h->xyz, h->xyz_stride}; }

// Sizes per SM from which the warp-cooperative density scan (particles) and
// the cell-wise boundary pressure (boundary particles) run, measured on B200.
// Below them the per-particle forms are faster (2M-particle dam break and its
// coarser versions: the density scans break even near 250k particles, the
// boundary passes between 376k and 848k boundary particles). The environment
// variables SPH_WARP_SCAN_MIN and SPH_ADAMI_CELLS_MIN, read at creation,
// replace them with absolute counts (0: always the warp-cooperative form).
#ifndef SPH_WARP_SCAN_MIN_PER_SM
#define SPH_WARP_SCAN_MIN_PER_SM 2048
#endif
#ifndef SPH_ADAMI_CELLS_MIN_PER_SM
#define SPH_ADAMI_CELLS_MIN_PER_SM 4096
#endif

// Lets the density kernels take up to 128 KiB of dynamic shared memory (the
// warp scan's per-warp scratch passes the default 48 KiB at 512 threads) on
// the current device. Set at handle creation, before any graph capture.
void allow_density_smem() {
  using namespace sph;
  auto set = [](const void* f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024);
  };
  set(reinterpret_cast<const void*>(k_density<OneSim, 0>));
  set(reinterpret_cast<const void*>(k_density<OneSim, 1>));
  set(reinterpret_cast<const void*>(k_density<OneSim, 2>));
  set(reinterpret_cast<const void*>(k_density<ManySim, 0>));
  set(reinterpret_cast<const void*>(k_density<ManySim, 1>));
  set(reinterpret_cast<const void*>(k_density<ManySim, 2>));
}

// Sorting scratch + binning of posU into the cell tables (k_bin or the
// xsph kernel fill `hist` first).
void enqueue_scan_fill(SphHandle* h) {
  using namespace sph;
  int nbk = h->nbsum;
  k_scan_reduce<<<nbk, kScanThreads, 0, h->st>>>(h->hist, h->C, h->bsum);
  k_scan_bsum<<<1, kScanThreads, 0, h->st>>>(h->bsum, nbk);
  k_scan_apply<<<nbk, kScanThreads, 0, h->st>>>(h->hist, h->C, h->bsum, h->lin_of_rank, h->cstart,
                                                h->ccount, h->cursor, h->ctab);
  k_fill<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->keyU, h->idU, h->cursor, h->tmp, h->tmpid);
  h->launches += 4;
}

void enqueue_density_only(SphHandle* h) {
  using namespace sph;
  int bs = h->bs_density;
  sph::ClosureBufs cb{h->cl_count, h->cl_slot, h->cl_feat, h->cl_rho, h->corr, h->vel, h->cl_wb, h->cl_wf};
  if (h->cl_mode) cudaMemsetAsync(h->cl_count, 0, sizeof(uint32_t), h->st);
  // the warp scan's scratch per warp; closure mode 2 adds a 16-sample network
  // tile per warp (the fused inference)
  const int warp_scan = h->n >= h->warp_scan_min ? 1 : 0;
  const size_t smem = warp_scan ? (bs / 32) * sizeof(ScanWarp) : 0;
  const size_t smem_cl = smem + (bs / 32) * kClTileWords * sizeof(uint32_t);
  dispatch(h, false, [&](auto kp) {
    using KPT = decltype(kp);
    const int grid = grid_for(h->n, bs);
    if (h->cl_mode == 2)
      k_density<KPT, 2><<<grid, bs, smem_cl, h->st>>>(kp, h->n, h->dt, h->pos, planes(h), h->rv, h->id, h->ctab,
                                                     h->bc_start, h->bc_list, h->bpos, h->rf, h->pr, h->err,
                                                     h->nbr, h->ncount, h->sdf, h->wall_tab, cb,
                                                  warp_scan);
    else if (h->cl_mode)
      k_density<KPT, 1><<<grid, bs, smem, h->st>>>(kp, h->n, h->dt, h->pos, planes(h), h->rv, h->id, h->ctab,
                                                  h->bc_start, h->bc_list, h->bpos, h->rf, h->pr, h->err,
                                                  h->nbr, h->ncount, h->sdf, h->wall_tab, cb,
                                                  warp_scan);
    else
      k_density<KPT, 0><<<grid, bs, smem, h->st>>>(kp, h->n, h->dt, h->pos, planes(h), h->rv, h->id, h->ctab,
                                                  h->bc_start, h->bc_list, h->bpos, h->rf, h->pr, h->err,
                                                  h->nbr, h->ncount, h->sdf, h->wall_tab, cb,
                                                  warp_scan);
  });
  h->launches += 1;
}

// boundary.rs:87-123: the Adami boundary pressure, for the boundary particles
// that an occupied cell lists (the others get the empty sum's 0)
void enqueue_adami(SphHandle* h) {
  using namespace sph;
  if (h->nb > 0) {
    cudaMemsetAsync(h->bact, 0, (size_t)h->nb, h->st);
    if (h->nbc_cells > 0)
      k_adami_mark<<<grid_for(h->nbc_cells, 8), 256, 0, h->st>>>(h->nbc_cells, h->bc_cells, h->ctab, h->bc_start,
                                                                  h->bc_list, h->bact);
    dispatch(h, true, [&](auto kp) {
      if (h->adami_cells && (size_t)h->nb >= h->adami_cells_min)
        k_adami_cells<<<grid_for(h->nb, kAdamiWarps * 32), kAdamiWarps * 32, 0, h->st>>>(
            kp, h->nb, h->border, h->bpos, h->bpress, h->pos, planes(h), h->rf, h->pr, h->id, h->ctab, h->err,
            h->bact);
      else
        k_adami<<<grid_for(h->nb, kAdamiWarps), kAdamiWarps * 32, 0, h->st>>>(
            kp, h->nb, h->bpos, h->bpress, h->pos, h->rf, h->pr, h->id, h->ctab, h->err, h->bact);
    });
    h->launches += 2;
  }
}

void enqueue_density_adami(SphHandle* h) {
  enqueue_density_only(h);
  enqueue_adami(h);
}

void enqueue_forces(SphHandle* h, float hdt_scale) {
  using namespace sph;
  cudaMemsetAsync(h->red, 0, 2 * sizeof(float) * h->ninst, h->st);
  int bs = h->bs_forces;
  dispatch(h, false, [&](auto kp) {
    using KPT = decltype(kp);
    if (h->cl_mode)
      k_forces<KPT, 1><<<grid_for(h->n, bs), bs, 0, h->st>>>(kp, h->n, h->dt, hdt_scale, h->pos, h->vel, h->rf,
                                                           h->pr, h->id, h->ctab, h->bc_start, h->bc_list,
                                                           h->bpos, h->bpress, h->acc, h->velout, h->red,
                                                           h->err, h->nbr, h->ncount, h->sdf, h->wall_tab,
                                                           h->corr);
    else
      k_forces<KPT, 0><<<grid_for(h->n, bs), bs, 0, h->st>>>(kp, h->n, h->dt, hdt_scale, h->pos, h->vel, h->rf,
                                                           h->pr, h->id, h->ctab, h->bc_start, h->bc_list,
                                                           h->bpos, h->bpress, h->acc, h->velout, h->red,
                                                           h->err, h->nbr, h->ncount, h->sdf, h->wall_tab,
                                                           h->corr);
  });
  h->launches += 1;
}

void enqueue_xsph(SphHandle* h, bool use_list) {
  using namespace sph;
  int bs = h->bs_xsph;
  dispatch(h, false, [&](auto kp) {
    k_xsph_prep<<<grid_for(h->n, 256), 256, 0, h->st>>>(kp, h->n, h->dt, h->pos, h->velout, h->acc, h->xrec,
                                                         h->err);
    k_xsph_drift<<<grid_for(h->n, bs), bs, 0, h->st>>>(kp, h->n, h->dt, h->pos, h->velout, h->acc, h->xrec, h->id,
                                                       h->ctab, h->rank_of_lin, h->posU, h->velU, h->idU,
                                                       h->keyU, h->hist, h->err,
                                                       use_list ? h->nbr : nullptr, h->ncount);
  });
  h->launches += 2;
}

void enqueue_sort(SphHandle* h) {
  using namespace sph;
  enqueue_scan_fill(h);
  k_reorder<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->tmp, h->tmpid, h->keyU, h->cstart, h->ccount,
                                                    h->posU, h->velU, h->pos, h->vel, h->rv, h->id, h->err,
                                                    nullptr, nullptr, nullptr, nullptr, nullptr, planes(h));
  h->launches += 1;
}

// lib.rs:287-335 after the bootstrap: kick1+XSPH+drift+clamp, grid + reorder,
// density, boundary pressure, forces + kick2.
void enqueue_body(SphHandle* h, bool use_list) {
  enqueue_xsph(h, use_list);
  enqueue_sort(h);
  enqueue_density_adami(h);
  enqueue_forces(h, 1.0f);
}

// lib.rs:295-298: compute_forces(dt) once before the first step.
void enqueue_bootstrap(SphHandle* h) {
  enqueue_density_adami(h);
  enqueue_forces(h, 0.0f);
}

void enqueue_dt_finalize(SphHandle* h, float* out) {
  sph::k_dt_finalize<<<grid_for(h->ninst, 128), 128, 0, h->st>>>(h->ninst, h->hcc, h->red, out);
  h->launches += 1;
}

void enqueue_set_dt(SphHandle* h, float dt) {
  sph::k_set_dt<<<1, 256, 0, h->st>>>(h->dt, h->ninst, dt);
  h->launches += 1;
}

int capture(SphHandle* h, bool with_finalize, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  uint64_t before = h->launches;
  SPH_TRY(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  if (with_finalize) enqueue_dt_finalize(h, h->dt);
  enqueue_body(h, true);
  cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (e != cudaSuccess) return cuda_status(h, e, "cudaStreamEndCapture");
  h->body_kernels = (int)(h->launches - before);
  h->launches = before;
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  return cuda_status(h, e, "cudaGraphInstantiate");
}

void drop_graphs(SphHandle* h) {
  if (h->g_step) cudaGraphExecDestroy(h->g_step);
  if (h->g_auto) cudaGraphExecDestroy(h->g_auto);
  if (h->g_opt) cudaGraphExecDestroy(h->g_opt);
  h->g_step = nullptr;
  h->g_auto = nullptr;
  h->g_opt = nullptr;
}

int check_device_flags(SphHandle* h) {
  uint32_t e = 0;
  SPH_TRY(h, cudaMemcpyAsync(&e, h->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  if (e & sph::kErrCellCap)
    return set_err(h, SPH_ERR_CAPACITY, "a grid cell exceeded 4096 particles");
  if (e & sph::kErrAdamiCap)
    return set_err(h, SPH_ERR_CAPACITY, "a boundary particle has more than 256 fluid particles in support");
  return SPH_OK;
}

void ensure_red(SphHandle* h) {
  if (h->red_valid) return;
  cudaMemsetAsync(h->red, 0, 2 * sizeof(float) * h->ninst, h->st);
  if (h->n > 0) {
    dispatch(h, false, [&](auto kp) {
      sph::k_timestep_reduce<<<grid_for(h->n, 256), 256, 0, h->st>>>(kp, h->n, h->velout, h->acc, h->red);
    });
    h->launches += 1;
  }
  h->red_valid = true;
}

void free_all(SphHandle* h) {
  drop_graphs(h);
  if (h->pool == 1) {  // back to the pool, in stream order
    for (void* p : h->allocs) cudaFreeAsync(p, h->st);
    cudaStreamSynchronize(h->st);
  } else {
    for (void* p : h->allocs) cudaFree(p);
  }
  h->allocs.clear();
  if (h->st) cudaStreamDestroy(h->st);
}

int check_views(const SphParams& P, const SphParticlesView* pv, const SphBoundaryView* bv) {
  if (!pv) return SPH_ERR_INVALID_ARG;
  if (!(P.h > 0.0f) || !std::isfinite(P.h) || !(P.speed_of_sound > 0.0f)) return SPH_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a)
    if (!(P.domain_max[a] > P.domain_min[a])) return SPH_ERR_INVALID_ARG;
  if (pv->n > 0x7fffffffull) return SPH_ERR_INVALID_ARG;
  if (P.cell_order != SPH_CELL_ORDER_MORTON && P.cell_order != SPH_CELL_ORDER_LINEAR &&
      P.cell_order != SPH_CELL_ORDER_ROWS)
    return SPH_ERR_INVALID_ARG;
  if (pv->n > 0 && (!pv->x || !pv->y || !pv->z || !pv->vx || !pv->vy || !pv->vz || !pv->ax || !pv->ay ||
                    !pv->az || !pv->density || !pv->pressure || !pv->mass || !pv->temperature ||
                    !pv->fluid_type))
    return SPH_ERR_INVALID_ARG;
  if (bv && bv->n > 0 && (!bv->x || !bv->y || !bv->z || !bv->mass)) return SPH_ERR_INVALID_ARG;
  if (bv && bv->n > 0x7fffffffull) return SPH_ERR_INVALID_ARG;
  if (P.boundary_mode != SPH_BOUNDARY_PARTICLES && P.boundary_mode != SPH_BOUNDARY_SDF)
    return SPH_ERR_INVALID_ARG;
  return SPH_OK;
}

// One handle for `ninst` independent simulations on one device. Each
// instance keeps its own grid, constants, boundary lists and dt; instances
// occupy disjoint ranges of the global cell ranks, so the global counting
// sort keeps every instance in a fixed contiguous slot range.
// Phase times of a host-side call on stderr when the environment sets
// SPH_TRACE (the creation's host tables, packing, allocation, uploads).
struct PhaseTrace {
  const char* what;
  bool on = std::getenv("SPH_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), last = t0;
  explicit PhaseTrace(const char* w) : what(w) {}
  void mark(const char* phase) {
    if (!on) return;
    auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "%s: %-24s %8.2f ms (total %8.2f ms)\n", what, phase,
            std::chrono::duration<double, std::milli>(now - last).count(),
            std::chrono::duration<double, std::milli>(now - t0).count());
    last = now;
  }
};

int create_impl(int ninst, const SphParams* PP, const SphParticlesView* pvs,
                const SphBoundaryView* const* bvs, const SphSdfView* sdfs, SphHandle** out) {
  if (!out) return SPH_ERR_INVALID_ARG;
  *out = nullptr;
  if (ninst < 1 || ninst > 65535 || !PP || !pvs) return SPH_ERR_INVALID_ARG;
  const bool sdf_mode = PP[0].boundary_mode == SPH_BOUNDARY_SDF;
  uint64_t ntot = 0, nbtot = 0;
  for (int q = 0; q < ninst; ++q) {
    const SphBoundaryView* bv = bvs ? bvs[q] : nullptr;
    int s = check_views(PP[q], &pvs[q], bv);
    if (s != SPH_OK) return s;
    if (PP[q].device != PP[0].device) return SPH_ERR_INVALID_ARG;
    if ((PP[q].boundary_mode == SPH_BOUNDARY_SDF) != sdf_mode) return SPH_ERR_INVALID_ARG;
    ntot += pvs[q].n;
    if (!sdf_mode && bv) nbtot += bv->n;
  }
  if (ntot > 0x7fffffffull || nbtot > 0x7fffffffull) return SPH_ERR_INVALID_ARG;
  // SDF wall mode: the domain box faces are walls; an instance's obstacle SDF
  // (optional: distances may be NULL) is concatenated on the device; one wall
  // table, so every instance must share the smoothing length.
  uint64_t sdf_nodes = 0;
  std::vector<uint64_t> sdf_off(ninst + 1, 0);
  if (sdf_mode) {
    for (int q = 0; q < ninst; ++q) {
      if (PP[q].h != PP[0].h) return SPH_ERR_INVALID_ARG;
      for (int a = 0; a < 3; ++a)
        if (!(PP[q].domain_max[a] - PP[q].domain_min[a] >= 4.0f * PP[q].h)) return SPH_ERR_INVALID_ARG;
      const SphSdfView* sd = sdfs ? &sdfs[q] : nullptr;
      uint64_t nodes = 0;
      if (sd && sd->distances) {
        if (!(sd->cell_size > 0.0f)) return SPH_ERR_INVALID_ARG;
        if (sd->dims[0] < 2 || sd->dims[1] < 2 || sd->dims[2] < 2) return SPH_ERR_INVALID_ARG;
        nodes = (uint64_t)sd->dims[0] * sd->dims[1] * sd->dims[2];
      }
      sdf_off[q + 1] = sdf_off[q] + nodes;
    }
    sdf_nodes = sdf_off[ninst];
  }
  const SphParams& P0 = PP[0];
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || P0.device < 0 || P0.device >= ndev) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  int major = 0;  // one attribute, not the whole property table (tens of ms)
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, P0.device) != cudaSuccess ||
      major != 10) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }

  PhaseTrace trace("sph_create");
  SphHandle* h = new (std::nothrow) SphHandle();
  if (!h) return SPH_ERR_OOM;
  h->prm = P0;
  h->dev = P0.device;
  h->ninst = ninst;
  h->n = (int)ntot;
  h->nb = (int)nbtot;
  std::thread allocator;  // device arrays, allocated while the host builds tables and packs
  cudaError_t ae = cudaSuccess;
  auto fail = [&](int code) {
    if (allocator.joinable()) allocator.join();
    free_all(h);
    delete h;
    return code;
  };
  if (cudaSetDevice(h->dev) != cudaSuccess) return fail(SPH_ERR_NO_DEVICE);

  // per-instance grids (neighbor.rs:29-46), constants and cell ranks: Morton
  // order within an instance (21 bits per axis; the 30-bit key when all dims
  // <= 1024) or linear order, instances one after another.
  std::vector<uint32_t> lin_of_rank, rank_of_lin, bstart, blist;
  std::vector<float4> hcc(ninst);
  h->ktab_h.resize(ninst);
  h->poff.assign(ninst + 1, 0);
  h->boff.assign(ninst + 1, 0);
  h->init_e.assign(ninst, 0.0);
  h->init_m.assign(ninst, 0.0);
  // grid sizes first: they size the device arrays, which another thread
  // allocates while this one builds the cell ranks and boundary lists
  uint64_t Ctot = 0;
  for (int q = 0; q < ninst; ++q) {
    float cell = 2.0f * PP[q].h;
    uint64_t Cq = 1;
    for (int a = 0; a < 3; ++a) {
      uint32_t d = (uint32_t)fmaxf(ceilf((PP[q].domain_max[a] - PP[q].domain_min[a]) / cell), 1.0f);
      if (d > (1u << 21)) return fail(SPH_ERR_INVALID_ARG);
      Cq *= d;
    }
    if (Ctot + Cq > (1ull << 30)) return fail(SPH_ERR_INVALID_ARG);
    Ctot += Cq;
  }
  const size_t n = (size_t)h->n, nb = (size_t)h->nb;
  h->C = (int)Ctot;
  h->nbsum = grid_for(h->C, sph::kScanTile);
  h->nparts = std::max(1, std::min(grid_for((long long)n, sph::kMetricThreads), 1184));
  auto allocate_all = [&, Ctot] {
    const uint64_t C = Ctot;
    if (cudaSetDevice(h->dev) != cudaSuccess) {
      ae = cudaErrorInvalidDevice;
      return;
    }
    ae = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    allow_density_smem();
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->dev) != cudaSuccess) sms = 148;
    h->warp_scan_min = sms * SPH_WARP_SCAN_MIN_PER_SM;
    h->adami_cells_min = (size_t)sms * SPH_ADAMI_CELLS_MIN_PER_SM;
    if (const char* v = std::getenv("SPH_WARP_SCAN_MIN")) h->warp_scan_min = std::atoi(v);
    if (const char* v = std::getenv("SPH_ADAMI_CELLS_MIN")) h->adami_cells_min = (size_t)std::atoll(v);
#define ALLOC(ptr, cnt) \
  if (ae == cudaSuccess) ae = dalloc(h, &h->ptr, (cnt))
    ALLOC(pos, n); ALLOC(vel, n); ALLOC(velout, n); ALLOC(acc, n);
    ALLOC(rv, n); ALLOC(rf, n); ALLOC(pr, n); ALLOC(id, n);
    ALLOC(posU, n); ALLOC(velU, n); ALLOC(idU, n); ALLOC(keyU, n); ALLOC(tmp, n); ALLOC(tmpid, n);
    ALLOC(hist, C); ALLOC(cstart, C); ALLOC(ccount, C); ALLOC(cursor, C); ALLOC(bsum, h->nbsum);
    ALLOC(rank_of_lin, C); ALLOC(lin_of_rank, C); ALLOC(ctab, C);
    ALLOC(bpos, nb); ALLOC(bpress, nb); ALLOC(bact, nb); ALLOC(bc_start, C + 1);
    ALLOC(dt, ninst); ALLOC(dt_query, ninst); ALLOC(red, 2 * ninst); ALLOC(err, 1); ALLOC(hcc, ninst);
    ALLOC(part_m, h->nparts); ALLOC(part_e, h->nparts); ALLOC(part_var, h->nparts); ALLOC(me, 2);
    ALLOC(var, 1); ALLOC(bad, 1);
    ALLOC(stage, 12 * n); ALLOC(stage_ft, n); ALLOC(diag, 2);
    ALLOC(nbr, (size_t)sph::kNbrCap * n); ALLOC(ncount, n); ALLOC(xrec, 2 * n);
    h->xyz_stride = ((size_t)n + 3) / 4 * 4 + 4;  // aligned groups of 4 may read past the last slot
    ALLOC(xyz, 3 * h->xyz_stride);
    if (ninst > 1) {
      ALLOC(ktab, ninst); ALLOC(inst_p, n); ALLOC(inst_b, nb);
    }
    if (sdf_mode) ALLOC(sdf, std::max<uint64_t>(sdf_nodes, 1));
#undef ALLOC
  };
  try {
    allocator = std::thread(allocate_all);
  } catch (...) {  // no thread to be had: allocate here, before the host tables
    allocate_all();
  }
  for (int q = 0; q < ninst; ++q) {
    const SphBoundaryView* bv = (sdf_mode || !bvs) ? nullptr : bvs[q];
    h->poff[q + 1] = h->poff[q] + pvs[q].n;
    h->boff[q + 1] = h->boff[q] + (bv ? bv->n : 0);
  }
  // upload staging (particles of instance q at [poff[q], poff[q+1]), ids
  // global), left uninitialised: every entry is written below, by host
  // threads that also take the first-touch page faults, while the device
  // arrays are being allocated
  std::unique_ptr<float4[]> hpos(new float4[n]), hvel(new float4[n]), hacc(new float4[n]), hb(new float4[nb]);
  std::unique_ptr<uint32_t[]> hid(new uint32_t[n]);
  std::unique_ptr<float[]> hpr(new float[n]);
  std::vector<uint16_t> hip(ninst > 1 ? n : 0), hib(ninst > 1 ? nb : 0);
  h->temperature.resize(n);
  for (int q = 0; q < ninst; ++q) {
    const SphParticlesView* pv = &pvs[q];
    size_t o = h->poff[q];
    parallel_chunks(pv->n, kHostThreads, [&](unsigned, size_t i0, size_t i1) {
      for (size_t i = i0; i < i1; ++i) {
        hpos[o + i] = make_float4(pv->x[i], pv->y[i], pv->z[i], pv->mass[i]);
        hvel[o + i] = make_float4(pv->vx[i], pv->vy[i], pv->vz[i], pv->density[i]);
        hacc[o + i] = make_float4(pv->ax[i], pv->ay[i], pv->az[i], 0.0f);
        hid[o + i] = (uint32_t)(o + i) | (pv->fluid_type[i] ? sph::kAirBit : 0u);
        hpr[o + i] = pv->pressure[i];
        h->temperature[o + i] = pv->temperature[i];
        if (ninst > 1) hip[o + i] = (uint16_t)q;
      }
    });
    const SphBoundaryView* bv = (sdf_mode || !bvs) ? nullptr : bvs[q];
    size_t bo = h->boff[q];
    for (size_t i = 0; bv && i < bv->n; ++i) {
      hb[bo + i] = make_float4(bv->x[i], bv->y[i], bv->z[i], bv->mass[i]);
      if (ninst > 1) hib[bo + i] = (uint16_t)q;
    }
  }
  trace.mark("staging packed");
  allocator.join();
  trace.mark("allocation joined");
  cudaError_t e = ae;
  if (e != cudaSuccess) return fail(e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA);
  float4* accU = nullptr;
  float* prU = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&accU, std::max<size_t>(1, n) * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&prU, std::max<size_t>(1, n) * sizeof(float));
  if (e != cudaSuccess) {
    if (accU) cudaFree(accU);
    return fail(SPH_ERR_OOM);
  }
  // the particle uploads (pageable copies hold the issuing thread) run on a
  // thread of their own while this one builds the cell tables
  cudaError_t ue = cudaSuccess;
  auto upload_particles = [&] {
    auto upq = [&](void* d, const void* src, size_t bytes) {
      if (ue == cudaSuccess && bytes) ue = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, h->st);
    };
    if (cudaSetDevice(h->dev) != cudaSuccess) {
      ue = cudaErrorInvalidDevice;
      return;
    }
    upq(h->posU, hpos.get(), n * sizeof(float4));
    upq(h->velU, hvel.get(), n * sizeof(float4));
    upq(accU, hacc.get(), n * sizeof(float4));
    upq(prU, hpr.get(), n * sizeof(float));
    upq(h->idU, hid.get(), n * sizeof(uint32_t));
    upq(h->bpos, hb.get(), nb * sizeof(float4));
    if (ninst > 1) {
      upq(h->inst_p, hip.data(), n * sizeof(uint16_t));
      upq(h->inst_b, hib.data(), nb * sizeof(uint16_t));
    }
  };
  std::thread uploader;
  try {
    uploader = std::thread(upload_particles);
  } catch (...) {  // no thread to be had: upload here, before the tables
    upload_particles();
  }
  // initial conservation totals, in the reference's order (lib.rs:152-156),
  // on a thread of their own while this one builds the tables
  auto initial_totals = [&] {
    for (int q = 0; q < ninst; ++q) {
      const SphParticlesView* pv = &pvs[q];
      const SphParams& P = PP[q];
      double m = 0.0, e = 0.0;
      for (size_t i = 0; i < pv->n; ++i) {  // two sums, each in index order
        double mi = (double)pv->mass[i];
        m += mi;
        double vx = pv->vx[i], vy = pv->vy[i], vz = pv->vz[i];
        e += 0.5 * mi * (vx * vx + vy * vy + vz * vz);
        double x = pv->x[i], y = pv->y[i], z = pv->z[i];
        e -= mi * ((double)P.gravity[0] * x + (double)P.gravity[1] * y + (double)P.gravity[2] * z);
      }
      h->init_m[q] = m;
      h->init_e[q] = e;
    }
  };
  // The boundary particles ordered by the global cell that holds them
  // (counting sort, ascending index within a cell), for k_adami_cells; the
  // cells are those of the grid built below (same f32 operations), on a
  // thread of its own while this one builds the tables.
  std::vector<uint32_t> border_h;
  h->adami_cells = nb > 0;
  for (int q = 0; q < ninst; ++q)
    h->adami_cells = h->adami_cells &&
                     (PP[q].cell_order == SPH_CELL_ORDER_LINEAR || PP[q].cell_order == SPH_CELL_ORDER_ROWS);
  auto boundary_order = [&] {
    uint64_t Ctot = 0;
    std::vector<uint64_t> coffs(ninst);
    std::vector<std::array<uint32_t, 3>> dimq(ninst);
    for (int q = 0; q < ninst; ++q) {
      const float cell = 2.0f * PP[q].h;
      uint64_t Cq = 1;
      for (int a = 0; a < 3; ++a) {
        dimq[q][a] = (uint32_t)fmaxf(ceilf((PP[q].domain_max[a] - PP[q].domain_min[a]) / cell), 1.0f);
        Cq *= dimq[q][a];
      }
      coffs[q] = Ctot;
      Ctot += Cq;
    }
    std::vector<uint32_t> bkey(nb), bnext(Ctot + 1, 0);
    for (int q = 0; q < ninst; ++q) {
      const float cell = 2.0f * PP[q].h;
      auto cell_of = [&](float p, int a) {  // axis_cell, in the same f32 operations
        float f = std::floor((p - PP[q].domain_min[a]) / cell);
        f = std::fmax(f, 0.0f);
        f = std::fmin(f, (float)(dimq[q][a] - 1));
        return (uint32_t)f;
      };
      for (size_t i = h->boff[q]; i < h->boff[q + 1]; ++i) {
        const float4 v = hb[i];
        bkey[i] = (uint32_t)coffs[q] + cell_of(v.x, 0) + dimq[q][0] * (cell_of(v.y, 1) + dimq[q][1] * cell_of(v.z, 2));
        ++bnext[bkey[i] + 1];
      }
    }
    for (uint64_t c = 0; c < Ctot; ++c) bnext[c + 1] += bnext[c];
    border_h.resize(nb);
    for (size_t i = 0; i < nb; ++i) border_h[bnext[bkey[i]]++] = (uint32_t)i;
  };
  std::thread border_thread;
  if (h->adami_cells) {
    try {
      border_thread = std::thread(boundary_order);
    } catch (...) {  // no thread to be had: order them here
      boundary_order();
    }
  }
  std::thread totals;
  try {
    totals = std::thread(initial_totals);
  } catch (...) {  // no thread to be had: compute them here
    initial_totals();
  }
  uint64_t C = 0;
  bstart.push_back(0);
  for (int q = 0; q < ninst; ++q) {
    const SphParams& P = PP[q];
    const SphParticlesView* pv = &pvs[q];
    const SphBoundaryView* bv = (sdf_mode || !bvs) ? nullptr : bvs[q];
    uint32_t dims[3];
    float cell = 2.0f * P.h;
    uint64_t Cq = 1;
    for (int a = 0; a < 3; ++a) {  // as above (checked there)
      dims[a] = (uint32_t)fmaxf(ceilf((P.domain_max[a] - P.domain_min[a]) / cell), 1.0f);
      Cq *= dims[a];
    }
    SimConst k = make_const(P, dims);
    k.rows = P.cell_order == SPH_CELL_ORDER_LINEAR || P.cell_order == SPH_CELL_ORDER_ROWS;
    k.inst = q;
    k.coff = (int)C;
    k.cfl = P.cfl_number;
    if (sdf_mode) {
      const SphSdfView* sd = sdfs ? &sdfs[q] : nullptr;
      k.sdf_mode = 1;
      k.has_geo = (sd && sd->distances) ? 1 : 0;
      if (k.has_geo) {
        for (int a = 0; a < 3; ++a) {
          k.sdf_origin[a] = sd->origin[a];
          k.sdf_dims[a] = (int)sd->dims[a];
        }
        k.sdf_cell = sd->cell_size;
      }
      k.sdf_off = (long long)sdf_off[q];
      k.wall_scale = wall_mass_scale(P.h, pv);
      k.feat_sdf = 1;
    }
    h->ktab_h[q] = k;
    hcc[q] = make_float4(P.h, P.speed_of_sound, P.cfl_number, 0.0f);
    lin_of_rank.resize(C + Cq);
    rank_of_lin.resize(C + Cq);
    auto set_rank = [&](uint64_t r, uint32_t lin) {
      lin_of_rank[C + r] = (uint32_t)(C + lin);
      rank_of_lin[C + lin] = (uint32_t)(C + r);
    };
    if (P.cell_order == SPH_CELL_ORDER_MORTON) {
      std::vector<std::pair<uint64_t, uint32_t>> cells(Cq);
      for (uint32_t cz = 0; cz < dims[2]; ++cz)
        for (uint32_t cy = 0; cy < dims[1]; ++cy)
          for (uint32_t cx = 0; cx < dims[0]; ++cx) {
            uint32_t lin = cx + cy * dims[0] + cz * dims[0] * dims[1];
            cells[lin] = {spread21(cx) | (spread21(cy) << 1) | (spread21(cz) << 2), lin};
          }
      std::sort(cells.begin(), cells.end());
      for (uint64_t r = 0; r < Cq; ++r) set_rank(r, cells[r].second);
    } else {
      // linear: rank = linear index; rows: the x-rows ranked by the Morton
      // code of (cy, cz), x fastest inside a row (only the rows are sorted)
      std::vector<std::pair<uint64_t, uint32_t>> rows((size_t)dims[1] * dims[2]);
      for (uint32_t cz = 0; cz < dims[2]; ++cz)
        for (uint32_t cy = 0; cy < dims[1]; ++cy) {
          uint32_t row = cy + cz * dims[1];
          rows[row] = {P.cell_order == SPH_CELL_ORDER_ROWS ? (spread2(cy) | (spread2(cz) << 1)) : row, row};
        }
      std::sort(rows.begin(), rows.end());
      for (size_t rr = 0; rr < rows.size(); ++rr)
        for (uint32_t cx = 0; cx < dims[0]; ++cx)
          set_rank((uint64_t)rr * dims[0] + cx, rows[rr].second * dims[0] + cx);
    }
    std::vector<uint32_t> s1, l1;
    build_boundary_lists(k, bv, (int)Cq, s1, l1);
    uint32_t base = (uint32_t)blist.size(), bbase = (uint32_t)h->boff[q];
    if (base == 0 && bbase == 0 && bstart.size() == 1) {  // the first instance: take the lists as they are
      bstart = std::move(s1);
      blist = std::move(l1);
    } else {
      bstart.reserve(bstart.size() + Cq);
      for (uint64_t c = 1; c <= Cq; ++c) bstart.push_back(base + s1[c]);
      blist.reserve(blist.size() + l1.size());
      for (uint32_t b : l1) blist.push_back(bbase + b);
    }
    C += Cq;
  }
  if (totals.joinable()) totals.join();
  trace.mark("cell ranks, lists, totals");
  if (border_thread.joinable()) border_thread.join();
  trace.mark("boundary order");
  h->k = h->ktab_h[0];
  h->C = (int)C;
  h->boundary_candidates = blist.size();
  std::vector<uint32_t> bcells;  // cells with boundary candidates (static: they bound k_adami_mark)
  for (uint64_t c = 0; c < C; ++c)
    if (bstart[c + 1] > bstart[c]) bcells.push_back((uint32_t)c);
  for (int q = 0; q < ninst; ++q) {
    h->init_mass += h->init_m[q];
    h->init_energy += h->init_e[q];
  }
  std::vector<float2> wall_host;
  if (sdf_mode) {
    float inv = 0.0f;
    float inv2 = 0.0f, inv3 = 0.0f;
    wall_host = make_wall_tables(P0.h, &inv, &inv2, &inv3);
    for (int q = 0; q < ninst; ++q) {
      h->ktab_h[q].wall_inv_step = inv;
      h->ktab_h[q].wall_inv2 = inv2;
      h->ktab_h[q].wall_inv3 = inv3;
    }
  }
  h->k = h->ktab_h[0];

  if (uploader.joinable()) uploader.join();
  trace.mark("particle uploads joined");
  if (e == cudaSuccess) e = ue;
  if (e == cudaSuccess) e = dalloc(h, &h->bc_list, blist.size());
  if (e == cudaSuccess) e = dalloc(h, &h->bc_cells, bcells.size());
  if (e == cudaSuccess && h->adami_cells) e = dalloc(h, &h->border, nb);
  h->nbc_cells = (int)bcells.size();
  if (e == cudaSuccess && sdf_mode) e = dalloc(h, &h->wall_tab, wall_host.size());
  if (e != cudaSuccess) {
    cudaFree(accU);
    cudaFree(prU);
    return fail(e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA);
  }
  auto up = [&](void* d, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, h->st);
  };
  up(h->rank_of_lin, rank_of_lin.data(), C * sizeof(uint32_t));
  up(h->lin_of_rank, lin_of_rank.data(), C * sizeof(uint32_t));
  up(h->bc_start, bstart.data(), (C + 1) * sizeof(uint32_t));
  up(h->bc_list, blist.data(), blist.size() * sizeof(uint32_t));
  up(h->bc_cells, bcells.data(), bcells.size() * sizeof(uint32_t));
  if (h->adami_cells) up(h->border, border_h.data(), nb * sizeof(uint32_t));
  up(h->hcc, hcc.data(), ninst * sizeof(float4));
  if (ninst > 1) up(h->ktab, h->ktab_h.data(), ninst * sizeof(SimConst));
  for (int q = 0; sdf_mode && q < ninst; ++q)
    if (sdf_off[q + 1] > sdf_off[q])
      up(h->sdf + sdf_off[q], sdfs[q].distances, (sdf_off[q + 1] - sdf_off[q]) * sizeof(float));
  if (sdf_mode) up(h->wall_tab, wall_host.data(), wall_host.size() * sizeof(float2));
  trace.mark("uploads issued");
  if (e == cudaSuccess) e = cudaMemsetAsync(h->hist, 0, C * sizeof(uint32_t), h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->bpress, 0, std::max<size_t>(1, nb) * sizeof(float), h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->err, 0, sizeof(uint32_t), h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->ctab, 0, C * sizeof(uint2), h->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->xyz, 0, 3 * h->xyz_stride * sizeof(float), h->st);
  if (e == cudaSuccess && n > 0) {
    using namespace sph;
    dispatch(h, false, [&](auto kp) {
      k_bin<<<grid_for(h->n, 256), 256, 0, h->st>>>(kp, h->n, h->posU, h->rank_of_lin, h->keyU, h->hist);
    });
    h->launches += 1;
    enqueue_scan_fill(h);
    k_reorder<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->tmp, h->tmpid, h->keyU, h->cstart,
                                                      h->ccount, h->posU, h->velU, h->pos, h->vel, h->rv,
                                                      h->id, h->err, accU, h->acc, prU, h->pr, h->velout,
                                                      planes(h));
    h->launches += 1;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  trace.mark("sort and sync");
  if (accU) cudaFree(accU);
  if (prU) cudaFree(prU);
  if (e != cudaSuccess) {
    fprintf(stderr, "sph_create: %s\n", cudaGetErrorString(e));
    return fail(e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA);
  }
  ensure_red(h);
  int st = check_device_flags(h);
  if (st != SPH_OK) return fail(st);
  trace.mark("done");
  *out = h;
  return SPH_OK;
}

}  // namespace

extern "C" {

void sph_params_default(SphParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->alpha = 1.0f;
  p->beta = 2.0f;
  p->boundary_mode = SPH_BOUNDARY_PARTICLES;
  p->cell_order = SPH_CELL_ORDER_ROWS;
  p->flags = SPH_FLAGS_REFERENCE;
  p->device = 0;
  p->cfl_number = 0.25f;
  p->sdf_wall_coef = 0.981f;
}

int sph_create(const SphParams* params, const SphParticlesView* pv, const SphBoundaryView* bv,
               const SphSdfView* sdf, SphHandle** out) {
  if (!out) return SPH_ERR_INVALID_ARG;
  *out = nullptr;
  if (!params || !pv) return SPH_ERR_INVALID_ARG;
  const SphBoundaryView* bvs[1] = {bv};
  return create_impl(1, params, pv, bvs, sdf, out);
}

int sph_batch_create(int ninst, const SphParams* params, const SphParticlesView* particles,
                     const SphBoundaryView* boundaries, SphHandle** out) {
  if (!out) return SPH_ERR_INVALID_ARG;
  *out = nullptr;
  if (ninst < 1 || !params || !particles) return SPH_ERR_INVALID_ARG;
  std::vector<const SphBoundaryView*> bvs(ninst, nullptr);
  for (int q = 0; q < ninst && boundaries; ++q) bvs[q] = boundaries[q].n ? &boundaries[q] : nullptr;
  for (int q = 0; q < ninst; ++q)
    if (params[q].boundary_mode != SPH_BOUNDARY_PARTICLES) return SPH_ERR_INVALID_ARG;
  return create_impl(ninst, params, particles, bvs.data(), nullptr, out);
}

int sph_batch_create_sdf(int ninst, const SphParams* params, const SphParticlesView* particles,
                         const SphSdfView* sdfs, SphHandle** out) {
  if (!out) return SPH_ERR_INVALID_ARG;
  *out = nullptr;
  if (ninst < 1 || !params || !particles) return SPH_ERR_INVALID_ARG;
  for (int q = 0; q < ninst; ++q)
    if (params[q].boundary_mode != SPH_BOUNDARY_SDF) return SPH_ERR_INVALID_ARG;
  return create_impl(ninst, params, particles, nullptr, sdfs, out);
}

void sph_destroy(SphHandle* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  if (h->st) cudaStreamSynchronize(h->st);
  free_all(h);
  delete h;
}

namespace {
// sph_step after the step's dt is in device memory
int step_enqueued_dt(SphHandle* h) {
  if (h->needs_init) {
    enqueue_bootstrap(h);
    h->needs_init = false;
    h->list_valid = true;
  }
  if (!h->list_valid) {
    // after a restore: XSPH rescans the stale grid with the restored positions
    enqueue_body(h, false);
  } else {
    if (!h->g_step) {
      int s = capture(h, false, &h->g_step);
      if (s != SPH_OK) return s;
    }
    SPH_TRY(h, cudaGraphLaunch(h->g_step, h->st));
    h->launches += h->body_kernels;
  }
  h->list_valid = true;
  h->red_valid = true;
  return cuda_status(h, cudaGetLastError(), "sph_step");
}
}  // namespace

int sph_step(SphHandle* h, float dt) {
  if (!h) return SPH_ERR_INVALID_ARG;
  if (!std::isfinite(dt)) return set_err(h, SPH_ERR_INVALID_ARG, "dt must be finite");
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n == 0) return SPH_OK;
  enqueue_set_dt(h, dt);
  return step_enqueued_dt(h);
}

int sph_batch_step(SphHandle* h, const float* dts) {
  if (!h || !dts) return SPH_ERR_INVALID_ARG;
  for (int q = 0; q < h->ninst; ++q)
    if (!std::isfinite(dts[q])) return set_err(h, SPH_ERR_INVALID_ARG, "dt must be finite");
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n == 0) return SPH_OK;
  SPH_TRY(h, cudaMemcpyAsync(h->dt, dts, sizeof(float) * h->ninst, cudaMemcpyHostToDevice, h->st));
  return step_enqueued_dt(h);
}

int sph_step_auto(SphHandle* h, int nsteps, float* dt_out) {
  if (!h || nsteps < 0) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n == 0) return SPH_OK;
  for (int s = 0; s < nsteps; ++s) {
    ensure_red(h);
    if (h->needs_init || !h->list_valid) {
      enqueue_dt_finalize(h, h->dt);
      if (h->needs_init) {
        enqueue_bootstrap(h);
        h->needs_init = false;
        h->list_valid = true;
      }
      enqueue_body(h, h->list_valid);
    } else {
      if (!h->g_auto) {
        int st = capture(h, true, &h->g_auto);
        if (st != SPH_OK) return st;
      }
      SPH_TRY(h, cudaGraphLaunch(h->g_auto, h->st));
      h->launches += h->body_kernels;
    }
    h->list_valid = true;
    h->red_valid = true;
  }
  if (dt_out) {
    SPH_TRY(h, cudaMemcpyAsync(dt_out, h->dt, sizeof(float), cudaMemcpyDeviceToHost, h->st));
    SPH_TRY(h, cudaStreamSynchronize(h->st));
    return check_device_flags(h);
  }
  return cuda_status(h, cudaGetLastError(), "sph_step_auto");
}

int sph_compute_timestep(SphHandle* h, float* dt_out) {
  if (!h || !dt_out) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n == 0) {
    float dt = h->prm.cfl_number * h->prm.h / h->prm.speed_of_sound;
    *dt_out = fminf(fmaxf(fminf(dt, 0.01f), 1.0e-8f), 0.01f);
    return SPH_OK;
  }
  ensure_red(h);
  enqueue_dt_finalize(h, h->dt_query);
  SPH_TRY(h, cudaMemcpyAsync(dt_out, h->dt_query, sizeof(float), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

int sph_step_profiled(SphHandle* h, float dt, SphStepProfile* prof) {
  if (!h || !prof) return SPH_ERR_INVALID_ARG;
  if (!std::isfinite(dt)) return set_err(h, SPH_ERR_INVALID_ARG, "dt must be finite");
  SPH_TRY(h, cudaSetDevice(h->dev));
  std::memset(prof, 0, sizeof(*prof));
  if (h->n == 0) return SPH_OK;
  enqueue_set_dt(h, dt);
  if (h->needs_init) {
    enqueue_bootstrap(h);
    h->needs_init = false;
    h->list_valid = true;
  }
  cudaEvent_t ev[6];
  for (int i = 0; i < 6; ++i) SPH_TRY(h, cudaEventCreate(&ev[i]));
  cudaEventRecord(ev[0], h->st);
  enqueue_xsph(h, h->list_valid);
  cudaEventRecord(ev[1], h->st);
  enqueue_sort(h);
  cudaEventRecord(ev[2], h->st);
  enqueue_density_only(h);
  cudaEventRecord(ev[3], h->st);
  enqueue_adami(h);
  cudaEventRecord(ev[4], h->st);
  enqueue_forces(h, 1.0f);
  cudaEventRecord(ev[5], h->st);
  cudaError_t e = cudaEventSynchronize(ev[5]);
  float t[5];
  for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
  for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
  if (e != cudaSuccess) return cuda_status(h, e, "sph_step_profiled");
  prof->xsph_drift_us = t[0] * 1e3f;
  prof->sort_us = t[1] * 1e3f;
  prof->density_us = t[2] * 1e3f;
  prof->boundary_pressure_us = t[3] * 1e3f;
  prof->forces_us = t[4] * 1e3f;
  prof->total_us = (t[0] + t[1] + t[2] + t[3] + t[4]) * 1e3f;
  h->red_valid = true;
  h->list_valid = true;
  return check_device_flags(h);
}

int sph_read_particles(SphHandle* h, SphParticlesMut* o) {
  if (!h || !o) return SPH_ERR_INVALID_ARG;
  if (o->n != (size_t)h->n) return set_err(h, SPH_ERR_INVALID_ARG, "particle count mismatch");
  SPH_TRY(h, cudaSetDevice(h->dev));
  size_t n = (size_t)h->n;
  if (n == 0) return SPH_OK;
  float* dst[12] = {o->x, o->y, o->z, o->vx, o->vy, o->vz, o->ax, o->ay, o->az, o->density, o->pressure, o->mass};
  for (int f = 0; f < 12; ++f)
    if (!dst[f]) return set_err(h, SPH_ERR_INVALID_ARG, "null output array");
  sph::k_unsort<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->pos, h->velout, h->acc, h->pr, h->id,
                                                       h->stage, h->stage_ft);
  h->launches += 1;
  for (int f = 0; f < 12; ++f)
    SPH_TRY(h, cudaMemcpyAsync(dst[f], h->stage + f * n, n * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  if (o->fluid_type)
    SPH_TRY(h, cudaMemcpyAsync(o->fluid_type, h->stage_ft, n, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  if (o->temperature) std::memcpy(o->temperature, h->temperature.data(), n * sizeof(float));
  return check_device_flags(h);
}

int sph_read_boundary_pressure(SphHandle* h, float* out, size_t nb) {
  if (!h || (nb && !out) || nb != (size_t)h->nb) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (nb) SPH_TRY(h, cudaMemcpyAsync(out, h->bpress, nb * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

namespace {
// FP64 mass / energy sums and the maximum density variation into h->me, h->var
void enqueue_metrics(SphHandle* h) {
  sph::k_metrics_partial<<<h->nparts, sph::kMetricThreads, 0, h->st>>>(h->k, h->n, h->pos, h->velout, h->id,
                                                                     h->part_m, h->part_e, h->part_var);
  sph::k_metrics_final<<<1, 32, 0, h->st>>>(h->nparts, h->part_m, h->part_e, h->part_var, h->me, h->var);
  h->launches += 2;
}

cudaError_t ensure_ck(SphHandle* h) {
  if (h->ck_pos) return cudaSuccess;
  size_t n = (size_t)h->n;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = dalloc(h, &h->ck_pos, n);
  if (e == cudaSuccess) e = dalloc(h, &h->ck_velout, n);
  if (e == cudaSuccess) e = dalloc(h, &h->ck_acc, n);
  if (e == cudaSuccess) e = dalloc(h, &h->ck_pr, n);
  if (e == cudaSuccess) e = dalloc(h, &h->ck_slot, n);
  return e;
}

void enqueue_save_ck(SphHandle* h) {
  size_t n = (size_t)h->n;
  cudaMemcpyAsync(h->ck_pos, h->pos, n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(h->ck_velout, h->velout, n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(h->ck_acc, h->acc, n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(h->ck_pr, h->pr, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st);
  sph::k_index_ids<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->id, h->ck_slot);
  h->launches += 1;
}

void enqueue_restore_ck(SphHandle* h) {
  sph::k_restore<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->id, h->ck_slot, h->ck_pos, h->ck_velout,
                                                        h->ck_acc, h->ck_pr, h->pos, h->velout, h->acc, h->pr,
                                                        planes(h));
  h->launches += 1;
}
}  // namespace

int sph_error_metrics(SphHandle* h, SphErrorMetrics* out) {
  if (!h || !out) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  double me[2] = {0.0, 0.0};
  float var = 0.0f;
  if (h->n > 0) {
    enqueue_metrics(h);
    SPH_TRY(h, cudaMemcpyAsync(me, h->me, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    SPH_TRY(h, cudaMemcpyAsync(&var, h->var, sizeof(float), cudaMemcpyDeviceToHost, h->st));
    SPH_TRY(h, cudaStreamSynchronize(h->st));
  }
  double E0 = h->init_energy, M0 = h->init_mass;
  out->max_density_variation = var;
  out->energy_conservation = std::fabs(E0) > 1.0e-12 ? (float)std::fabs((me[1] - E0) / E0) : (float)std::fabs(me[1] - E0);
  out->mass_conservation = std::fabs(M0) > 1.0e-12 ? (float)std::fabs((me[0] - M0) / M0) : (float)std::fabs(me[0] - M0);
  return check_device_flags(h);
}

size_t sph_particle_count(const SphHandle* h) { return h ? (size_t)h->n : 0; }

int sph_save_checkpoint(SphHandle* h) {
  if (!h) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  {
    cudaError_t e = ensure_ck(h);
    if (e != cudaSuccess) return cuda_status(h, e, "checkpoint allocation");
  }
  if (h->n) enqueue_save_ck(h);
  h->has_ck = true;
  return cuda_status(h, cudaGetLastError(), "sph_save_checkpoint");
}

int sph_restore_checkpoint(SphHandle* h) {
  if (!h) return SPH_ERR_INVALID_ARG;
  if (!h->has_ck) return set_err(h, SPH_ERR_NO_CHECKPOINT, "no checkpoint saved");
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n) enqueue_restore_ck(h);
  h->has_ck = false;
  h->red_valid = false;
  h->list_valid = false;
  ensure_red(h);
  return cuda_status(h, cudaGetLastError(), "sph_restore_checkpoint");
}

namespace {
// The optimistic step as one graph: the main part runs every time, the
// retry branch (restore + the step with dt_safe) only when k_opt_decide
// sets the conditional handle.
int capture_opt(SphHandle* h, float alpha, float limit, uint32_t cool) {
  using namespace sph;
  cudaGraph_t g = nullptr;
  SPH_TRY(h, cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle retry;
  cudaError_t e = cudaGraphConditionalHandleCreate(&retry, g, 0, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(h, e, "cudaGraphConditionalHandleCreate");
  }
  uint64_t before = h->launches;
  e = cudaStreamBeginCaptureToGraph(h->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(h, e, "cudaStreamBeginCaptureToGraph");
  }
  enqueue_dt_finalize(h, h->dt_safe_dev);
  k_opt_begin<<<1, 1, 0, h->st>>>(h->run, h->dt_safe_dev, h->dt, alpha);
  h->launches += 1;
  enqueue_save_ck(h);
  enqueue_body(h, true);
  enqueue_metrics(h);
  k_opt_decide<<<1, 1, 0, h->st>>>(h->run, h->var, limit, cool, retry);
  h->launches += 1;
  e = cudaStreamEndCapture(h->st, &g);
  h->opt_kernels = (int)(h->launches - before);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    h->launches = before;
    return cuda_status(h, e, "cudaStreamEndCapture");
  }
  // the retry branch depends on every leaf of the main part
  size_t nn = 0;
  cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn), leaves;
  cudaGraphGetNodes(g, nodes.data(), &nn);
  for (cudaGraphNode_t nd : nodes) {
    size_t nd_out = 0;
    cudaGraphNodeGetDependentNodes(nd, nullptr, &nd_out);
    if (nd_out == 0) leaves.push_back(nd);
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = retry;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t cn;
  e = cudaGraphAddNode(&cn, g, leaves.data(), leaves.size(), &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    h->launches = before;
    return cuda_status(h, e, "conditional node");
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  uint64_t mid = h->launches;
  e = cudaStreamBeginCaptureToGraph(h->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_restore_ck(h);
    k_opt_retry<<<1, 1, 0, h->st>>>(h->run, h->dt);
    h->launches += 1;
    enqueue_body(h, false);
    k_opt_commit<<<1, 1, 0, h->st>>>(h->run);
    h->launches += 1;
    e = cudaStreamEndCapture(h->st, &body);
  }
  h->retry_kernels = (int)(h->launches - mid);
  h->launches = before;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->g_opt, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) h->g_opt = nullptr;
  return cuda_status(h, e, "optimistic step graph");
}

// The same step through the public entry points (runner.rs:189-240 as
// written): the first step of a handle (whose force bootstrap the reference
// ties to its first step() call) and a step after a caller's restore.
int opt_step_host(SphHandle* h, float alpha, float limit, uint32_t cool) {
  sph::RunState r;
  SPH_TRY(h, cudaMemcpyAsync(&r, h->run, sizeof(r), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  float dt_safe = 0.0f, used = 0.0f;
  int st = sph_compute_timestep(h, &dt_safe);
  if (st != SPH_OK) return st;
  if (r.cooldown > 0u) {
    r.cooldown -= 1u;
    if ((st = sph_step(h, dt_safe)) != SPH_OK) return st;
    used = dt_safe;
  } else {
    if ((st = sph_save_checkpoint(h)) != SPH_OK) return st;
    float dt_try = dt_safe * alpha;
    if ((st = sph_step(h, dt_try)) != SPH_OK) return st;
    SphErrorMetrics m;
    if ((st = sph_error_metrics(h, &m)) != SPH_OK) return st;
    if (m.max_density_variation > limit) {
      if ((st = sph_restore_checkpoint(h)) != SPH_OK) return st;
      if ((st = sph_step(h, dt_safe)) != SPH_OK) return st;
      used = dt_safe;
      r.rejected += 1ull;
      r.cooldown = cool;
    } else {
      used = dt_try;
      r.accepted += 1ull;
    }
  }
  r.sim_time += (double)used;
  r.steps += 1ull;
  r.dt_safe = dt_safe;
  r.dt_used = used;
  SPH_TRY(h, cudaMemcpyAsync(h->run, &r, sizeof(r), cudaMemcpyHostToDevice, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  h->opt_rejected_counted = r.rejected;
  return SPH_OK;
}
}  // namespace

int sph_run_optimistic(SphHandle* h, int nsteps, float alpha, float density_limit, uint32_t cooldown_steps,
                       SphRunStats* stats) {
  if (!h || nsteps < 0 || !(alpha > 0.0f) || !std::isfinite(alpha) || !(density_limit >= 0.0f))
    return SPH_ERR_INVALID_ARG;
  if (h->ninst != 1) return set_err(h, SPH_ERR_INVALID_ARG, "the optimistic runner steps one simulation");
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (!h->run) {
    cudaError_t e = dalloc(h, &h->run, 1);
    if (e == cudaSuccess) e = dalloc(h, &h->dt_safe_dev, 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->run, 0, sizeof(sph::RunState), h->st);
    if (e != cudaSuccess) return cuda_status(h, e, "runner state");
  }
  {
    cudaError_t e = ensure_ck(h);
    if (e != cudaSuccess) return cuda_status(h, e, "checkpoint allocation");
  }
  for (int s = 0; s < nsteps && h->n > 0; ++s) {
    ensure_red(h);
    if (h->needs_init || !h->list_valid) {
      int st = opt_step_host(h, alpha, density_limit, cooldown_steps);
      if (st != SPH_OK) return st;
      continue;
    }
    if (h->g_opt && (h->opt_alpha != alpha || h->opt_limit != density_limit || h->opt_cool != cooldown_steps)) {
      cudaGraphExecDestroy(h->g_opt);
      h->g_opt = nullptr;
    }
    if (!h->g_opt) {
      int st = capture_opt(h, alpha, density_limit, cooldown_steps);
      if (st != SPH_OK) return st;
      h->opt_alpha = alpha;
      h->opt_limit = density_limit;
      h->opt_cool = cooldown_steps;
    }
    SPH_TRY(h, cudaGraphLaunch(h->g_opt, h->st));
    h->launches += h->opt_kernels;
    h->list_valid = true;
    h->red_valid = true;
    h->has_ck = true;
  }
  sph::RunState r;
  SPH_TRY(h, cudaMemcpyAsync(&r, h->run, sizeof(r), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  if (r.rejected > h->opt_rejected_counted) {  // retry branches the graphs ran
    h->launches += (r.rejected - h->opt_rejected_counted) * (uint64_t)h->retry_kernels;
    h->opt_rejected_counted = r.rejected;
  }
  if (stats) {
    stats->sim_time = r.sim_time;
    stats->steps = r.steps;
    stats->accepted = r.accepted;
    stats->rejected = r.rejected;
    stats->last_dt = r.dt_used;
    stats->cooldown = r.cooldown;
  }
  return check_device_flags(h);
}

int sph_scale_velocities(SphHandle* h, float factor) {
  if (!h || !std::isfinite(factor)) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n > 0) {
    sph::k_scale_velocities<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->velout, factor);
    h->launches += 1;
    SPH_TRY(h, cudaGetLastError());
  }
  return SPH_OK;
}

int sph_pack_frame(SphHandle* h, uint32_t subsample_count, uint64_t frame_number, double sim_time,
                   uint8_t* out, size_t cap, size_t* bytes) {
  if (!h || !bytes) return SPH_ERR_INVALID_ARG;
  size_t n = (size_t)h->n;
  size_t stride = subsample_count > 0 ? std::max<size_t>(n / subsample_count, 1) : 1;
  size_t count = std::min<size_t>(n / stride, subsample_count);
  size_t need = 21 + 20 * count;
  *bytes = need;
  if (!out) return SPH_OK;
  if (cap < need) return set_err(h, SPH_ERR_INVALID_ARG, "frame buffer too small");
  SPH_TRY(h, cudaSetDevice(h->dev));
  out[0] = 0x02;
  for (int b = 0; b < 8; ++b) out[1 + b] = (uint8_t)(frame_number >> (8 * b));
  uint32_t c32 = (uint32_t)count;
  for (int b = 0; b < 4; ++b) out[9 + b] = (uint8_t)(c32 >> (8 * b));
  uint64_t tb;
  std::memcpy(&tb, &sim_time, 8);
  for (int b = 0; b < 8; ++b) out[13 + b] = (uint8_t)(tb >> (8 * b));
  if (count == 0) return SPH_OK;
  if (!h->temp_dev) {
    float* t = nullptr;
    cudaError_t e = dalloc(h, &t, n);
    if (e != cudaSuccess) return cuda_status(h, e, "frame temperature");
    SPH_TRY(h, cudaMemcpyAsync(t, h->temperature.data(), n * sizeof(float), cudaMemcpyHostToDevice, h->st));
    h->temp_dev = t;
  }
  if (h->frame_cap < count) {
    uint32_t* f = nullptr;
    cudaError_t e = dalloc(h, &f, 5 * count);
    if (e != cudaSuccess) return cuda_status(h, e, "frame buffer");
    h->frame_dev = f;
    h->frame_cap = count;
  }
  sph::k_pack_frame<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->pos, h->velout, h->id, h->temp_dev,
                                                           (uint32_t)stride, (uint32_t)count, h->frame_dev);
  h->launches += 1;
  SPH_TRY(h, cudaMemcpyAsync(out + 21, h->frame_dev, 20 * count, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

int sph_synchronize(SphHandle* h) {
  if (!h) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

int sph_health(SphHandle* h, uint64_t* nonfinite) {
  if (!h || !nonfinite) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  unsigned long long bad = 0;
  SPH_TRY(h, cudaMemsetAsync(h->bad, 0, sizeof(unsigned long long), h->st));
  if (h->n) {
    sph::k_health<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->pos, h->velout, h->bad);
    h->launches += 1;
  }
  SPH_TRY(h, cudaMemcpyAsync(&bad, h->bad, sizeof(bad), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  *nonfinite = bad;
  int s = check_device_flags(h);
  if (s != SPH_OK) return s;
  return bad ? set_err(h, SPH_ERR_NONFINITE, "non-finite particle state") : SPH_OK;
}

const char* sph_last_error(const SphHandle* h) { return h ? h->error.c_str() : "null handle"; }

void* sph_stream(SphHandle* h) { return h ? (void*)h->st : nullptr; }

uint64_t sph_launch_count(const SphHandle* h) { return h ? h->launches : 0; }

int sph_set_geometry_sdf(SphHandle* h, const SphSdfView* g) {
  if (!h || !g || !g->distances || !(g->cell_size > 0.0f)) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  // force.rs:47-81: nodes with |d| <= 2h and d <= 0 and a unit normal, in
  // (i, j, k) order.
  float thr = 2.0f * h->prm.h;
  std::vector<float4> np_, nn_;
  for (uint32_t i = 0; i < g->dims[0]; ++i)
    for (uint32_t j = 0; j < g->dims[1]; ++j)
      for (uint32_t k = 0; k < g->dims[2]; ++k) {
        float px = g->origin[0] + (float)i * g->cell_size;
        float py = g->origin[1] + (float)j * g->cell_size;
        float pz = g->origin[2] + (float)k * g->cell_size;
        float d = host_sdf_sample(*g, px, py, pz);
        if (std::fabs(d) > thr || d > 0.0f) continue;
        float n[3];
        host_sdf_gradient(*g, px, py, pz, n);
        float mag = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (mag < 1e-8f) continue;
        np_.push_back(make_float4(px, py, pz, d));
        nn_.push_back(make_float4(n[0], n[1], n[2], 0.0f));
      }
  if (!h->geo_sum) {
    cudaError_t e = dalloc(h, &h->geo_sum, 6);
    if (e != cudaSuccess) return cuda_status(h, e, "geometry allocation");
  }
  h->geo_nodes = (int)np_.size();
  h->geo_area = g->cell_size * g->cell_size;
  cudaError_t e = cudaSuccess;
  if (h->geo_nodes) {
    e = dalloc(h, &h->geo_pos, np_.size());
    if (e == cudaSuccess) e = dalloc(h, &h->geo_nrm, nn_.size());
    if (e == cudaSuccess) e = dalloc(h, &h->geo_out, np_.size() * 6);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h->geo_pos, np_.data(), np_.size() * sizeof(float4), cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h->geo_nrm, nn_.data(), nn_.size() * sizeof(float4), cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  }
  return cuda_status(h, e, "sph_set_geometry_sdf");
}

int sph_surface_forces(SphHandle* h, SphSurfaceForce* out) {
  if (!h || !out) return SPH_ERR_INVALID_ARG;
  if (!h->geo_sum) return set_err(h, SPH_ERR_INVALID_ARG, "no geometry SDF registered");
  SPH_TRY(h, cudaSetDevice(h->dev));
  std::memset(out, 0, sizeof(*out));
  out->nodes = (uint32_t)h->geo_nodes;
  if (h->geo_nodes == 0 || h->n == 0) return SPH_OK;
  using namespace sph;
  k_surface_nodes<<<grid_for(h->geo_nodes, kSurfWarps), kSurfWarps * 32, 0, h->st>>>(
      h->k, h->geo_nodes, h->geo_pos, h->geo_nrm, h->geo_area, h->pos, h->pr, h->id, h->ctab, h->geo_out,
      h->err);
  k_sum_rows_f64<<<1, 256, 0, h->st>>>(h->geo_nodes, 6, h->geo_out, h->geo_sum);
  h->launches += 2;
  std::vector<float> rows((size_t)h->geo_nodes * 6);
  double sums[6];
  SPH_TRY(h, cudaMemcpyAsync(rows.data(), h->geo_out, rows.size() * 4, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaMemcpyAsync(sums, h->geo_sum, sizeof(sums), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  float f32[6] = {0, 0, 0, 0, 0, 0};
  for (int nd = 0; nd < h->geo_nodes; ++nd) {
    const float* r = &rows[(size_t)nd * 6];
    if (r[0] != 0.0f || r[1] != 0.0f || r[2] != 0.0f || r[3] != 0.0f || r[4] != 0.0f || r[5] != 0.0f)
      out->active_nodes++;
    for (int a = 0; a < 6; ++a) f32[a] += r[a];
  }
  for (int a = 0; a < 3; ++a) {
    out->force[a] = sums[a];
    out->moment[a] = sums[3 + a];
    out->force_f32[a] = f32[a];
    out->moment_f32[a] = f32[3 + a];
  }
  return check_device_flags(h);
}

int sph_body_force(SphHandle* h, uint32_t first, uint32_t count, SphBodyForce* out) {
  if (!h || !out) return SPH_ERR_INVALID_ARG;
  if ((uint64_t)first + count > (uint64_t)h->nb) return set_err(h, SPH_ERR_INVALID_ARG, "body range");
  SPH_TRY(h, cudaSetDevice(h->dev));
  std::memset(out, 0, sizeof(*out));
  if (h->n == 0 || count == 0) return SPH_OK;
  using namespace sph;
  int parts = grid_for(h->n, 256);
  if (parts > h->body_parts) {
    cudaError_t e = dalloc(h, &h->body_part, (size_t)parts * kBodyCols);
    if (e == cudaSuccess && !h->body_sum) e = dalloc(h, &h->body_sum, kBodyCols);
    if (e != cudaSuccess) return cuda_status(h, e, "body force allocation");
    h->body_parts = parts;
  }
  k_body_force<<<parts, 256, 0, h->st>>>(h->k, h->n, first, count, h->pos, h->vel, h->rf, h->pr, h->id,
                                         h->bc_start, h->bc_list, h->bpos, h->bpress, h->body_part);
  k_sum_parts_f64<<<1, 32, 0, h->st>>>(parts, kBodyCols, h->body_part, h->body_sum);
  h->launches += 2;
  double v[kBodyCols];
  SPH_TRY(h, cudaMemcpyAsync(v, h->body_sum, sizeof(v), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  double* dst[6] = {out->pressure_force, out->pressure_moment, out->repulsion_force,
                    out->repulsion_moment, out->viscous_force, out->viscous_moment};
  for (int t = 0; t < 6; ++t)
    for (int a = 0; a < 3; ++a) dst[t][a] = v[3 * t + a];
  return check_device_flags(h);
}

int sph_batch_info(const SphHandle* h, int* ninst, size_t* first, size_t* count) {
  if (!h || !ninst) return SPH_ERR_INVALID_ARG;
  *ninst = h->ninst;
  for (int q = 0; q < h->ninst; ++q) {
    if (first) first[q] = h->poff[q];
    if (count) count[q] = h->poff[q + 1] - h->poff[q];
  }
  return SPH_OK;
}

int sph_batch_timesteps(SphHandle* h, float* dt_out) {
  if (!h || !dt_out) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  if (h->n == 0) return SPH_ERR_INVALID_ARG;
  ensure_red(h);
  enqueue_dt_finalize(h, h->dt_query);
  SPH_TRY(h, cudaMemcpyAsync(dt_out, h->dt_query, sizeof(float) * h->ninst, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

int sph_set_launch(SphHandle* h, const SphLaunch* l) {
  if (!h || !l) return SPH_ERR_INVALID_ARG;
  int v[3] = {l->xsph_threads, l->density_threads, l->forces_threads};
  for (int x : v)
    if (x < 32 || x > 512 || (x & 31)) return set_err(h, SPH_ERR_INVALID_ARG, "threads per block");
  h->bs_xsph = v[0];
  h->bs_density = v[1];
  h->bs_forces = v[2];
  drop_graphs(h);  // recaptured with the new shapes on the next step
  return SPH_OK;
}

int sph_get_launch(const SphHandle* h, SphLaunch* l) {
  if (!h || !l) return SPH_ERR_INVALID_ARG;
  l->xsph_threads = h->bs_xsph;
  l->density_threads = h->bs_density;
  l->forces_threads = h->bs_forces;
  return SPH_OK;
}

// Autotuner cache: (device name, instance count, log2 histogram of instance
// sizes) -> best launch shapes.
static std::mutex g_tune_mu;
static std::map<std::string, SphLaunch> g_tune_cache;

static std::string tune_key(SphHandle* h) {
  cudaDeviceProp prop;
  std::string key = cudaGetDeviceProperties(&prop, h->dev) == cudaSuccess ? prop.name : "?";
  int hist[40] = {0};
  for (int q = 0; q < h->ninst; ++q) {
    size_t c = h->poff[q + 1] - h->poff[q];
    int b = 0;
    while ((c >> b) > 1 && b < 39) ++b;
    hist[b]++;
  }
  key += "|" + std::to_string(h->ninst);
  for (int b = 0; b < 40; ++b)
    if (hist[b]) key += "|" + std::to_string(b) + ":" + std::to_string(hist[b]);
  return key;
}

int sph_autotune(SphHandle* h, int trial_steps, SphLaunch* best) {
  if (!h || !best || trial_steps < 1) return SPH_ERR_INVALID_ARG;
  std::string key = tune_key(h);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      *best = it->second;
      return sph_set_launch(h, best);
    }
  }
  const int cand[4] = {64, 128, 256, 512};
  float t_best[3] = {1e30f, 1e30f, 1e30f};
  int s_best[3] = {256, 256, 256};
  float dt = 0.0f;
  int st = sph_compute_timestep(h, &dt);
  if (st != SPH_OK) return st;
  // one untimed step so that every trial starts from a stepped state
  SphStepProfile prof;
  st = sph_step_profiled(h, dt, &prof);
  if (st != SPH_OK) return st;
  for (int c : cand) {
    SphLaunch l{c, c, c};
    st = sph_set_launch(h, &l);
    if (st != SPH_OK) return st;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int r = 0; r < trial_steps; ++r) {
      st = sph_step_profiled(h, dt, &prof);
      if (st != SPH_OK) return st;
      acc[0] += prof.xsph_drift_us;
      acc[1] += prof.density_us;
      acc[2] += prof.forces_us;
    }
    for (int a = 0; a < 3; ++a)
      if (acc[a] < t_best[a]) { t_best[a] = acc[a]; s_best[a] = c; }
  }
  best->xsph_threads = s_best[0];
  best->density_threads = s_best[1];
  best->forces_threads = s_best[2];
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = *best;
  }
  return sph_set_launch(h, best);
}

static int upload_ktab(SphHandle* h) {
  h->k = h->ktab_h[0];
  drop_graphs(h);  // captured launches hold the old constants
  if (h->ninst > 1)
    SPH_TRY(h, cudaMemcpyAsync(h->ktab, h->ktab_h.data(), h->ninst * sizeof(SimConst), cudaMemcpyHostToDevice,
                               h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  return SPH_OK;
}

int sph_batch_set_feature_sdfs(SphHandle* h, const SphSdfView* sdfs) {
  if (!h || !sdfs) return SPH_ERR_INVALID_ARG;
  if (h->k.sdf_mode) return set_err(h, SPH_ERR_INVALID_ARG, "SDF wall mode uses its wall SDF for features");
  SPH_TRY(h, cudaSetDevice(h->dev));
  uint64_t total = 0;
  for (int q = 0; q < h->ninst; ++q) {
    const SphSdfView& g = sdfs[q];
    if (!g.distances || !(g.cell_size > 0.0f) || g.dims[0] < 2 || g.dims[1] < 2 || g.dims[2] < 2)
      return SPH_ERR_INVALID_ARG;
    total += (uint64_t)g.dims[0] * g.dims[1] * g.dims[2];
  }
  float* d = nullptr;
  cudaError_t e = dalloc(h, &d, total);
  if (e != cudaSuccess) return cuda_status(h, e, "feature SDF allocation");
  uint64_t off = 0;
  for (int q = 0; q < h->ninst; ++q) {
    const SphSdfView& g = sdfs[q];
    uint64_t cnt = (uint64_t)g.dims[0] * g.dims[1] * g.dims[2];
    SPH_TRY(h, cudaMemcpyAsync(d + off, g.distances, cnt * sizeof(float), cudaMemcpyHostToDevice, h->st));
    SimConst& k = h->ktab_h[q];
    k.feat_sdf = 1;
    k.sdf_off = (long long)off;
    k.sdf_cell = g.cell_size;
    for (int a = 0; a < 3; ++a) {
      k.sdf_origin[a] = g.origin[a];
      k.sdf_dims[a] = (int)g.dims[a];
    }
    off += cnt;
  }
  h->sdf = d;
  return upload_ktab(h);
}

int sph_set_feature_sdf(SphHandle* h, const SphSdfView* sdf) {
  if (!h || !sdf || h->ninst != 1) return SPH_ERR_INVALID_ARG;
  return sph_batch_set_feature_sdfs(h, sdf);
}

int sph_set_closure(SphHandle* h, int mode, const float* params) {
  if (!h || mode < 0 || mode > 2 || (mode == 2 && !params)) return SPH_ERR_INVALID_ARG;
  if (mode > 0 && !h->k.feat_sdf) return set_err(h, SPH_ERR_INVALID_ARG, "closure needs a geometry SDF");
  SPH_TRY(h, cudaSetDevice(h->dev));
  size_t n = (size_t)h->n;
  if (mode > 0 && !h->cl_count) {
    cudaError_t e = dalloc(h, &h->cl_count, 1);
    if (e == cudaSuccess) e = dalloc(h, &h->cl_slot, n);
    if (e == cudaSuccess) e = dalloc(h, &h->cl_feat, n * 16);
    if (e == cudaSuccess) e = dalloc(h, &h->cl_rho, n);
    if (e == cudaSuccess) e = dalloc(h, &h->corr, n);
    if (e == cudaSuccess) e = dalloc(h, &h->cl_wf, sphmlp::kParams);
    if (e == cudaSuccess) e = dalloc(h, &h->cl_wb, sphmlp::kBf16Count);
    if (e != cudaSuccess) return cuda_status(h, e, "closure allocation");
    SPH_TRY(h, cudaMemsetAsync(h->cl_count, 0, sizeof(uint32_t), h->st));
    SPH_TRY(h, cudaMemsetAsync(h->corr, 0, std::max<size_t>(n, 1) * sizeof(float4), h->st));
  }
  if (mode == 2) {
    std::vector<__nv_bfloat16> wb(sphmlp::kBf16Count);
    for (int i = 0; i < sphmlp::kParams; ++i) {
      int bi = sphmlp::bf16_index(i);
      if (bi >= 0) wb[bi] = __float2bfloat16_rn(params[i]);
    }
    SPH_TRY(h, cudaMemcpyAsync(h->cl_wf, params, sphmlp::kParams * sizeof(float), cudaMemcpyHostToDevice, h->st));
    SPH_TRY(h, cudaMemcpyAsync(h->cl_wb, wb.data(), wb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice,
                               h->st));
    SPH_TRY(h, cudaStreamSynchronize(h->st));
  }
  h->cl_mode = mode;
  drop_graphs(h);
  return SPH_OK;
}

int sph_closure_samples(SphHandle* h, size_t cap, uint32_t* ids, float* features, float* rho, size_t* count) {
  if (!h || !count || (cap && (!ids || !features || !rho))) return SPH_ERR_INVALID_ARG;
  if (!h->cl_mode) return set_err(h, SPH_ERR_INVALID_ARG, "closure capture is off");
  SPH_TRY(h, cudaSetDevice(h->dev));
  uint32_t c = 0;
  SPH_TRY(h, cudaMemcpyAsync(&c, h->cl_count, 4, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  *count = c;
  size_t m = std::min<size_t>(cap, c);
  if (m == 0) return SPH_OK;
  std::vector<uint32_t> slots(m), all_ids((size_t)h->n);
  SPH_TRY(h, cudaMemcpyAsync(slots.data(), h->cl_slot, m * 4, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaMemcpyAsync(all_ids.data(), h->id, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaMemcpyAsync(features, h->cl_feat, m * 16 * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaMemcpyAsync(rho, h->cl_rho, m * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  SPH_TRY(h, cudaStreamSynchronize(h->st));
  for (size_t q = 0; q < m; ++q) ids[q] = all_ids[slots[q]] & sph::kIdMask;
  return SPH_OK;
}

int sph_interpolate(SphHandle* h, const float* pts, size_t npts, float* out) {
  if (!h || (npts && (!pts || !out)) || h->ninst != 1 || npts > 0x7fffffffull) return SPH_ERR_INVALID_ARG;
  if (npts == 0 || h->n == 0) {
    if (npts) std::memset(out, 0, npts * 7 * sizeof(float));
    return SPH_OK;
  }
  SPH_TRY(h, cudaSetDevice(h->dev));
  std::vector<float4> p4(npts);
  for (size_t q = 0; q < npts; ++q) p4[q] = make_float4(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2], 0.0f);
  float4* dp = nullptr;
  float* dout = nullptr;
  cudaError_t e = cudaMalloc((void**)&dp, npts * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dout, npts * 7 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, p4.data(), npts * sizeof(float4), cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) {
    sph::k_interpolate<<<grid_for((long long)npts, 128), 128, 0, h->st>>>(sph::OneSim{h->k}, (int)npts, dp, h->pos,
                                                                          h->rf, h->pr, h->acc, h->ctab, dout);
    h->launches += 1;
    e = cudaMemcpyAsync(out, dout, npts * 7 * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (dp) cudaFree(dp);
  if (dout) cudaFree(dout);
  return cuda_status(h, e, "sph_interpolate");
}

int sph_grid_info(SphHandle* h, SphGridInfo* out) {
  if (!h || !out) return SPH_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a) {
    out->dims[a] = (uint32_t)h->k.dims[a];
    out->grid_min[a] = h->k.gmin[a];
  }
  out->total_cells = (uint32_t)h->C;
  out->cell_size = h->k.cell;
  out->boundary_candidates = h->boundary_candidates;
  return SPH_OK;
}

int sph_read_grid(SphHandle* h, uint32_t* cell_linear, uint32_t* morton_key, uint32_t* cell_count,
                  uint32_t* cell_start, uint32_t* slot_id) {
  if (!h) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  size_t n = (size_t)h->n, C = (size_t)h->C;
  uint32_t* d_lin = nullptr;
  uint32_t* d_mor = nullptr;
  if ((cell_linear || morton_key) && n) {
    SPH_TRY(h, cudaMalloc(&d_lin, n * sizeof(uint32_t)));
    cudaError_t e = cudaMalloc(&d_mor, n * sizeof(uint32_t));
    if (e != cudaSuccess) { cudaFree(d_lin); return cuda_status(h, e, "sph_read_grid"); }
    sph::k_grid_keys<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->k, h->n, h->pos, h->id, d_lin, d_mor);
    h->launches += 1;
    if (cell_linear) cudaMemcpyAsync(cell_linear, d_lin, n * 4, cudaMemcpyDeviceToHost, h->st);
    if (morton_key) cudaMemcpyAsync(morton_key, d_mor, n * 4, cudaMemcpyDeviceToHost, h->st);
  }
  std::vector<uint2> tab;
  if (cell_count || cell_start) {
    tab.resize(C);
    cudaMemcpyAsync(tab.data(), h->ctab, C * sizeof(uint2), cudaMemcpyDeviceToHost, h->st);
  }
  if (slot_id && n) cudaMemcpyAsync(slot_id, h->id, n * 4, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (d_lin) cudaFree(d_lin);
  if (d_mor) cudaFree(d_mor);
  if (e != cudaSuccess) return cuda_status(h, e, "sph_read_grid");
  for (size_t c = 0; c < tab.size(); ++c) {
    if (cell_start) cell_start[c] = tab[c].x;
    if (cell_count) cell_count[c] = tab[c].y;
  }
  if (slot_id)
    for (size_t s = 0; s < n; ++s) slot_id[s] &= sph::kIdMask;
  return check_device_flags(h);
}

int sph_neighbors(SphHandle* h, uint32_t id, uint32_t* out, size_t cap, size_t* count) {
  if (!h || !count || (cap && !out) || id >= (uint32_t)h->n) return SPH_ERR_INVALID_ARG;
  SPH_TRY(h, cudaSetDevice(h->dev));
  uint32_t* d_out = nullptr;
  size_t c2 = std::max<size_t>(cap, 1);
  SPH_TRY(h, cudaMalloc(&d_out, c2 * sizeof(uint32_t)));
  sph::k_find_slot<<<grid_for(h->n, 256), 256, 0, h->st>>>(h->n, h->id, id, h->diag);
  sph::k_list_neighbors<<<1, 1, 0, h->st>>>(h->k, h->pos, h->id, h->ctab, h->diag, d_out, (uint32_t)cap,
                                            h->diag + 1);
  h->launches += 2;
  uint32_t cnt = 0;
  cudaMemcpyAsync(&cnt, h->diag + 1, 4, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e == cudaSuccess && cap) {
    e = cudaMemcpy(out, d_out, std::min<size_t>(cap, cnt) * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  }
  cudaFree(d_out);
  if (e != cudaSuccess) return cuda_status(h, e, "sph_neighbors");
  *count = cnt;
  return SPH_OK;
}

}  // extern "C"
