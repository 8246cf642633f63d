/*
 * sph_cuda.h - C ABI of the B200 (sm_100a) WCSPH step.
 *
 * Drop-in for the reference crate `kernel`'s backend interface
 * (tim-ai-twin/ultraballpit, backend/crates/kernel/src/lib.rs:58-78):
 *
 *   pub trait SimulationKernel {
 *       fn step(&mut self, dt: f32);
 *       fn particles(&self) -> &ParticleArrays;
 *       fn error_metrics(&self) -> ErrorMetrics;
 *       fn particle_count(&self) -> usize;
 *       fn save_checkpoint(&mut self) -> bool;
 *       fn restore_checkpoint(&mut self) -> bool;
 *   }
 *
 * A Rust `CudaKernel` implements that trait over an opaque SphHandle through
 * a thin FFI module declaring these functions. Every entry point returns an
 * SphStatus (0 = ok) and never aborts; the handle is Send but not Sync:
 * calls on one handle must not overlap, and each call makes the handle's
 * device current, so the handle may move between host threads.
 *
 * All arrays are plain host pointers; the library copies inputs to its own
 * device memory at creation and owns every device allocation, stream and
 * CUDA graph it uses.
 *
 * Environment variables read at creation: SPH_TRACE (any value) prints the
 * creation's phase times on stderr; SPH_WARP_SCAN_MIN and
 * SPH_ADAMI_CELLS_MIN (counts) replace the sizes from which the density scan
 * and the boundary pressure take their warp-cooperative forms (2048 fluid
 * and 4096 boundary particles per SM; 0 = always). Both forms give the same
 * results bit for bit.
 */
#ifndef SPH_CUDA_H
#define SPH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH_ABI_VERSION 1

typedef struct SphHandle SphHandle;

typedef enum SphStatus {
  SPH_OK = 0,
  SPH_ERR_INVALID_ARG = 1,   /* null pointer, size mismatch, bad parameter */
  SPH_ERR_OOM = 2,           /* device allocation failed */
  SPH_ERR_CUDA = 3,          /* any other CUDA runtime error */
  SPH_ERR_NONFINITE = 4,     /* a NaN/Inf state was detected (sph_health) */
  SPH_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  SPH_ERR_CAPACITY = 6,      /* a per-cell / per-boundary-particle bound was exceeded */
  SPH_ERR_NO_DEVICE = 7,     /* no CUDA device, or not an sm_100 device */
  SPH_ERR_NO_CHECKPOINT = 8  /* restore without a saved checkpoint */
} SphStatus;

typedef enum SphBoundaryMode {
  SPH_BOUNDARY_PARTICLES = 0, /* reference walls: frozen particles, Adami pressure */
  SPH_BOUNDARY_SDF = 1        /* homogenised walls: the six faces of the domain box and an
                                 obstacle given by a trilinear SDF (no reference counterpart) */
} SphBoundaryMode;

typedef enum SphCellOrder {
  SPH_CELL_ORDER_MORTON = 0, /* particles stored by (30-bit Morton cell rank, id) */
  SPH_CELL_ORDER_LINEAR = 1, /* particles stored by (linear cell hash, id): the reference sorted_indices */
  SPH_CELL_ORDER_ROWS = 2    /* the cells of each x-row stored consecutively, the rows in Morton order
                                over (y, z): a neighbourhood's three cells of a row are one range */
} SphCellOrder;

/* Stage switches; SPH_FLAGS_REFERENCE keeps every reference stage on
 * (kernel/src/lib.rs:216-234, 310-324; boundary.rs:143-181, 239-291). */
typedef enum SphFlags {
  SPH_FLAG_DELTA_SPH = 1u << 0,
  SPH_FLAG_XSPH = 1u << 1,
  SPH_FLAG_REPULSION = 1u << 2,
  SPH_FLAG_DOMAIN_CLAMP = 1u << 3,
  SPH_FLAGS_REFERENCE = 0xFu
} SphFlags;

/* Arguments of CpuKernel::new (kernel/src/lib.rs:138-148) plus the stage
 * parameters the reference hardcodes (alpha = 1, beta = 2 at sph.rs:440-441). */
typedef struct SphParams {
  float h;                /* smoothing length; cell size is 2h */
  float gravity[3];
  float speed_of_sound;   /* used as given (no auto-tune, orchestrator lib.rs:157-159) */
  float cfl_number;
  float viscosity;        /* kept for the trait's constructor; unused, as in the reference */
  float domain_min[3];
  float domain_max[3];
  float alpha;            /* Monaghan alpha */
  float beta;             /* Monaghan beta */
  int32_t boundary_mode;  /* SphBoundaryMode */
  int32_t cell_order;     /* SphCellOrder */
  uint32_t flags;         /* SphFlags */
  int32_t device;         /* CUDA device ordinal */
  float sdf_wall_coef;    /* SPH_BOUNDARY_SDF: wall repulsion scale (m/s^2) */
} SphParams;

/* Fluid particles (kernel/src/particle.rs:22-58), host SoA, n entries each. */
typedef struct SphParticlesView {
  size_t n;
  const float *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  const float *density, *pressure, *mass, *temperature;
  const uint8_t *fluid_type; /* 0 = Water, 1 = Air */
} SphParticlesView;

typedef struct SphParticlesMut {
  size_t n;
  float *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  float *density, *pressure, *mass, *temperature;
  uint8_t *fluid_type;
} SphParticlesMut;

/* Boundary particles (kernel/src/boundary.rs:20-37); pressure starts at 0. */
typedef struct SphBoundaryView {
  size_t n;
  const float *x, *y, *z, *mass, *nx, *ny, *nz;
} SphBoundaryView;

/* GridSDF (orchestrator/src/geometry.rs:11-20): node (i,j,k) at
 * origin + (i,j,k) * cell_size, index i*ny*nz + j*nz + k. */
typedef struct SphSdfView {
  float origin[3];
  float cell_size;
  uint32_t dims[3];
  const float *distances;
} SphSdfView;

/* kernel/src/lib.rs:40-47 */
typedef struct SphErrorMetrics {
  float max_density_variation;
  float energy_conservation;
  float mass_conservation;
} SphErrorMetrics;

/* Per-stage device time of one step in microseconds (the counterpart of
 * GpuStepProfile, kernel/src/gpu/mod.rs:35-52). */
typedef struct SphStepProfile {
  float xsph_drift_us;        /* kick 1 + XSPH + drift + clamp + binning */
  float sort_us;              /* scan + fill + reorder */
  float density_us;           /* density + delta-SPH + EOS */
  float boundary_pressure_us; /* Adami boundary pressure */
  float forces_us;            /* pressure + viscosity + gravity + walls + kick 2 + dt reduce */
  float total_us;
} SphStepProfile;

/* Force and moment on a geometry from orchestrator force.rs:39-129
 * (compute_surface_forces): FP64 sums over the SDF surface nodes, and the
 * reference's own f32 sums in node order. Moments about the origin. */
typedef struct SphSurfaceForce {
  double force[3];
  double moment[3];
  float force_f32[3];
  float moment_f32[3];
  uint32_t nodes;        /* SDF nodes with -2h <= d <= 0 and a defined normal */
  uint32_t active_nodes; /* of those, nodes with fluid in support */
} SphSurfaceForce;

/* Reaction of the fluid on a range of boundary particles (a body), FP64:
 * pressure = the boundary pressure force (kernel/src/sph.rs:391-408) the
 * fluid receives from them, negated; repulsion = likewise for
 * boundary.rs:161-179; viscous = Monaghan viscosity with the body at rest
 * (a diagnostic: the reference applies no wall viscosity). Moments about the
 * origin, taken at the boundary particles. */
typedef struct SphBodyForce {
  double pressure_force[3], pressure_moment[3];
  double repulsion_force[3], repulsion_moment[3];
  double viscous_force[3], viscous_moment[3];
} SphBodyForce;

/* Threads per block of the three neighbour kernels (32..512, multiple of 32). */
typedef struct SphLaunch {
  int32_t xsph_threads;
  int32_t density_threads;
  int32_t forces_threads;
} SphLaunch;

typedef struct SphGridInfo {
  uint32_t dims[3];
  uint32_t total_cells;
  float cell_size;
  float grid_min[3];
  uint64_t boundary_candidates; /* entries of the static per-cell boundary lists */
} SphGridInfo;

/* Fill `p` with the reference defaults: alpha 1, beta 2, all reference
 * stages on, boundary particles, device 0; cell order SPH_CELL_ORDER_ROWS
 * (storage order only: the physics is the same in every order). */
void sph_params_default(SphParams *p);

/* CpuKernel::new / GpuKernel::new (lib.rs:138-174, gpu/mod.rs:190-200).
 * `boundary` may be NULL (no walls). With SPH_BOUNDARY_SDF the walls are
 * the faces of the domain box (which must span at least 4h on every axis)
 * plus the obstacle whose SDF `sdf` gives (NULL, or NULL distances: no
 * obstacle); otherwise `sdf` is ignored. Creation uses the host's hardware
 * threads (up to 32) for its tables and allocates the device arrays on a
 * second thread; it returns once the handle is ready. The device arrays come
 * from a memory pool the library keeps per device. */
int sph_create(const SphParams *params, const SphParticlesView *particles,
               const SphBoundaryView *boundary, const SphSdfView *sdf, SphHandle **out);
/* Releases the handle. Its device arrays go back to the library's pool,
 * which keeps them for the next handle created on that device (creating
 * simulations one after another then skips the driver's mapping of fresh
 * memory); the pool's memory stays reserved until the process exits. */
void sph_destroy(SphHandle *h);

/* SimulationKernel::step (lib.rs:287-335). Enqueued asynchronously. */
int sph_step(SphHandle *h, float dt);
/* `nsteps` steps whose dt is computed on the device from the state, exactly
 * as sph::compute_timestep (sph.rs:591-628) would on particles(); the last
 * dt is written to `dt_out` (may be NULL, no host sync then). */
int sph_step_auto(SphHandle *h, int nsteps, float *dt_out);
/* sph::compute_timestep(particles(), h, c, cfl_number) evaluated on the device. */
int sph_compute_timestep(SphHandle *h, float *dt_out);
/* One step run stage by stage with CUDA events; fills `prof` (host sync). */
int sph_step_profiled(SphHandle *h, float dt, SphStepProfile *prof);

/* SimulationKernel::particles: copy the state into caller-owned arrays in the
 * original particle order (synchronizes). `out->n` must equal the count. */
int sph_read_particles(SphHandle *h, SphParticlesMut *out);
/* Boundary pressures of the last force computation (n = boundary count). */
int sph_read_boundary_pressure(SphHandle *h, float *out, size_t n);
/* SimulationKernel::error_metrics (lib.rs:341-377): FP64 sums on the device. */
int sph_error_metrics(SphHandle *h, SphErrorMetrics *out);
/* SimulationKernel::particle_count */
size_t sph_particle_count(const SphHandle *h);
/* SimulationKernel::save_checkpoint / restore_checkpoint (lib.rs:383-395):
 * device-to-device copies; restore takes the checkpoint (a second restore
 * returns SPH_ERR_NO_CHECKPOINT). */
int sph_save_checkpoint(SphHandle *h);
int sph_restore_checkpoint(SphHandle *h);

/* The viewer's Frame message (server ws.rs:233-290) packed on the device:
 * tag 0x02, frame_number (u64), count (u32), sim_time (f64), then per
 * particle o = k * stride (stride = max(n / subsample_count, 1), k < count,
 * count = min(n / stride, subsample_count)): x, y, z, temperature (f32),
 * fluid type (u8), density ratio (u16), 0 (u8); little endian, no padding.
 * *bytes gets the message size (21 + 20 count); out NULL only queries it.
 * Reads back 20 bytes per sampled particle instead of the whole state. */
int sph_pack_frame(SphHandle *h, uint32_t subsample_count, uint64_t frame_number, double sim_time,
                   uint8_t *out, size_t cap, size_t *bytes);
/* The reference runner's optimistic time stepping (orchestrator
 * runner.rs:189-240) on the device: per step dt_safe = compute_timestep;
 * outside a cooldown a checkpoint, a step of dt_safe * alpha, and if the
 * maximum density variation then exceeds density_limit a restore, a step of
 * dt_safe and `cooldown_steps` steps without optimism. Each step is one
 * graph launch (a conditional node takes the retry branch), so the host
 * does not wait between steps. The reference's constants are alpha 1.5,
 * limit 0.03, cooldown 10; alpha must be positive and finite, the limit
 * non-negative (infinity accepts every step). Counters accumulate over calls; `stats` (may be
 * NULL) gets them after the last step. One simulation per handle; the
 * handle's checkpoint is the runner's, left at the start of its last step. */
typedef struct SphRunStats {
  double sim_time;
  uint64_t steps, accepted, rejected;
  float last_dt;
  uint32_t cooldown;
} SphRunStats;
int sph_run_optimistic(SphHandle *h, int nsteps, float alpha, float density_limit, uint32_t cooldown_steps,
                       SphRunStats *stats);
/* ---- domain setup (orchestrator domain.rs:36-402) on the device ---- */
#define SPH_FLUID_WATER 0
#define SPH_FLUID_AIR 1
#define SPH_FLUID_MIXED 2 /* y below the box's middle is water, above it air */
/* The SimulationConfig fields setup_domain reads (config.rs:9-64). */
typedef struct SphDomainSpec {
  float particle_spacing;
  float domain_min[3], domain_max[3];
  int fluid_type; /* SPH_FLUID_* (config.rs:66-73) */
  float initial_temperature;
  /* bit f set: face f is Simple(Wall); f = 0..5 is x_min, x_max, y_min,
   * y_max, z_min, z_max (BoundaryConditions::default() = 0x3f) */
  uint32_t wall_faces;
} SphDomainSpec;
typedef struct SphBoundaryMut {
  size_t n;
  float *x, *y, *z, *mass, *nx, *ny, *nz;
} SphBoundaryMut;
/* setup_domain(config, sdf) (domain.rs:36-83) on `device`: the fluid
 * particles of the lattice (domain.rs:88-160) and the boundary particles,
 * wall layers face by face (domain.rs:162-348) then geometry layers
 * (domain.rs:351-402), in the reference's order and bit for bit. The SDF's
 * distances are read from host or device memory. *n_fluid / *n_boundary get
 * the counts; with fluid and boundary both NULL nothing else happens.
 * Otherwise each non-NULL output (host or device arrays, capacity in its n
 * field) receives its particles; a capacity below the count returns
 * SPH_ERR_CAPACITY. The lattice may hold at most 2^31 - 1 points. */
int sph_setup_domain(int device, const SphDomainSpec *spec, const SphSdfView *sdf, SphParticlesMut *fluid,
                     SphBoundaryMut *boundary, size_t *n_fluid, size_t *n_boundary);

/* Multiply every particle's velocity by `factor` (no reference
 * counterpart). 0 between steps is kinetic damping: relaxing an initial
 * lattice into its equilibrium before a run. */
int sph_scale_velocities(SphHandle *h, float factor);
/* Wait for queued work; reports a deferred device-side error, if any. */
int sph_synchronize(SphHandle *h);
/* Count of particles with a non-finite position, velocity or density. */
int sph_health(SphHandle *h, uint64_t *nonfinite_out);
const char *sph_last_error(const SphHandle *h);
/* The cudaStream_t all work of the handle is enqueued on. */
void *sph_stream(SphHandle *h);
/* Total kernels this handle has launched (graph replays counted per node). */
uint64_t sph_launch_count(const SphHandle *h);

/* ---- batches of independent simulations (no reference counterpart) -----
 * `ninst` simulations on one device stepped by the same kernel launches
 * (one launch per stage for the whole batch), each with its own grid,
 * constants, walls and dt. Boundary-particle mode only; `boundaries` may be
 * NULL or hold n = 0 entries. Every single-simulation entry point works on
 * a batch handle: sph_step sets one dt for all instances, sph_step_auto
 * computes one dt per instance on the device, sph_read_particles returns
 * the instances one after another (see sph_batch_info), sph_error_metrics
 * sums over all instances. */
int sph_batch_create(int ninst, const SphParams *params, const SphParticlesView *particles,
                     const SphBoundaryView *boundaries, SphHandle **out);
/* A batch in SDF wall mode: one obstacle SDF per instance (NULL distances:
 * none; `sdfs` NULL: none anywhere), all instances with the same h, which
 * fixes the shared wall table. */
int sph_batch_create_sdf(int ninst, const SphParams *params, const SphParticlesView *particles,
                         const SphSdfView *sdfs, SphHandle **out);
/* Instance count, and per instance the first particle and particle count in
 * the concatenated order (first/count may be NULL, else ninst entries). */
int sph_batch_info(const SphHandle *h, int *ninst, size_t *first, size_t *count);
/* One step with instance q advanced by dts[q] (ninst floats, host). */
int sph_batch_step(SphHandle *h, const float *dts);
/* Per-instance sph::compute_timestep on the device (ninst floats). */
int sph_batch_timesteps(SphHandle *h, float *dt_out);
/* Launch shapes of the neighbour kernels (graphs are recaptured). */
int sph_set_launch(SphHandle *h, const SphLaunch *launch);
int sph_get_launch(const SphHandle *h, SphLaunch *launch);
/* Autotuner: times each kernel at 64/128/256/512 threads per block over
 * `trial_steps` profiled steps (after one untimed step) and applies the
 * fastest shape per kernel. Results are cached per process by device name
 * and instance-size histogram; a cache hit runs no step. The trial steps
 * advance the simulation: tune a scratch handle of the same workload. */
int sph_autotune(SphHandle *h, int trial_steps, SphLaunch *best);

/* ---- learned near-wall closure network (no reference counterpart) -----
 * MLP 16 -> 64 -> 64 -> 4 with SiLU; BF16 operands on the tensor cores with
 * FP32 accumulation, FP32 master weights and Adam state on the device.
 * Parameters (5,508 floats): W1[64][16], b1[64], W2[64][64], b2[64],
 * W3[4][64], b3[4]. Inputs x[n][16], targets t[n][4] (host, row-major). */
#define SPH_MLP_PARAMS 5508
typedef struct SphMlp SphMlp;
/* Weights and biases uniform in +-1/sqrt(fan_in) from `seed`. */
int sph_mlp_create(int device, uint64_t seed, SphMlp **out);
void sph_mlp_destroy(SphMlp *m);
int sph_mlp_set_params(SphMlp *m, const float *params); /* also resets Adam */
int sph_mlp_get_params(SphMlp *m, float *params);
int sph_mlp_forward(SphMlp *m, const float *x, size_t n, float *y);
/* Mean squared error over n x 4 outputs and its gradient (no update). */
int sph_mlp_loss_grad(SphMlp *m, const float *x, const float *t, size_t n, float *loss, float *grad);
/* Adam (beta 0.9 / 0.999, eps 1e-8) on shuffled mini-batches of `batch`;
 * epoch_loss (may be NULL) gets the mean training loss of each epoch. */
int sph_mlp_train(SphMlp *m, const float *x, const float *t, size_t n, int batch, int epochs, float lr,
                  uint64_t shuffle_seed, float *epoch_loss);

/* ---- closure in the WCSPH step ------------------------------------------
 * The closure acts on fluid particles within 2h of the geometry SDF (the
 * merged walls and obstacles; SDF wall mode uses its own SDF). */
/* Geometry SDF of the closure features: one simulation, or one per instance. */
int sph_set_feature_sdf(SphHandle *h, const SphSdfView *sdf);
int sph_batch_set_feature_sdfs(SphHandle *h, const SphSdfView *sdfs);
/* mode 0: off (the plain step). 1: the density pass records the features of
 * near-geometry particles (sph_closure_samples) without changing the step.
 * 2: also evaluates the network (`params`, SPH_MLP_PARAMS floats) on the
 * tensor cores after the density pass: density += y0 rho0 SPH_CLOSURE_DRHO_UNIT with the
 * EOS re-evaluated, acceleration += (y1, y2, y3) |g| in the force kernel,
 * y0 clamped to +-SPH_CLOSURE_MAX_DRHO and y1..3 to +-SPH_CLOSURE_MAX_ACC_G.
 * Features (d = SDF distance, n = SDF gradient):
 *   0 d/h, 1-3 n, 4 1 - Shepard kernel sum, 5 listed neighbours / 73,
 *   6 |v|/c, 7 dt c/h, 8 h * Laplacian of the SDF (clamped to +-4),
 *   9 wall-table kernel mass at d (SDF mode; else boundary density / rho0),
 *   10 n.g/|g|, 11 (d/h)^2, 12 f8 f0, 13 f10 f0,
 *   14 boundary particles in support / 30, 15 1. */
#define SPH_CLOSURE_DRHO_UNIT 1e-4f /* y0 in units of 0.01 % of rho0 */
#define SPH_CLOSURE_MAX_DRHO 30.0f   /* 0.3 % of rho0 */
#define SPH_CLOSURE_MAX_ACC_G 2.5f
int sph_set_closure(SphHandle *h, int mode, const float *params);
/* Samples of the last density pass: original particle ids, 16 features each
 * (row-major), density before correction; *count gets the total. */
int sph_closure_samples(SphHandle *h, size_t cap, uint32_t *ids, float *features, float *rho, size_t *count);
/* Shepard interpolation of the current state at points pts[n][3]:
 * out[n][7] = (rho, p, ax, ay, az, weight sum, neighbour count). */
int sph_interpolate(SphHandle *h, const float *pts, size_t n, float *out);

/* ---- force extraction ------------------------------------------------- */
/* Register the geometry SDF whose surface force sph_surface_forces returns
 * (the obstacle's SDF, as orchestrator/src/force.rs uses it): selects the
 * nodes with -2h <= d <= 0 and a nonzero gradient once, on the host. */
int sph_set_geometry_sdf(SphHandle *h, const SphSdfView *sdf);
/* compute_surface_forces(particles(), sdf, h) on the current state. */
int sph_surface_forces(SphHandle *h, SphSurfaceForce *out);
/* Fluid reaction on boundary particles [first, first + count) from the last
 * force computation (boundary-particle mode). */
int sph_body_force(SphHandle *h, uint32_t first, uint32_t count, SphBodyForce *out);

/* ---- grid diagnostics (the bit-exact grid/sort checks) ---------------- */
int sph_grid_info(SphHandle *h, SphGridInfo *out);
/* Grid of the last force computation. Per particle, in original order:
 * linear cell hash (neighbor.rs:75-77) and 30-bit Morton key of (cx,cy,cz).
 * Per linear cell: count and storage start. Per storage slot: original id.
 * Any pointer may be NULL. */
int sph_read_grid(SphHandle *h, uint32_t *cell_linear, uint32_t *morton_key,
                  uint32_t *cell_count, uint32_t *cell_start, uint32_t *slot_id);
/* Neighbour list of particle `id` (original index) in the reference visit
 * order (neighbor.rs:129-182) on the current grid; `*count` gets the full
 * length, at most `cap` ids are written. */
int sph_neighbors(SphHandle *h, uint32_t id, uint32_t *out, size_t cap, size_t *count);

/* ---- neighbour grid without device allocation ------------------------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc:
 * a host engine that owns all device memory through its own pool or budget
 * and lets no library allocate, or a caller whose other streams must not be
 * stalled by the device synchronization that cudaMalloc/cudaFree can cause.
 *
 * Builds NeighborGrid::update (kernel/src/neighbor.rs:82-122) on the device
 * from caller-owned device arrays: d_cell_index[n] (linear cell hash per
 * particle), d_cell_offsets[C] and d_cell_counts[C] (exclusive scan and
 * count per linear cell, C = product of the grid dims of NeighborGrid::new
 * for domain_min/max and cell_size, which must not exceed cells_capacity),
 * d_sorted[n] (particle indices grouped by cell, ascending within a cell).
 * domain_min/max are host arrays; `stream` is a cudaStream_t (NULL = legacy
 * default stream). The call returns after the stream has finished it.
 *
 * It allocates nothing: its scratch is a static device array of
 * SPH_NOALLOC_MAX_CELLS cursors plus tile sums (2 MiB + 1 KiB) that every
 * GPU which loads this library holds until the process exits. Grids with
 * more than SPH_NOALLOC_MAX_CELLS cells, or a cell holding more than 1024
 * particles, return SPH_ERR_CAPACITY. The first call on a device looks up
 * the array's device address (with that device current); make that first
 * call before any stream capture. `stream` must belong to the current
 * device; since the call waits on the host for the stream, a stream of
 * another device or a stream that is capturing is rejected with
 * SPH_ERR_INVALID_ARG before anything is enqueued. All calls share the one
 * array, so calls that overlap on the GPU (different streams or host
 * threads, same device) race and must be serialized by the caller. */
#define SPH_NOALLOC_MAX_CELLS (1u << 19)
int sph_grid_sort_noalloc(const float *d_x, const float *d_y, const float *d_z, uint32_t n,
                          const float domain_min[3], const float domain_max[3], float cell_size,
                          uint32_t *d_cell_index, uint32_t *d_cell_offsets, uint32_t *d_cell_counts,
                          uint32_t *d_sorted, size_t cells_capacity, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SPH_CUDA_H */
