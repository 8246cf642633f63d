//! Raw declarations of include/sph_cuda.h (SPH_ABI_VERSION 1).
//!
//! Every struct is `#[repr(C)]` with the header's field order and types, and
//! every function has the header's parameters; tests/test_rust_binding.py
//! checks both against a C compiler's view of the header.
#![allow(non_camel_case_types, dead_code)]
use std::os::raw::{c_char, c_int, c_void};

pub const SPH_ABI_VERSION: c_int = 1;

/// Opaque simulation handle (one simulation, or a batch of them).
#[repr(C)]
pub struct SphHandle {
    _p: [u8; 0],
}
/// Opaque closure network (16 -> 64 -> 64 -> 4, BF16 tensor-core kernels).
#[repr(C)]
pub struct SphMlp {
    _p: [u8; 0],
}

// SphStatus
pub const SPH_OK: c_int = 0;
pub const SPH_ERR_INVALID_ARG: c_int = 1;
pub const SPH_ERR_OOM: c_int = 2;
pub const SPH_ERR_CUDA: c_int = 3;
pub const SPH_ERR_NONFINITE: c_int = 4;
pub const SPH_ERR_TIMEOUT: c_int = 5;
pub const SPH_ERR_CAPACITY: c_int = 6;
pub const SPH_ERR_NO_DEVICE: c_int = 7;
pub const SPH_ERR_NO_CHECKPOINT: c_int = 8;
// SphBoundaryMode
pub const SPH_BOUNDARY_PARTICLES: i32 = 0;
pub const SPH_BOUNDARY_SDF: i32 = 1;
// SphCellOrder
pub const SPH_CELL_ORDER_MORTON: i32 = 0;
pub const SPH_CELL_ORDER_LINEAR: i32 = 1;
pub const SPH_CELL_ORDER_ROWS: i32 = 2;
// SphFlags
pub const SPH_FLAG_DELTA_SPH: u32 = 1 << 0;
pub const SPH_FLAG_XSPH: u32 = 1 << 1;
pub const SPH_FLAG_REPULSION: u32 = 1 << 2;
pub const SPH_FLAG_DOMAIN_CLAMP: u32 = 1 << 3;
pub const SPH_FLAGS_REFERENCE: u32 = 0xF;
// SphDomainSpec::fluid_type
pub const SPH_FLUID_WATER: c_int = 0;
pub const SPH_FLUID_AIR: c_int = 1;
pub const SPH_FLUID_MIXED: c_int = 2;
pub const SPH_MLP_PARAMS: usize = 5508;
pub const SPH_NOALLOC_MAX_CELLS: u32 = 1 << 19;

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct SphParams {
    pub h: f32,
    pub gravity: [f32; 3],
    pub speed_of_sound: f32,
    pub cfl_number: f32,
    pub viscosity: f32,
    pub domain_min: [f32; 3],
    pub domain_max: [f32; 3],
    pub alpha: f32,
    pub beta: f32,
    pub boundary_mode: i32,
    pub cell_order: i32,
    pub flags: u32,
    pub device: i32,
    pub sdf_wall_coef: f32,
}

#[repr(C)]
pub struct SphParticlesView {
    pub n: usize,
    pub x: *const f32,
    pub y: *const f32,
    pub z: *const f32,
    pub vx: *const f32,
    pub vy: *const f32,
    pub vz: *const f32,
    pub ax: *const f32,
    pub ay: *const f32,
    pub az: *const f32,
    pub density: *const f32,
    pub pressure: *const f32,
    pub mass: *const f32,
    pub temperature: *const f32,
    pub fluid_type: *const u8,
}

#[repr(C)]
pub struct SphParticlesMut {
    pub n: usize,
    pub x: *mut f32,
    pub y: *mut f32,
    pub z: *mut f32,
    pub vx: *mut f32,
    pub vy: *mut f32,
    pub vz: *mut f32,
    pub ax: *mut f32,
    pub ay: *mut f32,
    pub az: *mut f32,
    pub density: *mut f32,
    pub pressure: *mut f32,
    pub mass: *mut f32,
    pub temperature: *mut f32,
    pub fluid_type: *mut u8,
}

#[repr(C)]
pub struct SphBoundaryView {
    pub n: usize,
    pub x: *const f32,
    pub y: *const f32,
    pub z: *const f32,
    pub mass: *const f32,
    pub nx: *const f32,
    pub ny: *const f32,
    pub nz: *const f32,
}

#[repr(C)]
pub struct SphSdfView {
    pub origin: [f32; 3],
    pub cell_size: f32,
    pub dims: [u32; 3],
    pub distances: *const f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphErrorMetrics {
    pub max_density_variation: f32,
    pub energy_conservation: f32,
    pub mass_conservation: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphStepProfile {
    pub xsph_drift_us: f32,
    pub sort_us: f32,
    pub density_us: f32,
    pub boundary_pressure_us: f32,
    pub forces_us: f32,
    pub total_us: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphSurfaceForce {
    pub force: [f64; 3],
    pub moment: [f64; 3],
    pub force_f32: [f32; 3],
    pub moment_f32: [f32; 3],
    pub nodes: u32,
    pub active_nodes: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphBodyForce {
    pub pressure_force: [f64; 3],
    pub pressure_moment: [f64; 3],
    pub repulsion_force: [f64; 3],
    pub repulsion_moment: [f64; 3],
    pub viscous_force: [f64; 3],
    pub viscous_moment: [f64; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphLaunch {
    pub xsph_threads: i32,
    pub density_threads: i32,
    pub forces_threads: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphGridInfo {
    pub dims: [u32; 3],
    pub total_cells: u32,
    pub cell_size: f32,
    pub grid_min: [f32; 3],
    pub boundary_candidates: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SphRunStats {
    pub sim_time: f64,
    pub steps: u64,
    pub accepted: u64,
    pub rejected: u64,
    pub last_dt: f32,
    pub cooldown: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct SphDomainSpec {
    pub particle_spacing: f32,
    pub domain_min: [f32; 3],
    pub domain_max: [f32; 3],
    pub fluid_type: c_int,
    pub initial_temperature: f32,
    pub wall_faces: u32,
}

#[repr(C)]
pub struct SphBoundaryMut {
    pub n: usize,
    pub x: *mut f32,
    pub y: *mut f32,
    pub z: *mut f32,
    pub mass: *mut f32,
    pub nx: *mut f32,
    pub ny: *mut f32,
    pub nz: *mut f32,
}

extern "C" {
    pub fn sph_params_default(p: *mut SphParams);
    pub fn sph_create(params: *const SphParams, particles: *const SphParticlesView,
                      boundary: *const SphBoundaryView, sdf: *const SphSdfView, out: *mut *mut SphHandle) -> c_int;
    pub fn sph_destroy(h: *mut SphHandle);
    pub fn sph_step(h: *mut SphHandle, dt: f32) -> c_int;
    pub fn sph_step_auto(h: *mut SphHandle, nsteps: c_int, dt_out: *mut f32) -> c_int;
    pub fn sph_compute_timestep(h: *mut SphHandle, dt_out: *mut f32) -> c_int;
    pub fn sph_step_profiled(h: *mut SphHandle, dt: f32, prof: *mut SphStepProfile) -> c_int;
    pub fn sph_read_particles(h: *mut SphHandle, out: *mut SphParticlesMut) -> c_int;
    pub fn sph_read_boundary_pressure(h: *mut SphHandle, out: *mut f32, n: usize) -> c_int;
    pub fn sph_error_metrics(h: *mut SphHandle, out: *mut SphErrorMetrics) -> c_int;
    pub fn sph_particle_count(h: *const SphHandle) -> usize;
    pub fn sph_save_checkpoint(h: *mut SphHandle) -> c_int;
    pub fn sph_restore_checkpoint(h: *mut SphHandle) -> c_int;
    pub fn sph_pack_frame(h: *mut SphHandle, subsample_count: u32, frame_number: u64, sim_time: f64,
                          out: *mut u8, cap: usize, bytes: *mut usize) -> c_int;
    pub fn sph_run_optimistic(h: *mut SphHandle, nsteps: c_int, alpha: f32, density_limit: f32,
                              cooldown_steps: u32, stats: *mut SphRunStats) -> c_int;
    pub fn sph_setup_domain(device: c_int, spec: *const SphDomainSpec, sdf: *const SphSdfView,
                            fluid: *mut SphParticlesMut, boundary: *mut SphBoundaryMut, n_fluid: *mut usize,
                            n_boundary: *mut usize) -> c_int;
    pub fn sph_scale_velocities(h: *mut SphHandle, factor: f32) -> c_int;
    pub fn sph_synchronize(h: *mut SphHandle) -> c_int;
    pub fn sph_health(h: *mut SphHandle, nonfinite_out: *mut u64) -> c_int;
    pub fn sph_last_error(h: *const SphHandle) -> *const c_char;
    pub fn sph_stream(h: *mut SphHandle) -> *mut c_void;
    pub fn sph_launch_count(h: *const SphHandle) -> u64;
    pub fn sph_batch_create(ninst: c_int, params: *const SphParams, particles: *const SphParticlesView,
                            boundaries: *const SphBoundaryView, out: *mut *mut SphHandle) -> c_int;
    pub fn sph_batch_create_sdf(ninst: c_int, params: *const SphParams, particles: *const SphParticlesView,
                                sdfs: *const SphSdfView, out: *mut *mut SphHandle) -> c_int;
    pub fn sph_batch_info(h: *const SphHandle, ninst: *mut c_int, first: *mut usize, count: *mut usize) -> c_int;
    pub fn sph_batch_step(h: *mut SphHandle, dts: *const f32) -> c_int;
    pub fn sph_batch_timesteps(h: *mut SphHandle, dt_out: *mut f32) -> c_int;
    pub fn sph_set_launch(h: *mut SphHandle, launch: *const SphLaunch) -> c_int;
    pub fn sph_get_launch(h: *const SphHandle, launch: *mut SphLaunch) -> c_int;
    pub fn sph_autotune(h: *mut SphHandle, trial_steps: c_int, best: *mut SphLaunch) -> c_int;
    pub fn sph_mlp_create(device: c_int, seed: u64, out: *mut *mut SphMlp) -> c_int;
    pub fn sph_mlp_destroy(m: *mut SphMlp);
    pub fn sph_mlp_set_params(m: *mut SphMlp, params: *const f32) -> c_int;
    pub fn sph_mlp_get_params(m: *mut SphMlp, params: *mut f32) -> c_int;
    pub fn sph_mlp_forward(m: *mut SphMlp, x: *const f32, n: usize, y: *mut f32) -> c_int;
    pub fn sph_mlp_loss_grad(m: *mut SphMlp, x: *const f32, t: *const f32, n: usize, loss: *mut f32,
                             grad: *mut f32) -> c_int;
    pub fn sph_mlp_train(m: *mut SphMlp, x: *const f32, t: *const f32, n: usize, batch: c_int, epochs: c_int,
                         lr: f32, shuffle_seed: u64, epoch_loss: *mut f32) -> c_int;
    pub fn sph_set_feature_sdf(h: *mut SphHandle, sdf: *const SphSdfView) -> c_int;
    pub fn sph_batch_set_feature_sdfs(h: *mut SphHandle, sdfs: *const SphSdfView) -> c_int;
    pub fn sph_set_closure(h: *mut SphHandle, mode: c_int, params: *const f32) -> c_int;
    pub fn sph_closure_samples(h: *mut SphHandle, cap: usize, ids: *mut u32, features: *mut f32, rho: *mut f32,
                               count: *mut usize) -> c_int;
    pub fn sph_interpolate(h: *mut SphHandle, pts: *const f32, n: usize, out: *mut f32) -> c_int;
    pub fn sph_set_geometry_sdf(h: *mut SphHandle, sdf: *const SphSdfView) -> c_int;
    pub fn sph_surface_forces(h: *mut SphHandle, out: *mut SphSurfaceForce) -> c_int;
    pub fn sph_body_force(h: *mut SphHandle, first: u32, count: u32, out: *mut SphBodyForce) -> c_int;
    pub fn sph_grid_info(h: *mut SphHandle, out: *mut SphGridInfo) -> c_int;
    pub fn sph_read_grid(h: *mut SphHandle, cell_linear: *mut u32, morton_key: *mut u32, cell_count: *mut u32,
                         cell_start: *mut u32, slot_id: *mut u32) -> c_int;
    pub fn sph_neighbors(h: *mut SphHandle, id: u32, out: *mut u32, cap: usize, count: *mut usize) -> c_int;
    pub fn sph_grid_sort_noalloc(d_x: *const f32, d_y: *const f32, d_z: *const f32, n: u32,
                                 domain_min: *const f32, domain_max: *const f32, cell_size: f32,
                                 d_cell_index: *mut u32, d_cell_offsets: *mut u32, d_cell_counts: *mut u32,
                                 d_sorted: *mut u32, cells_capacity: usize, stream: *mut c_void) -> c_int;
}
