//! The `cuda` backend of the kernel crate: `CudaKernel` implements
//! `kernel::SimulationKernel` (backend/crates/kernel/src/lib.rs:58-78) over
//! one handle of libsph_cuda.so, so the orchestrator's runner, the server and
//! force extraction call it unchanged. There is no CPU fallback inside this
//! backend: a failed `sph_create` is an error of the constructor, like
//! `GpuKernel::new`'s `GpuInitError` (kernel/src/gpu/mod.rs:158-168).
//!
//! Wiring: place this crate at backend/crates/kernel-cuda,
//! add `BackendType::Cuda` (orchestrator/src/config.rs:9-22) and its arm in
//! `create_kernel` (orchestrator/src/lib.rs:142-266).
pub mod ffi;

use ffi::*;
use kernel::{BoundaryParticles, ErrorMetrics, FluidType, ParticleArrays, SimulationKernel};
use std::cell::{Cell, RefCell};
use std::ffi::CStr;

/// `sph_create` returned a non-zero status (one of the `SPH_ERR_*` codes).
#[derive(Debug)]
pub struct CudaInitError {
    pub status: i32,
    pub message: String,
}

impl std::fmt::Display for CudaInitError {
    fn fmt(&self, f: &mut std::fmt::Formatter) -> std::fmt::Result {
        write!(f, "sph_create failed with status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for CudaInitError {}

/// Construction options beyond `CpuKernel::new`'s arguments.
#[derive(Clone, Copy, Debug)]
pub struct CudaOptions {
    /// Monaghan alpha and beta (the reference hardcodes 1 and 2, sph.rs:440-441).
    pub alpha: f32,
    pub beta: f32,
    /// `SPH_FLAG_*` stage switches; `SPH_FLAGS_REFERENCE` keeps every stage.
    pub flags: u32,
    /// CUDA device ordinal.
    pub device: i32,
}

impl Default for CudaOptions {
    fn default() -> Self {
        Self { alpha: 1.0, beta: 2.0, flags: SPH_FLAGS_REFERENCE, device: 0 }
    }
}

pub struct CudaKernel {
    h: *mut SphHandle,
    host: RefCell<ParticleArrays>,
    dirty: Cell<bool>,
}

// A handle may move between threads (every entry point makes its device
// current and uses the handle's own stream); calls must not overlap.
unsafe impl Send for CudaKernel {}

fn last_error(h: *const SphHandle) -> String {
    let p = unsafe { sph_last_error(h) };
    if p.is_null() {
        return String::new();
    }
    unsafe { CStr::from_ptr(p) }.to_string_lossy().into_owned()
}

impl CudaKernel {
    /// Same arguments as `CpuKernel::new` (kernel/src/lib.rs:138-148).
    #[allow(clippy::too_many_arguments)]
    pub fn new(particles: ParticleArrays, boundary: BoundaryParticles, h: f32, gravity: [f32; 3],
               speed_of_sound: f32, cfl_number: f32, viscosity: f32, domain_min: [f32; 3],
               domain_max: [f32; 3]) -> Result<Self, CudaInitError> {
        Self::with_options(particles, boundary, h, gravity, speed_of_sound, cfl_number, viscosity, domain_min,
                           domain_max, CudaOptions::default())
    }

    #[allow(clippy::too_many_arguments)]
    pub fn with_options(particles: ParticleArrays, boundary: BoundaryParticles, h: f32, gravity: [f32; 3],
                        speed_of_sound: f32, cfl_number: f32, viscosity: f32, domain_min: [f32; 3],
                        domain_max: [f32; 3], opt: CudaOptions) -> Result<Self, CudaInitError> {
        let mut p = unsafe {
            let mut p = std::mem::zeroed::<SphParams>();
            sph_params_default(&mut p);
            p
        };
        p.h = h;
        p.gravity = gravity;
        p.speed_of_sound = speed_of_sound;
        p.cfl_number = cfl_number;
        p.viscosity = viscosity;
        p.domain_min = domain_min;
        p.domain_max = domain_max;
        p.alpha = opt.alpha;
        p.beta = opt.beta;
        p.flags = opt.flags;
        p.device = opt.device;
        let ft: Vec<u8> = particles.fluid_type.iter().map(|t| *t as u8).collect();
        let pv = SphParticlesView {
            n: particles.len(),
            x: particles.x.as_ptr(),
            y: particles.y.as_ptr(),
            z: particles.z.as_ptr(),
            vx: particles.vx.as_ptr(),
            vy: particles.vy.as_ptr(),
            vz: particles.vz.as_ptr(),
            ax: particles.ax.as_ptr(),
            ay: particles.ay.as_ptr(),
            az: particles.az.as_ptr(),
            density: particles.density.as_ptr(),
            pressure: particles.pressure.as_ptr(),
            mass: particles.mass.as_ptr(),
            temperature: particles.temperature.as_ptr(),
            fluid_type: ft.as_ptr(),
        };
        let bv = SphBoundaryView {
            n: boundary.x.len(),
            x: boundary.x.as_ptr(),
            y: boundary.y.as_ptr(),
            z: boundary.z.as_ptr(),
            mass: boundary.mass.as_ptr(),
            nx: boundary.nx.as_ptr(),
            ny: boundary.ny.as_ptr(),
            nz: boundary.nz.as_ptr(),
        };
        let mut h = std::ptr::null_mut();
        let st = unsafe { sph_create(&p, &pv, &bv, std::ptr::null(), &mut h) };
        if st != SPH_OK {
            return Err(CudaInitError { status: st, message: String::new() });
        }
        Ok(Self { h, host: RefCell::new(particles), dirty: Cell::new(false) })
    }

    fn check(&self, st: i32, what: &str) {
        assert_eq!(st, SPH_OK, "{what} failed with status {st}: {}", last_error(self.h));
    }

    /// `sph::compute_timestep(particles(), h, c, cfl)` on the device, without
    /// reading the state back (kernel/src/sph.rs:591-628).
    pub fn suggest_dt(&self) -> f32 {
        let mut dt = 0.0f32;
        self.check(unsafe { sph_compute_timestep(self.h, &mut dt) }, "sph_compute_timestep");
        dt
    }

    /// `n` steps with the CFL dt computed on the device each step; returns
    /// the dt of the last one. No host round trip between steps.
    pub fn step_auto(&mut self, n: i32) -> f32 {
        let mut dt = 0.0f32;
        self.check(unsafe { sph_step_auto(self.h, n, &mut dt) }, "sph_step_auto");
        self.dirty.set(true);
        dt
    }

    /// Per-stage device times of one step (the `GpuStepProfile` counterpart).
    pub fn step_profiled(&mut self, dt: f32) -> SphStepProfile {
        let mut prof = SphStepProfile::default();
        self.check(unsafe { sph_step_profiled(self.h, dt, &mut prof) }, "sph_step_profiled");
        self.dirty.set(true);
        prof
    }

    /// The orchestrator's optimistic time stepping (runner.rs:189-240) on the
    /// device: `n` steps, one graph launch each; counters accumulate.
    pub fn run_optimistic(&mut self, n: i32, alpha: f32, density_limit: f32, cooldown: u32) -> SphRunStats {
        let mut s = SphRunStats::default();
        self.check(unsafe { sph_run_optimistic(self.h, n, alpha, density_limit, cooldown, &mut s) },
                   "sph_run_optimistic");
        self.dirty.set(true);
        s
    }

    /// force.rs:39-129 on the device for `sdf` (set once per geometry).
    pub fn surface_forces(&mut self, sdf: &SphSdfView) -> SphSurfaceForce {
        let mut out = SphSurfaceForce::default();
        self.check(unsafe { sph_set_geometry_sdf(self.h, sdf) }, "sph_set_geometry_sdf");
        self.check(unsafe { sph_surface_forces(self.h, &mut out) }, "sph_surface_forces");
        out
    }

    /// The viewer's Frame message (server ws.rs:233-290), packed on the device.
    pub fn pack_frame(&self, subsample_count: u32, frame_number: u64, sim_time: f64) -> Vec<u8> {
        let mut len = 0usize;
        self.check(unsafe {
            sph_pack_frame(self.h, subsample_count, frame_number, sim_time, std::ptr::null_mut(), 0, &mut len)
        }, "sph_pack_frame");
        let mut buf = vec![0u8; len];
        self.check(unsafe {
            sph_pack_frame(self.h, subsample_count, frame_number, sim_time, buf.as_mut_ptr(), len, &mut len)
        }, "sph_pack_frame");
        buf.truncate(len);
        buf
    }
}

impl SimulationKernel for CudaKernel {
    fn step(&mut self, dt: f32) {
        self.check(unsafe { sph_step(self.h, dt) }, "sph_step");
        self.dirty.set(true);
    }

    fn particles(&self) -> &ParticleArrays {
        if self.dirty.get() {
            // lazy readback, as GpuKernel does (gpu/mod.rs:979-988)
            let mut p = self.host.borrow_mut();
            let mut ft = vec![0u8; p.len()];
            let mut out = SphParticlesMut {
                n: p.len(),
                x: p.x.as_mut_ptr(),
                y: p.y.as_mut_ptr(),
                z: p.z.as_mut_ptr(),
                vx: p.vx.as_mut_ptr(),
                vy: p.vy.as_mut_ptr(),
                vz: p.vz.as_mut_ptr(),
                ax: p.ax.as_mut_ptr(),
                ay: p.ay.as_mut_ptr(),
                az: p.az.as_mut_ptr(),
                density: p.density.as_mut_ptr(),
                pressure: p.pressure.as_mut_ptr(),
                mass: p.mass.as_mut_ptr(),
                temperature: p.temperature.as_mut_ptr(),
                fluid_type: ft.as_mut_ptr(),
            };
            self.check(unsafe { sph_read_particles(self.h, &mut out) }, "sph_read_particles");
            for (t, v) in p.fluid_type.iter_mut().zip(ft) {
                *t = if v == 0 { FluidType::Water } else { FluidType::Air };
            }
            self.dirty.set(false);
        }
        // SAFETY: the only mutable borrow is the one above, which has ended.
        unsafe { &*self.host.as_ptr() }
    }

    fn error_metrics(&self) -> ErrorMetrics {
        let mut m = SphErrorMetrics::default();
        self.check(unsafe { sph_error_metrics(self.h, &mut m) }, "sph_error_metrics");
        ErrorMetrics {
            max_density_variation: m.max_density_variation,
            energy_conservation: m.energy_conservation,
            mass_conservation: m.mass_conservation,
        }
    }

    fn particle_count(&self) -> usize {
        unsafe { sph_particle_count(self.h) }
    }

    fn save_checkpoint(&mut self) -> bool {
        unsafe { sph_save_checkpoint(self.h) == SPH_OK }
    }

    fn restore_checkpoint(&mut self) -> bool {
        let ok = unsafe { sph_restore_checkpoint(self.h) == SPH_OK };
        if ok {
            self.dirty.set(true);
        }
        ok
    }
}

impl Drop for CudaKernel {
    fn drop(&mut self) {
        unsafe { sph_destroy(self.h) }
    }
}
