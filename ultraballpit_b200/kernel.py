"""Host-side mirror of the reference ``SimulationKernel`` trait over the C ABI.

``CudaKernel`` is the ``cuda`` backend of ``kernel/src/lib.rs:58-78``: the same
constructor arguments as ``CpuKernel::new`` (``lib.rs:138-148``) and the same
methods (``step``, ``particles``, ``error_metrics``, ``particle_count``,
``save_checkpoint``, ``restore_checkpoint``). Every call goes through
``libsph_cuda.so`` (include/sph_cuda.h); there is no CPU fallback: a missing
library or device raises ``SphError``.

Like ``GpuKernel`` (``gpu/mod.rs:979-988``), ``particles()`` reads back lazily:
the host copy is refreshed only after the state changed.
"""
from __future__ import annotations

import ctypes as C
import os
from abc import ABC, abstractmethod

import numpy as np

from .particles import (BOUNDARY_FIELDS, PARTICLE_FIELDS, BoundaryParticles, ErrorMetrics,
                        GridSDF, ParticleArrays)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libsph_cuda.so")

SPH_OK = 0
STATUS_NAMES = {0: "SPH_OK", 1: "SPH_ERR_INVALID_ARG", 2: "SPH_ERR_OOM", 3: "SPH_ERR_CUDA",
                4: "SPH_ERR_NONFINITE", 5: "SPH_ERR_TIMEOUT", 6: "SPH_ERR_CAPACITY",
                7: "SPH_ERR_NO_DEVICE", 8: "SPH_ERR_NO_CHECKPOINT"}
BOUNDARY_PARTICLES, BOUNDARY_SDF = 0, 1
CELL_ORDER_MORTON, CELL_ORDER_LINEAR, CELL_ORDER_ROWS = 0, 1, 2
FLAG_DELTA_SPH, FLAG_XSPH, FLAG_REPULSION, FLAG_DOMAIN_CLAMP = 1, 2, 4, 8
FLAGS_REFERENCE = 0xF

# every entry point declared in include/sph_cuda.h
EXPORTS = (
    "sph_params_default", "sph_create", "sph_destroy", "sph_step", "sph_step_auto",
    "sph_compute_timestep", "sph_step_profiled", "sph_read_particles",
    "sph_read_boundary_pressure", "sph_error_metrics", "sph_particle_count",
    "sph_save_checkpoint", "sph_restore_checkpoint", "sph_scale_velocities", "sph_synchronize", "sph_health",
    "sph_last_error", "sph_stream", "sph_launch_count", "sph_grid_info", "sph_read_grid",
    "sph_neighbors", "sph_grid_sort_noalloc", "sph_set_geometry_sdf", "sph_surface_forces",
    "sph_body_force", "sph_batch_create", "sph_batch_info", "sph_batch_timesteps", "sph_set_launch",
    "sph_get_launch", "sph_autotune", "sph_mlp_create", "sph_mlp_destroy", "sph_mlp_set_params",
    "sph_mlp_get_params", "sph_mlp_forward", "sph_mlp_loss_grad", "sph_mlp_train",
    "sph_set_feature_sdf", "sph_batch_set_feature_sdfs", "sph_set_closure", "sph_closure_samples",
    "sph_interpolate", "sph_batch_create_sdf", "sph_batch_step", "sph_pack_frame", "sph_run_optimistic", "sph_setup_domain",
)


class SphError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


class SphParams(C.Structure):
    _fields_ = [("h", C.c_float), ("gravity", C.c_float * 3), ("speed_of_sound", C.c_float),
                ("cfl_number", C.c_float), ("viscosity", C.c_float),
                ("domain_min", C.c_float * 3), ("domain_max", C.c_float * 3),
                ("alpha", C.c_float), ("beta", C.c_float), ("boundary_mode", C.c_int32),
                ("cell_order", C.c_int32), ("flags", C.c_uint32), ("device", C.c_int32),
                ("sdf_wall_coef", C.c_float)]


_FP = C.POINTER(C.c_float)
_U8P = C.POINTER(C.c_uint8)
_U32P = C.POINTER(C.c_uint32)


class SphParticlesView(C.Structure):
    _fields_ = [("n", C.c_size_t)] + [(f, _FP) for f in PARTICLE_FIELDS] + [("fluid_type", _U8P)]


class SphParticlesMut(SphParticlesView):
    pass


class SphBoundaryView(C.Structure):
    _fields_ = [("n", C.c_size_t)] + [(f, _FP) for f in BOUNDARY_FIELDS]


class SphSdfView(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("cell_size", C.c_float), ("dims", C.c_uint32 * 3),
                ("distances", _FP)]


class SphDomainSpec(C.Structure):
    _fields_ = [("particle_spacing", C.c_float), ("domain_min", C.c_float * 3), ("domain_max", C.c_float * 3),
                ("fluid_type", C.c_int), ("initial_temperature", C.c_float), ("wall_faces", C.c_uint32)]


class SphBoundaryMut(C.Structure):
    _fields_ = [("n", C.c_size_t)] + [(f, _FP) for f in BOUNDARY_FIELDS]


class SphRunStats(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("steps", C.c_uint64), ("accepted", C.c_uint64),
                ("rejected", C.c_uint64), ("last_dt", C.c_float), ("cooldown", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: (float if k in ("sim_time", "last_dt") else int)(getattr(self, k)) for k, _ in self._fields_}


class SphErrorMetrics(C.Structure):
    _fields_ = [("max_density_variation", C.c_float), ("energy_conservation", C.c_float),
                ("mass_conservation", C.c_float)]


class SphStepProfile(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("xsph_drift_us", "sort_us", "density_us",
                                         "boundary_pressure_us", "forces_us", "total_us")]

    def as_dict(self) -> dict:
        return {k: float(getattr(self, k)) for k, _ in self._fields_}


class SphSurfaceForce(C.Structure):
    _fields_ = [("force", C.c_double * 3), ("moment", C.c_double * 3), ("force_f32", C.c_float * 3),
                ("moment_f32", C.c_float * 3), ("nodes", C.c_uint32), ("active_nodes", C.c_uint32)]


class SphBodyForce(C.Structure):
    _fields_ = [(k, C.c_double * 3) for k in ("pressure_force", "pressure_moment", "repulsion_force",
                                              "repulsion_moment", "viscous_force", "viscous_moment")]


class SphLaunch(C.Structure):
    _fields_ = [("xsph_threads", C.c_int32), ("density_threads", C.c_int32), ("forces_threads", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class SphGridInfo(C.Structure):
    _fields_ = [("dims", C.c_uint32 * 3), ("total_cells", C.c_uint32), ("cell_size", C.c_float),
                ("grid_min", C.c_float * 3), ("boundary_candidates", C.c_uint64)]


_lib = None


def load_library(path: str | None = None):
    """Load libsph_cuda.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise SphError(7, f"{p} is missing: run python -m ultraballpit_b200.build")
    L = C.CDLL(p)
    vp, H = C.c_void_p, C.c_void_p
    L.sph_params_default.argtypes = [C.POINTER(SphParams)]
    L.sph_params_default.restype = None
    L.sph_create.argtypes = [C.POINTER(SphParams), C.POINTER(SphParticlesView),
                             C.POINTER(SphBoundaryView), C.POINTER(SphSdfView), C.POINTER(vp)]
    L.sph_destroy.argtypes = [H]
    L.sph_destroy.restype = None
    L.sph_step.argtypes = [H, C.c_float]
    L.sph_step_auto.argtypes = [H, C.c_int, _FP]
    L.sph_compute_timestep.argtypes = [H, _FP]
    L.sph_step_profiled.argtypes = [H, C.c_float, C.POINTER(SphStepProfile)]
    L.sph_read_particles.argtypes = [H, C.POINTER(SphParticlesMut)]
    L.sph_read_boundary_pressure.argtypes = [H, _FP, C.c_size_t]
    L.sph_error_metrics.argtypes = [H, C.POINTER(SphErrorMetrics)]
    L.sph_particle_count.argtypes = [H]
    L.sph_particle_count.restype = C.c_size_t
    L.sph_save_checkpoint.argtypes = [H]
    L.sph_restore_checkpoint.argtypes = [H]
    L.sph_pack_frame.argtypes = [H, C.c_uint32, C.c_uint64, C.c_double, C.POINTER(C.c_uint8), C.c_size_t,
                                 C.POINTER(C.c_size_t)]
    L.sph_pack_frame.restype = C.c_int
    L.sph_batch_step.argtypes = [H, _FP]
    L.sph_batch_step.restype = C.c_int
    L.sph_setup_domain.argtypes = [C.c_int, C.POINTER(SphDomainSpec), C.POINTER(SphSdfView),
                                   C.POINTER(SphParticlesMut), C.POINTER(SphBoundaryMut), C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_size_t)]
    L.sph_setup_domain.restype = C.c_int
    L.sph_run_optimistic.argtypes = [H, C.c_int, C.c_float, C.c_float, C.c_uint32, C.POINTER(SphRunStats)]
    L.sph_run_optimistic.restype = C.c_int
    L.sph_scale_velocities.argtypes = [H, C.c_float]
    L.sph_scale_velocities.restype = C.c_int
    L.sph_synchronize.argtypes = [H]
    L.sph_health.argtypes = [H, C.POINTER(C.c_uint64)]
    L.sph_last_error.argtypes = [H]
    L.sph_last_error.restype = C.c_char_p
    L.sph_stream.argtypes = [H]
    L.sph_stream.restype = vp
    L.sph_launch_count.argtypes = [H]
    L.sph_launch_count.restype = C.c_uint64
    L.sph_grid_info.argtypes = [H, C.POINTER(SphGridInfo)]
    L.sph_read_grid.argtypes = [H, _U32P, _U32P, _U32P, _U32P, _U32P]
    L.sph_neighbors.argtypes = [H, C.c_uint32, _U32P, C.c_size_t, C.POINTER(C.c_size_t)]
    L.sph_batch_create.argtypes = [C.c_int, C.POINTER(SphParams), C.POINTER(SphParticlesView),
                                   C.POINTER(SphBoundaryView), C.POINTER(vp)]
    L.sph_batch_create_sdf.argtypes = [C.c_int, C.POINTER(SphParams), C.POINTER(SphParticlesView),
                                       C.POINTER(SphSdfView), C.POINTER(vp)]
    L.sph_batch_create_sdf.restype = C.c_int
    L.sph_batch_info.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.sph_batch_timesteps.argtypes = [H, _FP]
    L.sph_set_launch.argtypes = [H, C.POINTER(SphLaunch)]
    L.sph_get_launch.argtypes = [H, C.POINTER(SphLaunch)]
    L.sph_autotune.argtypes = [H, C.c_int, C.POINTER(SphLaunch)]
    L.sph_set_feature_sdf.argtypes = [H, C.POINTER(SphSdfView)]
    L.sph_batch_set_feature_sdfs.argtypes = [H, C.POINTER(SphSdfView)]
    L.sph_set_closure.argtypes = [H, C.c_int, _FP]
    L.sph_closure_samples.argtypes = [H, C.c_size_t, _U32P, _FP, _FP, C.POINTER(C.c_size_t)]
    L.sph_interpolate.argtypes = [H, _FP, C.c_size_t, _FP]
    for f in ("sph_set_feature_sdf", "sph_batch_set_feature_sdfs", "sph_set_closure", "sph_closure_samples",
              "sph_interpolate"):
        getattr(L, f).restype = C.c_int
    L.sph_set_geometry_sdf.argtypes = [H, C.POINTER(SphSdfView)]
    L.sph_surface_forces.argtypes = [H, C.POINTER(SphSurfaceForce)]
    L.sph_body_force.argtypes = [H, C.c_uint32, C.c_uint32, C.POINTER(SphBodyForce)]
    for name in EXPORTS:
        fn = getattr(L, name)
        if getattr(fn, "restype", None) is C.c_int or name in (
                "sph_create", "sph_step", "sph_step_auto", "sph_compute_timestep", "sph_step_profiled",
                "sph_read_particles", "sph_read_boundary_pressure", "sph_error_metrics",
                "sph_save_checkpoint", "sph_restore_checkpoint", "sph_synchronize", "sph_health",
                "sph_grid_info", "sph_read_grid", "sph_neighbors", "sph_set_geometry_sdf",
                "sph_surface_forces", "sph_body_force", "sph_batch_create", "sph_batch_info",
                "sph_batch_timesteps", "sph_set_launch", "sph_get_launch", "sph_autotune"):
            fn.restype = C.c_int
    _lib = L
    return L


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _u32p(a):
    return None if a is None else a.ctypes.data_as(_U32P)


def default_params() -> SphParams:
    p = SphParams()
    load_library().sph_params_default(C.byref(p))
    return p


class SimulationKernel(ABC):
    """``kernel/src/lib.rs:58-78``."""

    @abstractmethod
    def step(self, dt: float) -> None: ...

    @abstractmethod
    def particles(self) -> ParticleArrays: ...

    @abstractmethod
    def error_metrics(self) -> ErrorMetrics: ...

    @abstractmethod
    def particle_count(self) -> int: ...

    def save_checkpoint(self) -> bool:
        return False

    def restore_checkpoint(self) -> bool:
        return False


def make_params(h, gravity, speed_of_sound, cfl_number, viscosity, domain_min, domain_max, *,
                alpha=1.0, beta=2.0, boundary_mode=BOUNDARY_PARTICLES, cell_order=CELL_ORDER_ROWS,
                flags=FLAGS_REFERENCE, device=0, sdf_wall_coef=0.981) -> SphParams:
    prm = default_params()
    prm.h = h
    prm.gravity = (C.c_float * 3)(*map(float, gravity))
    prm.speed_of_sound = speed_of_sound
    prm.cfl_number = cfl_number
    prm.viscosity = viscosity
    prm.domain_min = (C.c_float * 3)(*map(float, domain_min))
    prm.domain_max = (C.c_float * 3)(*map(float, domain_max))
    prm.alpha, prm.beta = alpha, beta
    prm.boundary_mode, prm.cell_order, prm.flags, prm.device = boundary_mode, cell_order, flags, device
    prm.sdf_wall_coef = sdf_wall_coef
    return prm


def _particles_view(particles: ParticleArrays, keep: list):
    arrs = [np.ascontiguousarray(getattr(particles, f), np.float32) for f in PARTICLE_FIELDS]
    ft = np.ascontiguousarray(particles.fluid_type, np.uint8)
    keep.extend(arrs + [ft])
    return SphParticlesView(len(particles), *[_fp(a) for a in arrs], ft.ctypes.data_as(_U8P))


def _boundary_view(boundary: BoundaryParticles | None, keep: list):
    if boundary is None or len(boundary) == 0:
        return SphBoundaryView(0, *([None] * 7))
    arrs = [np.ascontiguousarray(getattr(boundary, f), np.float32) for f in BOUNDARY_FIELDS]
    keep.extend(arrs)
    return SphBoundaryView(len(boundary), *[_fp(a) for a in arrs])


class CudaKernel(SimulationKernel):
    """The ``cuda`` backend: one simulation on one B200 through libsph_cuda.so.

    ``boundary_mode`` BOUNDARY_SDF replaces the boundary particles by
    homogenised walls on the six faces of the domain box plus the obstacle
    whose SDF ``sdf`` gives (None: no obstacle)."""

    def __init__(self, particles: ParticleArrays, boundary: BoundaryParticles | None, h: float,
                 gravity, speed_of_sound: float, cfl_number: float, viscosity: float,
                 domain_min, domain_max, *, alpha: float = 1.0, beta: float = 2.0,
                 boundary_mode: int = BOUNDARY_PARTICLES, sdf: GridSDF | None = None,
                 cell_order: int = CELL_ORDER_ROWS, flags: int = FLAGS_REFERENCE,
                 device: int = 0, sdf_wall_coef: float = 0.981):
        L = load_library()
        particles.validate()
        self._lib = L
        self._n = len(particles)
        self._nb = len(boundary) if boundary is not None else 0
        self.h = float(h)
        self.speed_of_sound = float(speed_of_sound)
        self.cfl_number = float(cfl_number)
        prm = default_params()
        prm.h = h
        prm.gravity = (C.c_float * 3)(*map(float, gravity))
        prm.speed_of_sound = speed_of_sound
        prm.cfl_number = cfl_number
        prm.viscosity = viscosity
        prm.domain_min = (C.c_float * 3)(*map(float, domain_min))
        prm.domain_max = (C.c_float * 3)(*map(float, domain_max))
        prm.alpha, prm.beta = alpha, beta
        prm.boundary_mode, prm.cell_order, prm.flags, prm.device = boundary_mode, cell_order, flags, device
        prm.sdf_wall_coef = sdf_wall_coef
        keep = [np.ascontiguousarray(getattr(particles, f), np.float32) for f in PARTICLE_FIELDS]
        ft = np.ascontiguousarray(particles.fluid_type, np.uint8)
        pv = SphParticlesView(self._n, *[_fp(a) for a in keep], ft.ctypes.data_as(_U8P))
        bv_p = None
        if boundary is not None and self._nb:
            bkeep = [np.ascontiguousarray(getattr(boundary, f), np.float32) for f in BOUNDARY_FIELDS]
            bv = SphBoundaryView(self._nb, *[_fp(a) for a in bkeep])
            bv_p = C.byref(bv)
        sdf_p = None
        if sdf is not None:
            dist = np.ascontiguousarray(sdf.distances, np.float32)
            sv = SphSdfView((C.c_float * 3)(*map(float, sdf.origin)), float(sdf.cell_size),
                            (C.c_uint32 * 3)(*map(int, sdf.dimensions)), _fp(dist))
            sdf_p = C.byref(sv)
        handle = C.c_void_p()
        st = L.sph_create(C.byref(prm), C.byref(pv), bv_p, sdf_p, C.byref(handle))
        if st != SPH_OK:
            raise SphError(st, "sph_create failed")
        self._h = handle
        self._cache: ParticleArrays | None = None

    # -- lifecycle -------------------------------------------------------------
    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.sph_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str) -> None:
        if st != SPH_OK:
            msg = self._lib.sph_last_error(self._h) if self._h is not None else b""
            raise SphError(st, f"{what}: {msg.decode(errors='replace') if msg else ''}")

    # -- SimulationKernel ------------------------------------------------------
    def step(self, dt: float) -> None:
        self._check(self._lib.sph_step(self._h, float(dt)), "sph_step")
        self._cache = None

    def particles(self) -> ParticleArrays:
        if self._cache is None:
            p = ParticleArrays.empty(self._n)
            out = SphParticlesMut(self._n, *[_fp(getattr(p, f)) for f in PARTICLE_FIELDS],
                                  p.fluid_type.ctypes.data_as(_U8P))
            self._check(self._lib.sph_read_particles(self._h, C.byref(out)), "sph_read_particles")
            self._cache = p
        return self._cache

    def error_metrics(self) -> ErrorMetrics:
        m = SphErrorMetrics()
        self._check(self._lib.sph_error_metrics(self._h, C.byref(m)), "sph_error_metrics")
        return ErrorMetrics(float(m.max_density_variation), float(m.energy_conservation),
                            float(m.mass_conservation))

    def particle_count(self) -> int:
        return int(self._lib.sph_particle_count(self._h))

    def save_checkpoint(self) -> bool:
        self._check(self._lib.sph_save_checkpoint(self._h), "sph_save_checkpoint")
        return True

    def restore_checkpoint(self) -> bool:
        st = self._lib.sph_restore_checkpoint(self._h)
        if st == 8:
            return False
        self._check(st, "sph_restore_checkpoint")
        self._cache = None
        return True

    # -- device-side helpers beyond the trait ----------------------------------
    def compute_timestep(self) -> float:
        """``sph::compute_timestep(particles(), h, c, cfl)`` on the device."""
        out = C.c_float()
        self._check(self._lib.sph_compute_timestep(self._h, C.byref(out)), "sph_compute_timestep")
        return float(out.value)

    def step_auto(self, nsteps: int, want_dt: bool = True) -> float | None:
        out = C.c_float()
        st = self._lib.sph_step_auto(self._h, int(nsteps), C.byref(out) if want_dt else None)
        self._check(st, "sph_step_auto")
        self._cache = None
        return float(out.value) if want_dt else None

    def step_profiled(self, dt: float) -> dict:
        prof = SphStepProfile()
        self._check(self._lib.sph_step_profiled(self._h, float(dt), C.byref(prof)), "sph_step_profiled")
        self._cache = None
        return prof.as_dict()

    def pack_frame(self, subsample_count: int, frame_number: int, sim_time: float) -> bytes:
        """The viewer's Frame message (server ws.rs:233-290) of the current
        state, packed on the device."""
        size = C.c_size_t()
        self._check(self._lib.sph_pack_frame(self._h, int(subsample_count), int(frame_number), float(sim_time),
                                             None, 0, C.byref(size)), "sph_pack_frame")
        buf = (C.c_uint8 * size.value)()
        self._check(self._lib.sph_pack_frame(self._h, int(subsample_count), int(frame_number), float(sim_time),
                                             buf, size.value, C.byref(size)), "sph_pack_frame")
        return bytes(buf)

    def run_optimistic(self, nsteps: int, alpha: float = 1.5, density_limit: float = 0.03,
                       cooldown_steps: int = 10) -> dict:
        """``nsteps`` steps of the orchestrator's optimistic time stepping
        (orchestrator runner.rs:189-240) on the device, one graph launch a
        step. Returns the run's counters (sim_time, steps, accepted,
        rejected, last_dt, cooldown), which accumulate over calls."""
        stats = SphRunStats()
        self._check(self._lib.sph_run_optimistic(self._h, int(nsteps), float(alpha), float(density_limit),
                                                 int(cooldown_steps), C.byref(stats)), "sph_run_optimistic")
        self._cache = None
        return stats.as_dict()

    def scale_velocities(self, factor: float) -> None:
        """velocity *= factor for every particle; 0 between steps is kinetic
        damping (relaxing an initial lattice before a run)."""
        self._check(self._lib.sph_scale_velocities(self._h, float(factor)), "sph_scale_velocities")
        self._cache = None

    def synchronize(self) -> None:
        self._check(self._lib.sph_synchronize(self._h), "sph_synchronize")

    def boundary_pressure(self) -> np.ndarray:
        out = np.zeros(self._nb, np.float32)
        self._check(self._lib.sph_read_boundary_pressure(self._h, _fp(out), self._nb),
                    "sph_read_boundary_pressure")
        return out

    def health(self) -> int:
        bad = C.c_uint64()
        st = self._lib.sph_health(self._h, C.byref(bad))
        if st not in (SPH_OK, 4):
            self._check(st, "sph_health")
        return int(bad.value)

    def stream(self) -> int:
        return int(self._lib.sph_stream(self._h) or 0)

    def launch_count(self) -> int:
        return int(self._lib.sph_launch_count(self._h))

    def grid_info(self) -> dict:
        g = SphGridInfo()
        self._check(self._lib.sph_grid_info(self._h, C.byref(g)), "sph_grid_info")
        return dict(dims=tuple(g.dims), total_cells=int(g.total_cells), cell_size=float(g.cell_size),
                    grid_min=tuple(g.grid_min), boundary_candidates=int(g.boundary_candidates))

    def read_grid(self) -> dict:
        info = self.grid_info()
        n, Cn = self._n, info["total_cells"]
        out = dict(cell_linear=np.zeros(n, np.uint32), morton_key=np.zeros(n, np.uint32),
                   cell_count=np.zeros(Cn, np.uint32), cell_start=np.zeros(Cn, np.uint32),
                   slot_id=np.zeros(n, np.uint32))
        self._check(self._lib.sph_read_grid(self._h, *[_u32p(out[k]) for k in (
            "cell_linear", "morton_key", "cell_count", "cell_start", "slot_id")]), "sph_read_grid")
        out.update(info)
        return out

    def set_geometry_sdf(self, sdf: GridSDF) -> None:
        """Register the obstacle SDF used by ``surface_forces``."""
        self._geo = np.ascontiguousarray(sdf.distances, np.float32)
        sv = SphSdfView((C.c_float * 3)(*map(float, sdf.origin)), float(sdf.cell_size),
                        (C.c_uint32 * 3)(*map(int, sdf.dimensions)), _fp(self._geo))
        self._check(self._lib.sph_set_geometry_sdf(self._h, C.byref(sv)), "sph_set_geometry_sdf")

    def surface_forces(self) -> dict:
        """``compute_surface_forces`` (force.rs:39-129) on the device."""
        o = SphSurfaceForce()
        self._check(self._lib.sph_surface_forces(self._h, C.byref(o)), "sph_surface_forces")
        return dict(force=np.array(o.force), moment=np.array(o.moment),
                    force_f32=np.array(o.force_f32, np.float32), moment_f32=np.array(o.moment_f32, np.float32),
                    nodes=int(o.nodes), active_nodes=int(o.active_nodes))

    def body_force(self, first: int, count: int) -> dict:
        """Fluid reaction on boundary particles [first, first + count)."""
        o = SphBodyForce()
        self._check(self._lib.sph_body_force(self._h, int(first), int(count), C.byref(o)), "sph_body_force")
        return {k: np.array(getattr(o, k)) for k, _ in SphBodyForce._fields_}

    def neighbors(self, pid: int, cap: int = 4096) -> np.ndarray:
        out = np.zeros(cap, np.uint32)
        cnt = C.c_size_t()
        self._check(self._lib.sph_neighbors(self._h, int(pid), _u32p(out), cap, C.byref(cnt)),
                    "sph_neighbors")
        return out[:min(cap, cnt.value)].copy()

    # -- learned closure ---------------------------------------------------------
    @staticmethod
    def _sdf_view(sdf: GridSDF, keep: list) -> SphSdfView:
        d = np.ascontiguousarray(sdf.distances, np.float32)
        keep.append(d)
        return SphSdfView((C.c_float * 3)(*map(float, sdf.origin)), float(sdf.cell_size),
                          (C.c_uint32 * 3)(*map(int, sdf.dimensions)), _fp(d))

    def set_feature_sdf(self, sdf: GridSDF) -> None:
        """Geometry SDF (walls and obstacles) of the closure features."""
        keep = []
        sv = self._sdf_view(sdf, keep)
        self._check(self._lib.sph_set_feature_sdf(self._h, C.byref(sv)), "sph_set_feature_sdf")

    def set_closure(self, mode: int, params=None) -> None:
        """0 off, 1 record features, 2 record and apply ``params``."""
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        self._check(self._lib.sph_set_closure(self._h, int(mode), None if p is None else _fp(p)), "sph_set_closure")

    def closure_samples(self):
        """(ids, features[n, 16], density before correction) of the last density pass."""
        cnt = C.c_size_t()
        self._check(self._lib.sph_closure_samples(self._h, 0, None, None, None, C.byref(cnt)), "sph_closure_samples")
        n = cnt.value
        ids = np.zeros(n, np.uint32)
        feat = np.zeros((n, 16), np.float32)
        rho = np.zeros(n, np.float32)
        self._check(self._lib.sph_closure_samples(self._h, n, _u32p(ids), _fp(feat), _fp(rho), C.byref(cnt)),
                    "sph_closure_samples")
        return ids, feat, rho

    def interpolate(self, pts) -> np.ndarray:
        """Shepard interpolation at pts[n, 3]: columns rho, p, ax, ay, az, wsum, count."""
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.zeros((pts.shape[0], 7), np.float32)
        self._check(self._lib.sph_interpolate(self._h, _fp(pts), pts.shape[0], _fp(out)), "sph_interpolate")
        return out

    # -- launch shapes ---------------------------------------------------------
    def launch(self) -> dict:
        l = SphLaunch()
        self._check(self._lib.sph_get_launch(self._h, C.byref(l)), "sph_get_launch")
        return l.as_dict()

    def set_launch(self, xsph_threads: int, density_threads: int, forces_threads: int) -> None:
        l = SphLaunch(xsph_threads, density_threads, forces_threads)
        self._check(self._lib.sph_set_launch(self._h, C.byref(l)), "sph_set_launch")

    def autotune(self, trial_steps: int = 3) -> dict:
        """Native autotuner; advances this simulation by its trial steps."""
        l = SphLaunch()
        self._check(self._lib.sph_autotune(self._h, int(trial_steps), C.byref(l)), "sph_autotune")
        return l.as_dict()


class CudaBatch(CudaKernel):
    """Many independent simulations stepped by the same kernel launches
    (``sph_batch_create``). ``scenarios`` hold what ``CpuKernel::new`` takes
    per instance (``domain.Scenario``); ``particles()`` returns the instances
    one after another, ``instance(q)`` slices one out."""

    def __init__(self, scenarios, device: int = 0, cell_order: int = CELL_ORDER_ROWS,
                 boundary_mode: int = BOUNDARY_PARTICLES):
        L = load_library()
        self._lib = L
        self._keep = []
        nq = len(scenarios)
        prms = (SphParams * nq)()
        views = (SphParticlesView * nq)()
        bviews = (SphBoundaryView * nq)()
        sviews = (SphSdfView * nq)()
        for q, sc in enumerate(scenarios):
            sc.particles.validate()
            prms[q] = make_params(sc.h, sc.gravity, sc.speed_of_sound, sc.cfl_number, sc.viscosity,
                                  sc.domain_min, sc.domain_max, alpha=sc.alpha, beta=sc.beta,
                                  cell_order=cell_order, device=device, boundary_mode=boundary_mode)
            views[q] = _particles_view(sc.particles, self._keep)
            bviews[q] = _boundary_view(sc.boundary, self._keep)
            if boundary_mode == BOUNDARY_SDF and sc.obstacle_sdf is not None:
                sviews[q] = self._sdf_view(sc.obstacle_sdf, self._keep)
        handle = C.c_void_p()
        if boundary_mode == BOUNDARY_SDF:
            st = L.sph_batch_create_sdf(nq, prms, views, sviews, C.byref(handle))
        else:
            st = L.sph_batch_create(nq, prms, views, bviews, C.byref(handle))
        self._keep = []
        if st != SPH_OK:
            raise SphError(st, "sph_batch_create failed")
        self._h = handle
        self._cache = None
        self._n = sum(len(sc.particles) for sc in scenarios)
        self._nb = 0 if boundary_mode == BOUNDARY_SDF else sum(
            len(sc.boundary) if sc.boundary is not None else 0 for sc in scenarios)
        self.ninst = nq
        first = (C.c_size_t * nq)()
        count = (C.c_size_t * nq)()
        ni = C.c_int()
        self._check(L.sph_batch_info(self._h, C.byref(ni), first, count), "sph_batch_info")
        self.first = np.array(first[:], np.int64)
        self.count = np.array(count[:], np.int64)

    def set_feature_sdfs(self, sdfs) -> None:
        keep = []
        arr = (SphSdfView * len(sdfs))(*[self._sdf_view(sd, keep) for sd in sdfs])
        self._check(self._lib.sph_batch_set_feature_sdfs(self._h, arr), "sph_batch_set_feature_sdfs")

    def step_each(self, dts) -> None:
        """One step with instance q advanced by dts[q]."""
        d = np.ascontiguousarray(dts, np.float32)
        if d.shape != (self.ninst,):
            raise ValueError("one dt per instance")
        self._check(self._lib.sph_batch_step(self._h, _fp(d)), "sph_batch_step")
        self._cache = None

    def timesteps(self) -> np.ndarray:
        out = np.zeros(self.ninst, np.float32)
        self._check(self._lib.sph_batch_timesteps(self._h, _fp(out)), "sph_batch_timesteps")
        return out

    def instance(self, q: int) -> ParticleArrays:
        p = self.particles()
        a, b = int(self.first[q]), int(self.first[q] + self.count[q])
        out = ParticleArrays(**{f: getattr(p, f)[a:b].copy() for f in PARTICLE_FIELDS})
        out.fluid_type = p.fluid_type[a:b].copy()
        return out


def setup_domain(spec, sdf: GridSDF, device: int = 0) -> tuple[ParticleArrays, BoundaryParticles]:
    """``setup_domain(config, sdf)`` (orchestrator domain.rs:36-402) on the
    device: the fluid lattice, the wall layers and the geometry layers, in
    the reference's order and bit for bit. ``spec`` is a
    ``particles.DomainSpec``."""
    L = load_library()
    s = SphDomainSpec(float(spec.particle_spacing), (C.c_float * 3)(*map(float, spec.domain_min)),
                      (C.c_float * 3)(*map(float, spec.domain_max)), int(spec.fluid_type),
                      float(spec.initial_temperature), int(spec.wall_faces))
    keep = []
    sv = CudaKernel._sdf_view(sdf, keep)
    nf, nb = C.c_size_t(), C.c_size_t()

    def check(st):
        if st != SPH_OK:
            raise SphError(st, "sph_setup_domain")
    check(L.sph_setup_domain(int(device), C.byref(s), C.byref(sv), None, None, C.byref(nf), C.byref(nb)))
    p = ParticleArrays.empty(nf.value)
    b = BoundaryParticles.from_arrays(*[np.zeros(nb.value, np.float32) for _ in range(7)])
    pm = SphParticlesMut(nf.value, *[_fp(getattr(p, f)) for f in PARTICLE_FIELDS],
                         p.fluid_type.ctypes.data_as(C.POINTER(C.c_uint8)))
    bm = SphBoundaryMut(nb.value, *[_fp(getattr(b, f)) for f in BOUNDARY_FIELDS])
    check(L.sph_setup_domain(int(device), C.byref(s), C.byref(sv), C.byref(pm), C.byref(bm), C.byref(nf),
                             C.byref(nb)))
    return p, b
