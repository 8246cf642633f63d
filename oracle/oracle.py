"""ctypes wrapper of the CPU oracle (``oracle/sph_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py. The product path never imports this module.

``OracleKernel`` mirrors the reference ``CpuKernel`` (``kernel/src/lib.rs:91-396``)
with two tiers: ``tier=0`` keeps the reference's O(N * N_b) boundary scans,
``tier=1`` visits the same boundary terms through grid candidate lists and gives
identical results. ``pow_mode=0`` evaluates the Tait power with libm ``powf``
(the reference on Linux); ``pow_mode=1`` with the correctly rounded power that
the CUDA step uses.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from ultraballpit_b200.particles import (BOUNDARY_FIELDS, PARTICLE_FIELDS, BoundaryParticles,
                                         ErrorMetrics, ParticleArrays)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle_sph.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ only)."""
    src = os.path.join(_HERE, "sph_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "CXX=g++"], check=True, capture_output=True)
    return LIB_PATH


class OrcParams(C.Structure):
    _fields_ = [("h", C.c_float), ("gravity", C.c_float * 3), ("speed_of_sound", C.c_float),
                ("cfl_number", C.c_float), ("viscosity", C.c_float),
                ("domain_min", C.c_float * 3), ("domain_max", C.c_float * 3),
                ("alpha", C.c_float), ("beta", C.c_float), ("tier", C.c_int),
                ("threads", C.c_int), ("pow_mode", C.c_int), ("boundary_mode", C.c_int),
                ("sdf_wall_coef", C.c_float), ("sdf_origin", C.c_float * 3), ("sdf_cell", C.c_float),
                ("sdf_dims", C.c_uint32 * 3), ("sdf", C.POINTER(C.c_float)), ("flags", C.c_uint32)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        fp, u32p, vp = C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_void_p
        L.orc_wendland.restype = C.c_float
        L.orc_wendland.argtypes = [C.c_float, C.c_float]
        L.orc_wendland_gradient.argtypes = [C.c_float] * 5 + [fp]
        L.orc_tait.restype = C.c_float
        L.orc_tait.argtypes = [C.c_float] * 4 + [C.c_int]
        L.orc_norm.restype = C.c_float
        L.orc_grid_dims.argtypes = [C.c_float, fp, fp, u32p]
        L.orc_grid_build.argtypes = [C.c_size_t, fp, fp, fp, C.c_float, fp, fp] + [u32p] * 7
        L.orc_neighbors.restype = C.c_size_t
        L.orc_neighbors.argtypes = [C.c_size_t, fp, fp, fp, C.c_float, fp, fp, C.c_size_t, u32p, C.c_size_t]
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_size_t, C.POINTER(fp), C.POINTER(C.c_uint8),
                                 C.c_size_t, C.POINTER(fp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_step.argtypes = [vp, C.c_float]
        L.orc_compute_forces.argtypes = [vp, C.c_float]
        L.orc_particle_count.restype = C.c_size_t
        L.orc_particle_count.argtypes = [vp]
        L.orc_get.argtypes = [vp, C.POINTER(fp), C.POINTER(C.c_uint8)]
        L.orc_get_boundary_pressure.argtypes = [vp, fp]
        L.orc_error_metrics.argtypes = [vp, fp]
        L.orc_compute_timestep.restype = C.c_float
        L.orc_compute_timestep.argtypes = [vp, C.c_float]
        L.orc_save_checkpoint.restype = C.c_int
        L.orc_save_checkpoint.argtypes = [vp]
        L.orc_restore_checkpoint.restype = C.c_int
        L.orc_restore_checkpoint.argtypes = [vp]
        L.orc_boundary_list_size.restype = C.c_size_t
        L.orc_boundary_list_size.argtypes = [vp]
        L.orc_compute_timestep_arrays.restype = C.c_float
        L.orc_compute_timestep_arrays.argtypes = [C.c_size_t] + [fp] * 6 + [C.c_float] * 3
        L.orc_sdf_sample.restype = C.c_float
        L.orc_sdf_sample.argtypes = [fp, u32p, fp, C.c_float, fp]
        L.orc_sdf_gradient.argtypes = [fp, u32p, fp, C.c_float, fp, fp]
        L.orc_surface_forces.argtypes = [vp, fp, u32p, fp, C.c_float, fp, C.POINTER(C.c_double),
                                         C.POINTER(C.c_uint32)]
        L.orc_body_force.argtypes = [vp, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]
        L.orc_wall_table.restype = C.c_int
        L.orc_wall_table.argtypes = [C.c_float, fp, fp, fp]
        L.orc_wall_tables_box.restype = C.c_int
        L.orc_wall_tables_box.argtypes = [C.c_float, fp, fp, fp, fp, fp, fp]
        L.orc_setup_domain.argtypes = [C.c_float, fp, fp, C.c_int, C.c_uint32, fp, u32p, fp, C.c_float,
                                       C.POINTER(C.c_uint64)] + [fp] * 5 + [C.POINTER(C.c_uint8)] + [fp] * 7
        L.orc_sdf_sample_clamped.restype = C.c_float
        L.orc_sdf_sample_clamped.argtypes = [fp, u32p, fp, C.c_float, fp]
        L.orc_sdf_gradient_clamped.argtypes = [fp, u32p, fp, C.c_float, fp, fp]
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


# ---- scalar functions -------------------------------------------------------

def wendland(r: float, h: float) -> float:
    return lib().orc_wendland(r, h)


def wendland_gradient(dx, dy, dz, r, h):
    out = np.zeros(3, np.float32)
    lib().orc_wendland_gradient(dx, dy, dz, r, h, _fp(out))
    return out


def tait(rho, rho0, c, gamma, pow_mode: int = 0) -> float:
    return lib().orc_tait(rho, rho0, c, gamma, pow_mode)


def norm() -> float:
    return lib().orc_norm()


# ---- grid -------------------------------------------------------------------

def grid_dims(cell, dmin, dmax):
    out = np.zeros(3, np.uint32)
    lib().orc_grid_dims(cell, _f3(dmin), _f3(dmax), _u32p(out))
    return tuple(int(v) for v in out)


def grid_build(x, y, z, cell, dmin, dmax) -> dict:
    """Reference ``NeighborGrid::update`` outputs plus the Morton layout."""
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    n = x.shape[0]
    dims = grid_dims(cell, dmin, dmax)
    tc = dims[0] * dims[1] * dims[2]
    out = dict(cell_idx=np.zeros(n, np.uint32), counts=np.zeros(tc, np.uint32),
               offsets=np.zeros(tc, np.uint32), sorted=np.zeros(n, np.uint32),
               morton_key=np.zeros(n, np.uint32), morton_offsets=np.zeros(tc, np.uint32),
               morton_perm=np.zeros(n, np.uint32))
    lib().orc_grid_build(n, _fp(x), _fp(y), _fp(z), cell, _f3(dmin), _f3(dmax),
                         *[_u32p(out[k]) for k in ("cell_idx", "counts", "offsets", "sorted",
                                                   "morton_key", "morton_offsets", "morton_perm")])
    out["dims"] = dims
    return out


def neighbors(x, y, z, h, dmin, dmax, i, cap=4096) -> np.ndarray:
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    out = np.zeros(cap, np.uint32)
    k = lib().orc_neighbors(x.shape[0], _fp(x), _fp(y), _fp(z), h, _f3(dmin), _f3(dmax), i, _u32p(out), cap)
    return out[:min(k, cap)].copy()


def sdf_sample(sdf, pt) -> float:
    dims = np.asarray(sdf.dimensions, np.uint32)
    return lib().orc_sdf_sample(_fp(sdf.distances), _u32p(dims), _f3(sdf.origin), sdf.cell_size,
                                _f3(pt))


def sdf_gradient(sdf, pt) -> np.ndarray:
    dims = np.asarray(sdf.dimensions, np.uint32)
    out = np.zeros(3, np.float32)
    lib().orc_sdf_gradient(_fp(sdf.distances), _u32p(dims), _f3(sdf.origin), sdf.cell_size,
                           _f3(pt), _fp(out))
    return out


WALL_N = 512


def wall_table(h):
    """(phi, grad, inv_step) of the SDF wall at smoothing length h."""
    phi = np.zeros(WALL_N + 1, np.float32)
    grad = np.zeros(WALL_N + 1, np.float32)
    inv = np.zeros(1, np.float32)
    lib().orc_wall_table(h, _fp(phi), _fp(grad), _fp(inv))
    return phi, grad, float(inv[0])


WALL_N2, WALL_N3 = 64, 24


def wall_tables_box(h):
    """Edge tables (phi2, grad2)[(N2 + 1), (N2 + 1)] and corner tables
    (phi3, grad3)[(N3 + 1),] * 3 of the SDF-mode box walls, with their
    inverse steps."""
    n2, n3 = WALL_N2 + 1, WALL_N3 + 1
    phi2, grad2 = np.zeros(n2 * n2, np.float32), np.zeros(n2 * n2, np.float32)
    phi3, grad3 = np.zeros(n3 ** 3, np.float32), np.zeros(n3 ** 3, np.float32)
    inv = np.zeros(2, np.float32)
    code = lib().orc_wall_tables_box(h, _fp(phi2), _fp(grad2), _fp(phi3), _fp(grad3), _fp(inv[:1]), _fp(inv[1:]))
    assert code == WALL_N2 * 1000 + WALL_N3
    return (phi2.reshape(n2, n2), grad2.reshape(n2, n2), phi3.reshape(n3, n3, n3), grad3.reshape(n3, n3, n3),
            float(inv[0]), float(inv[1]))


def sdf_sample_clamped(sdf, pt) -> float:
    dims = np.asarray(sdf.dimensions, np.uint32)
    return lib().orc_sdf_sample_clamped(_fp(sdf.distances), _u32p(dims), _f3(sdf.origin), sdf.cell_size,
                                        _f3(pt))


def compute_timestep_arrays(p: ParticleArrays, h, c, cfl) -> float:
    return lib().orc_compute_timestep_arrays(len(p), *[_fp(getattr(p, f)) for f in
                                                       ("vx", "vy", "vz", "ax", "ay", "az")], h, c, cfl)


# ---- kernel -----------------------------------------------------------------

class OracleKernel:
    """CPU restatement of ``CpuKernel`` (``lib.rs:91-396``)."""

    def __init__(self, particles: ParticleArrays, boundary: BoundaryParticles, h, gravity,
                 speed_of_sound, cfl_number, viscosity, domain_min, domain_max, *,
                 alpha: float = 1.0, beta: float = 2.0, tier: int = 1, threads: int = 1,
                 pow_mode: int = 0, boundary_mode: int = 0, sdf=None, sdf_wall_coef: float = 0.981,
                 flags: int = 0xF):
        particles.validate()
        self._n = len(particles)
        self._nb = len(boundary)
        prm = OrcParams(h=h, gravity=_f3(gravity), speed_of_sound=speed_of_sound,
                        cfl_number=cfl_number, viscosity=viscosity, domain_min=_f3(domain_min),
                        domain_max=_f3(domain_max), alpha=alpha, beta=beta, tier=tier,
                        threads=threads, pow_mode=pow_mode, boundary_mode=boundary_mode,
                        sdf_wall_coef=sdf_wall_coef, flags=flags)
        if boundary_mode == 1 and sdf is not None:  # the obstacle; the box faces are walls anyway
            self._sdf = np.ascontiguousarray(sdf.distances, np.float32)
            prm.sdf_origin = _f3(sdf.origin)
            prm.sdf_cell = float(sdf.cell_size)
            prm.sdf_dims = (C.c_uint32 * 3)(*map(int, sdf.dimensions))
            prm.sdf = _fp(self._sdf)
        self.h, self.speed_of_sound = float(h), float(speed_of_sound)
        keep = [np.ascontiguousarray(getattr(particles, f), np.float32) for f in PARTICLE_FIELDS]
        fields = (C.POINTER(C.c_float) * 13)(*[_fp(a) for a in keep])
        ft = np.ascontiguousarray(particles.fluid_type, np.uint8)
        bkeep = [np.ascontiguousarray(getattr(boundary, f), np.float32) for f in BOUNDARY_FIELDS]
        bfields = (C.POINTER(C.c_float) * 7)(*[_fp(a) for a in bkeep])
        self._h = lib().orc_create(C.byref(prm), self._n, fields,
                                   ft.ctypes.data_as(C.POINTER(C.c_uint8)), self._nb, bfields)
        if not self._h:
            raise RuntimeError("orc_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def step(self, dt: float) -> None:
        lib().orc_step(self._h, dt)

    def compute_forces(self, dt: float) -> None:
        lib().orc_compute_forces(self._h, dt)

    def particles(self) -> ParticleArrays:
        p = ParticleArrays.empty(self._n)
        fields = (C.POINTER(C.c_float) * 13)(*[_fp(getattr(p, f)) for f in PARTICLE_FIELDS])
        lib().orc_get(self._h, fields, p.fluid_type.ctypes.data_as(C.POINTER(C.c_uint8)))
        return p

    def boundary_pressure(self) -> np.ndarray:
        out = np.zeros(self._nb, np.float32)
        lib().orc_get_boundary_pressure(self._h, _fp(out))
        return out

    def error_metrics(self) -> ErrorMetrics:
        out = np.zeros(3, np.float32)
        lib().orc_error_metrics(self._h, _fp(out))
        return ErrorMetrics(float(out[0]), float(out[1]), float(out[2]))

    def particle_count(self) -> int:
        return self._n

    def compute_timestep(self, cfl: float) -> float:
        return lib().orc_compute_timestep(self._h, cfl)

    def save_checkpoint(self) -> bool:
        return bool(lib().orc_save_checkpoint(self._h))

    def restore_checkpoint(self) -> bool:
        return bool(lib().orc_restore_checkpoint(self._h))

    def surface_forces(self, sdf) -> dict:
        """force.rs:39-129 literally (f32) plus the same nodes summed in FP64."""
        dims = np.asarray(sdf.dimensions, np.uint32)
        dist = np.ascontiguousarray(sdf.distances, np.float32)
        f32 = np.zeros(6, np.float32)
        f64 = np.zeros(6, np.float64)
        nodes = C.c_uint32()
        lib().orc_surface_forces(self._h, _fp(dist), _u32p(dims), _f3(sdf.origin), sdf.cell_size, _fp(f32),
                                 f64.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nodes))
        return dict(force_f32=f32[:3], moment_f32=f32[3:], force=f64[:3], moment=f64[3:], nodes=nodes.value)

    def body_force(self, first: int, count: int) -> dict:
        """Fluid reaction on boundary particles [first, first + count) from
        the last force computation."""
        out = np.zeros(18, np.float64)
        lib().orc_body_force(self._h, first, count, out.ctypes.data_as(C.POINTER(C.c_double)))
        keys = ("pressure_force", "pressure_moment", "repulsion_force", "repulsion_moment", "viscous_force",
                "viscous_moment")
        return {k: out[3 * i:3 * i + 3] for i, k in enumerate(keys)}

    def boundary_list_size(self) -> int:
        return int(lib().orc_boundary_list_size(self._h))


def setup_domain(spec, sdf):
    """``setup_domain(config, sdf)`` (orchestrator domain.rs:36-402) by the
    literal restatement: (ParticleArrays, BoundaryParticles)."""
    L = lib()
    dims = np.asarray(sdf.dimensions, np.uint32)
    dist = np.ascontiguousarray(sdf.distances, np.float32)
    args = (C.c_float(spec.particle_spacing), _f3(spec.domain_min), _f3(spec.domain_max), int(spec.fluid_type),
            int(spec.wall_faces), _fp(dist), _u32p(dims), _f3(sdf.origin), C.c_float(sdf.cell_size))
    counts = (C.c_uint64 * 2)()
    nul = C.POINTER(C.c_float)()
    L.orc_setup_domain(*args, counts, nul, nul, nul, nul, nul, C.POINTER(C.c_uint8)(), *([nul] * 7))
    n, nb = int(counts[0]), int(counts[1])
    p = ParticleArrays.empty(n)
    b = BoundaryParticles.from_arrays(*[np.zeros(nb, np.float32) for _ in range(7)])
    L.orc_setup_domain(*args, counts, _fp(p.x), _fp(p.y), _fp(p.z), _fp(p.mass), _fp(p.density),
                       p.fluid_type.ctypes.data_as(C.POINTER(C.c_uint8)),
                       *[_fp(getattr(b, f)) for f in BOUNDARY_FIELDS])
    p.temperature[:] = np.float32(spec.initial_temperature)
    return p, b
