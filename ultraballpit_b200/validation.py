"""The reference's validation benchmarks, driven through the kernel interface.

Restates the harness of ``backend/reference-tests/src/benchmarks.rs``:

* T086 dam break (``benchmarks.rs:53-223``, ``configs/dam-break-2d.json``):
  boundary particles from ``setup_domain`` of the config, the water column
  placed by hand in the left quarter of the slab (``benchmarks.rs:80-108``),
  ``CpuKernel::new`` with the config's speed of sound (no auto-tune), the
  host loop ``dt = min(compute_timestep(..), t_end - t)`` with a snapshot each
  time the simulated time passes a multiple of 0.01 s
  (``benchmarks.rs:128-157``), and the water front ``max x`` of every
  snapshot as ``Z* = x / a`` against ``T* = t sqrt(2 g / a)`` up to
  ``T* = 3.5`` (``benchmarks.rs:176-196``);
* T087 hydrostatic (``benchmarks.rs:242-343``,
  ``configs/hydrostatic-hires.json``): fluid and boundary particles from
  ``setup_domain`` (``reference-tests/src/lib.rs:490-528``), the same loop to
  ``t = 1 s``, and the mean pressure of the particles in 10 depth bands of
  half-width ``H / 20`` against ``rho g depth``.

The configs' geometry is ``geometries/null-obstacle.stl``: a 1 mm cube at
``(-1, -1, -1)`` m, outside both domains. Its SDF (``mesh_to_sdf`` 0.3.0, not
vendored) is about 1.7 m at every node, so ``setup_domain`` keeps every
lattice point as fluid and places no geometry layers; the Euclidean distance
to that cube on the same node grid (origin ``domain.min``, cell
``0.5 * spacing``, ``ceil(extent / cell) + 1`` nodes, ``geometry.rs:44-90``)
gives the same particles.

The runs take any object with the ``SimulationKernel`` methods plus
``compute_timestep`` (``CudaKernel``, or the oracle behind an adapter in the
tests), so the CUDA path and the CPU restatement run the same loop.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .domain import Scenario, sdf_node_grid, smoothing_length
from .particles import DomainSpec, FluidType, GridSDF, ParticleArrays

f32 = np.float32
WATER_REST_DENSITY = f32(1000.0)  # kernel/src/eos.rs:7

# configs/dam-break-2d.json and configs/hydrostatic-hires.json: the fields
# setup_domain and CpuKernel::new read (orchestrator/src/config.rs:26-64)
DAM_BREAK_2D = dict(domain_min=(0.0, 0.0, 0.0), domain_max=(0.05, 0.10, 0.004), particle_spacing=0.002,
                    walls=("x_min", "y_min", "z_min", "z_max"), gravity=(0.0, -9.81, 0.0),
                    speed_of_sound=20.0, viscosity=0.001, cfl_number=0.4, max_time=0.5)
HYDROSTATIC_HIRES = dict(domain_min=(0.0, 0.0, 0.0), domain_max=(0.005, 0.05, 0.005), particle_spacing=0.001,
                         walls=("x_min", "x_max", "y_min", "y_max", "z_min", "z_max"),
                         gravity=(0.0, -9.81, 0.0), speed_of_sound=20.0, viscosity=0.001, cfl_number=0.4)
NULL_OBSTACLE = ((-1.0, -1.0, -1.0), (-0.999, -0.999, -0.999))  # geometries/null-obstacle.stl bounds


def null_obstacle_sdf(domain_min, domain_max, spacing) -> GridSDF:
    """Distance to the null obstacle on the mesh_to_sdf node grid of the
    domain (cell 0.5 spacing, geometry.rs:36-90): positive everywhere."""
    cell = f32(0.5) * f32(spacing)
    dims, (ax, ay, az) = sdf_node_grid(domain_min, domain_max, cell)
    lo, hi = (np.asarray(v, np.float64) for v in NULL_OBSTACLE)
    X, Y, Z = np.meshgrid(ax.astype(np.float64), ay.astype(np.float64), az.astype(np.float64), indexing="ij")
    d = [np.maximum(np.maximum(lo[a] - P, P - hi[a]), 0.0) for a, P in enumerate((X, Y, Z))]
    dist = np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
    return GridSDF(tuple(float(v) for v in domain_min), float(cell), dims, dist.astype(np.float32).ravel())


def _spec(cfg) -> DomainSpec:
    return DomainSpec(float(f32(cfg["particle_spacing"])), cfg["domain_min"], cfg["domain_max"],
                      wall_faces=DomainSpec.faces_mask(cfg["walls"]))


def dam_break_2d(setup_domain) -> tuple[Scenario, float]:
    """T086's initial state (benchmarks.rs:63-124): (scenario, column width a).

    ``setup_domain(spec, sdf)`` is the domain builder to use (the device's
    ``kernel.setup_domain`` or the oracle's restatement); only its boundary
    particles are kept, as the reference does."""
    cfg = DAM_BREAK_2D
    sdf = null_obstacle_sdf(cfg["domain_min"], cfg["domain_max"], cfg["particle_spacing"])
    _, boundary = setup_domain(_spec(cfg), sdf)
    spacing = f32(cfg["particle_spacing"])
    dmin = [f32(v) for v in cfg["domain_min"]]
    dmax = [f32(v) for v in cfg["domain_max"]]
    a = f32(f32(dmax[0] - dmin[0]) / f32(4.0))
    column_height = f32(f32(2.0) * a)
    water_mass = f32(WATER_REST_DENSITY * f32(f32(spacing * spacing) * spacing))
    nx = int(math.ceil(f32(a / spacing)))
    ny = int(math.ceil(f32(column_height / spacing)))
    nz = int(math.ceil(f32(f32(dmax[2] - dmin[2]) / spacing)))
    p = ParticleArrays()
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                x = f32(dmin[0] + f32(f32(f32(i) + f32(0.5)) * spacing))
                y = f32(dmin[1] + f32(f32(f32(j) + f32(0.5)) * spacing))
                z = f32(dmin[2] + f32(f32(f32(k) + f32(0.5)) * spacing))
                if x <= f32(dmin[0] + a) and y <= f32(dmin[1] + column_height) and z <= dmax[2]:
                    p.push_particle(x, y, z, water_mass, WATER_REST_DENSITY, 293.15, FluidType.Water)
    h = smoothing_length(float(spacing))
    sc = Scenario("dam_break_2d", p, boundary, float(h), cfg["gravity"], cfg["speed_of_sound"],
                  cfg["cfl_number"], cfg["viscosity"], cfg["domain_min"], cfg["domain_max"])
    return sc, float(a)


def hydrostatic_hires(setup_domain) -> Scenario:
    """T087's initial state: setup_domain of the config (lib.rs:497-528)."""
    cfg = HYDROSTATIC_HIRES
    sdf = null_obstacle_sdf(cfg["domain_min"], cfg["domain_max"], cfg["particle_spacing"])
    fluid, boundary = setup_domain(_spec(cfg), sdf)
    h = smoothing_length(float(f32(cfg["particle_spacing"])))
    return Scenario("hydrostatic_hires", fluid, boundary, float(h), cfg["gravity"], cfg["speed_of_sound"],
                    cfg["cfl_number"], cfg["viscosity"], cfg["domain_min"], cfg["domain_max"])


@dataclass
class Run:
    """Snapshots of a run: (time, x, y, pressure) in original particle order."""

    times: list = field(default_factory=list)
    x: list = field(default_factory=list)
    y: list = field(default_factory=list)
    pressure: list = field(default_factory=list)
    steps: int = 0

    def add(self, t: float, p: ParticleArrays) -> None:
        self.times.append(t)
        self.x.append(p.x.copy())
        self.y.append(p.y.copy())
        self.pressure.append(p.pressure.copy())


def run_to_time(kernel, target_time: float, snapshot_interval: float, stop_time: float | None = None) -> Run:
    """The reference loop (benchmarks.rs:128-157, lib.rs:530-566): host dt
    from ``compute_timestep`` clamped to the remaining time, a snapshot when
    the simulated time (f64) passes the next multiple of the interval, and a
    final snapshot. ``stop_time`` ends the loop early (a prefix of the same
    run: the clamp only acts on the last step before ``target_time``)."""
    run = Run()
    t, nxt = 0.0, snapshot_interval
    run.add(t, kernel.particles())
    end = target_time if stop_time is None else min(stop_time, target_time)
    while t < end:
        dt = f32(kernel.compute_timestep())
        dt = min(dt, f32(target_time - t))
        if dt <= 0.0:
            break
        kernel.step(float(dt))
        t += float(dt)
        run.steps += 1
        if t >= nxt:
            run.add(t, kernel.particles())
            nxt += snapshot_interval
    run.add(t, kernel.particles())
    return run


def front_positions(run: Run, a: float, g: float = 9.81, domain_min_x: float = 0.0,
                    t_star_max: float = 3.5) -> list[tuple[float, float]]:
    """(T*, Z*) of every snapshot up to T* = 3.5 (benchmarks.rs:176-196):
    the front is the largest x of any particle, from domain.min.x."""
    gg = float(abs(f32(g)))
    out = []
    for t, x in zip(run.times, run.x):
        if t < 1e-6:
            continue
        t_star = t * math.sqrt(2.0 * gg / float(f32(a)))
        if t_star > t_star_max:
            break
        front = max(f32(domain_min_x), f32(x.max())) if x.size else f32(domain_min_x)
        out.append((t_star, float(front) / float(f32(a))))
    return out


def hydrostatic_bands(y: np.ndarray, pressure: np.ndarray, domain_min_y: float, domain_max_y: float,
                      g: float = 9.81, n_levels: int = 10) -> list[dict]:
    """Mean pressure in 10 depth bands (benchmarks.rs:273-333): band centres
    at depth (level + 0.5) H / 10 below domain.max.y, half-width H / 20."""
    ymax, ymin = float(f32(domain_max_y)), float(f32(domain_min_y))
    height = ymax - ymin
    rho, gg = float(WATER_REST_DENSITY), float(abs(f32(g)))
    yy, pp = y.astype(np.float64), pressure.astype(np.float64)
    out = []
    for level in range(n_levels):
        frac = (level + 0.5) / n_levels
        y_target = ymax - frac * height
        depth = ymax - y_target
        band = height / (2.0 * n_levels)
        sel = np.abs(yy - y_target) < band
        expected = rho * gg * depth
        if not sel.any():
            out.append(dict(depth=depth, p_sim=None, p_ana=expected, count=0))
            continue
        avg = float(sum(pp[sel].tolist()) / int(sel.sum()))  # sequential sum, as the reference's iter().sum()
        out.append(dict(depth=depth, p_sim=avg, p_ana=expected, count=int(sel.sum()),
                        error=abs(avg - expected) / expected if expected > 1.0 else abs(avg - expected)))
    return out
