"""Particle and boundary containers mirroring the reference kernel crate's types.

``ParticleArrays`` follows ``kernel/src/particle.rs:22-120`` (struct of arrays,
13 f32 fields plus a u8 fluid type), ``BoundaryParticles`` follows
``kernel/src/boundary.rs:20-76`` and ``ErrorMetrics`` follows
``kernel/src/lib.rs:40-47``. ``GridSDF`` holds the node grid of
``orchestrator/src/geometry.rs:11-20`` (index ``i*ny*nz + j*nz + k``, z fastest).

All arrays are numpy ``float32`` (``uint8`` for the fluid type) so that host
data crosses the C ABI without conversion.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field

import numpy as np

PARTICLE_FIELDS = (
    "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az",
    "density", "pressure", "mass", "temperature",
)
BOUNDARY_FIELDS = ("x", "y", "z", "mass", "nx", "ny", "nz")


class FluidType(enum.IntEnum):
    """``kernel/src/particle.rs:9-14`` (``repr(u8)``)."""

    Water = 0
    Air = 1


def _f32(n: int = 0) -> np.ndarray:
    return np.zeros(n, dtype=np.float32)


@dataclass
class ParticleArrays:
    """Struct-of-arrays fluid particle storage (``particle.rs:22-58``)."""

    x: np.ndarray = field(default_factory=_f32)
    y: np.ndarray = field(default_factory=_f32)
    z: np.ndarray = field(default_factory=_f32)
    vx: np.ndarray = field(default_factory=_f32)
    vy: np.ndarray = field(default_factory=_f32)
    vz: np.ndarray = field(default_factory=_f32)
    ax: np.ndarray = field(default_factory=_f32)
    ay: np.ndarray = field(default_factory=_f32)
    az: np.ndarray = field(default_factory=_f32)
    density: np.ndarray = field(default_factory=_f32)
    pressure: np.ndarray = field(default_factory=_f32)
    mass: np.ndarray = field(default_factory=_f32)
    temperature: np.ndarray = field(default_factory=_f32)
    fluid_type: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint8))

    @classmethod
    def empty(cls, n: int) -> "ParticleArrays":
        p = cls(**{f: _f32(n) for f in PARTICLE_FIELDS})
        p.fluid_type = np.zeros(n, dtype=np.uint8)
        return p

    @classmethod
    def from_positions(cls, x, y, z, mass, density=1000.0, temperature=293.15,
                       fluid_type: FluidType = FluidType.Water) -> "ParticleArrays":
        """Vectorised ``push_particle`` (``particle.rs:96-120``): zero v, a, p."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        p = cls.empty(n)
        p.x[:] = x
        p.y[:] = np.asarray(y, dtype=np.float32)
        p.z[:] = np.asarray(z, dtype=np.float32)
        p.mass[:] = np.float32(mass) if np.isscalar(mass) else np.asarray(mass, np.float32)
        p.density[:] = np.float32(density) if np.isscalar(density) else np.asarray(density, np.float32)
        p.temperature[:] = np.float32(temperature)
        p.fluid_type[:] = int(fluid_type)
        return p

    def push_particle(self, px, py, pz, mass, density, temperature, fluid_type) -> None:
        """``particle.rs:96-120``."""
        vals = dict(x=px, y=py, z=pz, vx=0.0, vy=0.0, vz=0.0, ax=0.0, ay=0.0, az=0.0,
                    density=density, pressure=0.0, mass=mass, temperature=temperature)
        for k, v in vals.items():
            setattr(self, k, np.append(getattr(self, k), np.float32(v)).astype(np.float32))
        self.fluid_type = np.append(self.fluid_type, np.uint8(int(fluid_type))).astype(np.uint8)

    def __len__(self) -> int:
        return int(self.x.shape[0])

    def is_empty(self) -> bool:
        return len(self) == 0

    def copy(self) -> "ParticleArrays":
        p = ParticleArrays(**{f: getattr(self, f).copy() for f in PARTICLE_FIELDS})
        p.fluid_type = self.fluid_type.copy()
        return p

    def validate(self) -> None:
        n = len(self)
        for f in PARTICLE_FIELDS:
            a = getattr(self, f)
            if a.dtype != np.float32 or a.shape != (n,):
                raise ValueError(f"field {f} must be float32[{n}], got {a.dtype}{a.shape}")
        if self.fluid_type.dtype != np.uint8 or self.fluid_type.shape != (n,):
            raise ValueError("fluid_type must be uint8[n]")


@dataclass
class BoundaryParticles:
    """Static wall particles (``boundary.rs:20-37``); pressure starts at 0."""

    x: np.ndarray = field(default_factory=_f32)
    y: np.ndarray = field(default_factory=_f32)
    z: np.ndarray = field(default_factory=_f32)
    mass: np.ndarray = field(default_factory=_f32)
    nx: np.ndarray = field(default_factory=_f32)
    ny: np.ndarray = field(default_factory=_f32)
    nz: np.ndarray = field(default_factory=_f32)
    pressure: np.ndarray = field(default_factory=_f32)

    @classmethod
    def from_arrays(cls, x, y, z, mass, nx, ny, nz) -> "BoundaryParticles":
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z, mass, nx, ny, nz)]
        n = arrs[0].shape[0]
        return cls(*arrs, pressure=_f32(n))

    def push(self, x, y, z, mass, nx, ny, nz) -> None:
        """``boundary.rs:67-76``."""
        for k, v in dict(x=x, y=y, z=z, mass=mass, nx=nx, ny=ny, nz=nz, pressure=0.0).items():
            setattr(self, k, np.append(getattr(self, k), np.float32(v)).astype(np.float32))

    def __len__(self) -> int:
        return int(self.x.shape[0])

    def is_empty(self) -> bool:
        return len(self) == 0


@dataclass(frozen=True)
class ErrorMetrics:
    """``kernel/src/lib.rs:40-47``."""

    max_density_variation: float
    energy_conservation: float
    mass_conservation: float


@dataclass
class GridSDF:
    """Signed-distance node grid (``orchestrator/src/geometry.rs:11-20``)."""

    origin: tuple
    cell_size: float
    dimensions: tuple
    distances: np.ndarray  # float32[nx*ny*nz], z fastest

    def __post_init__(self):
        self.distances = np.ascontiguousarray(self.distances, dtype=np.float32)
        nx, ny, nz = self.dimensions
        if self.distances.shape != (nx * ny * nz,):
            raise ValueError("distances must have nx*ny*nz entries")


FLUID_WATER, FLUID_AIR, FLUID_MIXED = 0, 1, 2
FACES = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")


@dataclass
class DomainSpec:
    """The ``SimulationConfig`` fields ``setup_domain`` reads
    (``orchestrator/src/config.rs:9-64``): the particle spacing, the domain
    box, the fluid type (``config.rs:66-73``: water, air, or mixed = water
    below the box's middle in y, air above), the initial temperature, and
    which faces are ``Simple(Wall)`` (bit f of ``wall_faces`` for face
    ``FACES[f]``; the default has all six)."""

    particle_spacing: float
    domain_min: tuple
    domain_max: tuple
    fluid_type: int = FLUID_WATER
    initial_temperature: float = 293.15
    wall_faces: int = 0x3F

    @staticmethod
    def faces_mask(walls) -> int:
        """Mask of the faces named in ``walls`` (names from ``FACES``)."""
        return sum(1 << FACES.index(f) for f in walls)
