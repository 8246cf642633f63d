"""Host-side scenario construction (initial particles, wall particles, analytic SDFs).

Restates the reference orchestrator's setup in vectorised numpy with the same
f32 arithmetic:

* wall boundary particles: ``orchestrator/src/domain.rs:162-348`` (3 layers at
  ``(layer + 0.5) * dx`` outside each wall face, tangential lattice
  ``min + (j + 0.5) * dx`` with ``ceil(extent / dx)`` points per axis);
* geometry boundary particles: ``domain.rs:351-402`` (fluid-lattice points with
  ``0 < sdf < 0.5 dx`` get 3 layers along ``-grad(sdf)``);
* ``GridSDF::sample`` / ``gradient``: ``orchestrator/src/geometry.rs:99-175``;
* smoothing length ``1.3 * dx``: ``orchestrator/src/config.rs:269-271``;
* the dam-break column: ``reference-tests/src/benchmarks.rs:89-109`` (lattice
  block in the domain corner).

The SDFs of the dam-break workloads are analytic (box, sphere), sampled at the
node positions ``origin + i * cell`` that ``GridSDF::sample`` assumes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .particles import BoundaryParticles, FluidType, GridSDF, ParticleArrays

f32 = np.float32
FMAX = np.float32(3.4028235e38)


def smoothing_length(dx: float) -> np.float32:
    """``config.rs:269-271``: ``1.3 * particle_spacing`` in f32."""
    return f32(f32(1.3) * f32(dx))


def particle_mass(dx: float, rest_density: float = 1000.0) -> np.float32:
    """``domain.rs:43-44``: ``rho0 * dx^3`` in f32."""
    dx = f32(dx)
    return f32(f32(rest_density) * f32(f32(dx * dx) * dx))


def _axis_count(lo, hi, dx) -> int:
    return int(np.ceil(f32(f32(hi) - f32(lo)) / f32(dx)))


def _lattice(lo, n, dx) -> np.ndarray:
    """``lo + (i + 0.5) * dx`` for i < n, each op rounded to f32."""
    i = np.arange(n, dtype=np.float32)
    return (f32(lo) + (i + f32(0.5)) * f32(dx)).astype(np.float32)


WALL_FACES = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")


def wall_boundary_particles(domain_min, domain_max, dx, mass,
                            walls=WALL_FACES, n_layers: int = 3) -> BoundaryParticles:
    """``domain.rs:162-348`` in the reference's face and loop order."""
    mn = [f32(v) for v in domain_min]
    mx = [f32(v) for v in domain_max]
    dx = f32(dx)
    out = {k: [] for k in ("x", "y", "z", "nx", "ny", "nz")}
    for face in WALL_FACES:
        if face not in walls:
            continue
        axis = "xyz".index(face[0])
        t0, t1 = [a for a in range(3) if a != axis]
        n0 = _axis_count(mn[t0], mx[t0], dx)
        n1 = _axis_count(mn[t1], mx[t1], dx)
        u = _lattice(mn[t0], n0, dx)
        v = _lattice(mn[t1], n1, dx)
        uu, vv = np.meshgrid(u, v, indexing="ij")
        sign = 1.0 if face.endswith("min") else -1.0
        for layer in range(n_layers):
            off = f32(f32(layer) + f32(0.5)) * dx
            c = f32(mn[axis] - off) if face.endswith("min") else f32(mx[axis] + off)
            pos = [None, None, None]
            pos[axis] = np.full(uu.size, c, dtype=np.float32)
            pos[t0] = uu.ravel()
            pos[t1] = vv.ravel()
            nrm = [np.zeros(uu.size, np.float32) for _ in range(3)]
            nrm[axis][:] = sign
            for k, a in zip(("x", "y", "z"), pos):
                out[k].append(a)
            for k, a in zip(("nx", "ny", "nz"), nrm):
                out[k].append(a)
    cat = {k: (np.concatenate(v) if v else np.zeros(0, np.float32)) for k, v in out.items()}
    n = cat["x"].shape[0]
    return BoundaryParticles.from_arrays(cat["x"], cat["y"], cat["z"],
                                         np.full(n, f32(mass), np.float32),
                                         cat["nx"], cat["ny"], cat["nz"])


def concat_boundary(*parts: BoundaryParticles) -> BoundaryParticles:
    cols = {k: np.concatenate([getattr(p, k) for p in parts]).astype(np.float32)
            for k in ("x", "y", "z", "mass", "nx", "ny", "nz")}
    return BoundaryParticles.from_arrays(**cols)


# ---------------------------------------------------------------------------
# GridSDF (geometry.rs:99-175), vectorised
# ---------------------------------------------------------------------------

def sdf_sample(sdf: GridSDF, pts: np.ndarray) -> np.ndarray:
    """Trilinear sample at points ``pts[..., 3]`` (f32); f32::MAX off-grid."""
    pts = np.asarray(pts, dtype=np.float32)
    o = [f32(v) for v in sdf.origin]
    cs = f32(sdf.cell_size)
    nx, ny, nz = (int(v) for v in sdf.dimensions)
    g = [((pts[..., k] - o[k]) / cs).astype(np.float32) for k in range(3)]
    i0 = [np.floor(gk).astype(np.int64) for gk in g]
    ok = (i0[0] >= 0) & (i0[1] >= 0) & (i0[2] >= 0)
    ok &= (i0[0] + 1 < nx) & (i0[1] + 1 < ny) & (i0[2] + 1 < nz)
    ii = [np.where(ok, a, 0) for a in i0]
    fr = [(g[k] - ii[k].astype(np.float32)).astype(np.float32) for k in range(3)]
    d = sdf.distances

    def at(di, dj, dk):
        return d[(ii[0] + di) * ny * nz + (ii[1] + dj) * nz + (ii[2] + dk)]

    one = f32(1.0)
    fx, fy, fz = fr
    c00 = at(0, 0, 0) * (one - fz) + at(0, 0, 1) * fz
    c01 = at(0, 1, 0) * (one - fz) + at(0, 1, 1) * fz
    c10 = at(1, 0, 0) * (one - fz) + at(1, 0, 1) * fz
    c11 = at(1, 1, 0) * (one - fz) + at(1, 1, 1) * fz
    c0 = c00 * (one - fy) + c01 * fy
    c1 = c10 * (one - fy) + c11 * fy
    val = (c0 * (one - fx) + c1 * fx).astype(np.float32)
    return np.where(ok, val, FMAX).astype(np.float32)


def sdf_gradient(sdf: GridSDF, pts: np.ndarray) -> np.ndarray:
    """Central differences at +-0.5 cell, normalised (geometry.rs:153-175)."""
    pts = np.asarray(pts, dtype=np.float32)
    h = f32(f32(sdf.cell_size) * f32(0.5))
    g = []
    for k in range(3):
        a = pts.copy()
        b = pts.copy()
        a[..., k] = (pts[..., k] + h).astype(np.float32)
        b[..., k] = (pts[..., k] - h).astype(np.float32)
        with np.errstate(over="ignore", invalid="ignore"):
            g.append(((sdf_sample(sdf, a) - sdf_sample(sdf, b)) / f32(f32(2.0) * h)).astype(np.float32))
    with np.errstate(over="ignore", invalid="ignore"):
        mag = np.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]).astype(np.float32)
        good = mag > f32(1e-8)
        out = np.stack([np.where(good, gk / np.where(good, mag, 1), f32(0)) for gk in g], axis=-1)
    return out.astype(np.float32)


def sdf_node_grid(domain_min, domain_max, cell):
    """Node counts ``ceil(extent / cell) + 1`` (geometry.rs:52-54) and positions."""
    dims = tuple(_axis_count(domain_min[k], domain_max[k], cell) + 1 for k in range(3))
    axes = [(f32(domain_min[k]) + np.arange(dims[k], dtype=np.float32) * f32(cell)).astype(np.float32)
            for k in range(3)]
    return dims, axes


def box_sdf(domain_min, domain_max, cell) -> GridSDF:
    """Distance to the nearest wall of the domain box: positive inside."""
    dims, (ax, ay, az) = sdf_node_grid(domain_min, domain_max, cell)
    X, Y, Z = np.meshgrid(ax.astype(np.float64), ay.astype(np.float64), az.astype(np.float64), indexing="ij")
    d = np.minimum.reduce([X - domain_min[0], domain_max[0] - X, Y - domain_min[1],
                           domain_max[1] - Y, Z - domain_min[2], domain_max[2] - Z])
    return GridSDF(tuple(float(v) for v in domain_min), float(f32(cell)), dims,
                   d.astype(np.float32).ravel())


def sphere_sdf(domain_min, domain_max, cell, center, radius) -> GridSDF:
    """Signed distance to a solid sphere: negative inside the solid."""
    dims, (ax, ay, az) = sdf_node_grid(domain_min, domain_max, cell)
    X, Y, Z = np.meshgrid(ax.astype(np.float64), ay.astype(np.float64), az.astype(np.float64), indexing="ij")
    d = np.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Z - center[2]) ** 2) - radius
    return GridSDF(tuple(float(v) for v in domain_min), float(f32(cell)), dims,
                   d.astype(np.float32).ravel())


def merge_sdf(a: GridSDF, b: GridSDF) -> GridSDF:
    """Union of solids: node-wise min of two SDFs on the same grid."""
    assert a.dimensions == b.dimensions and a.cell_size == b.cell_size
    return GridSDF(a.origin, a.cell_size, a.dimensions, np.minimum(a.distances, b.distances))


def lattice_box_walls(domain_min, domain_max, dx, mass, n_layers: int = 3) -> BoundaryParticles:
    """Walls of the domain box on the fluid lattice: per axis the lattice
    ``lo + (i + 0.5) dx`` inside and ``n_layers`` sites beyond each face
    (``lo - (l + 0.5) dx``, ``hi + (l + 0.5) dx``), every combination with a
    coordinate outside the box. Unlike the reference's per-face layers
    (domain.rs:162-348), which span only the box in the tangential
    directions, this fills the edge and corner columns, so a particle in an
    edge or corner sees as much wall mass as one beside a face. Normals
    point from the site to the nearest point of the box."""
    dx = f32(dx)
    axes, inside = [], []
    for k in range(3):
        lo, hi = f32(domain_min[k]), f32(domain_max[k])
        n = _axis_count(lo, hi, dx)
        layers = (np.arange(n_layers, dtype=np.float32) + f32(0.5)) * dx
        a = np.concatenate([(lo - layers[::-1]).astype(np.float32), _lattice(lo, n, dx),
                            (hi + layers).astype(np.float32)])
        axes.append(a)
        inside.append((a > lo) & (a < hi))
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    I = np.meshgrid(*inside, indexing="ij")
    sel = ~(I[0] & I[1] & I[2])
    pts = np.stack([X[sel], Y[sel], Z[sel]], axis=-1).astype(np.float64)
    lo = np.asarray(domain_min, np.float64)
    hi = np.asarray(domain_max, np.float64)
    nrm = np.clip(pts, lo, hi) - pts
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
    pts = pts.astype(np.float32)
    return BoundaryParticles.from_arrays(pts[:, 0], pts[:, 1], pts[:, 2], np.full(len(pts), f32(mass)),
                                         nrm[:, 0], nrm[:, 1], nrm[:, 2])


def lattice_solid_particles(sdf: GridSDF, domain_min, domain_max, dx, mass,
                            n_layers: int = 3) -> BoundaryParticles:
    """Boundary particles at the fluid lattice's own sites (``lo + (i + 0.5)
    dx``) inside the solid, within ``n_layers`` spacings of its surface
    (-n_layers dx <= SDF < 0), normals from the SDF gradient. With the fluid
    seeded at the sites where SDF >= 0, fluid and wall tile one lattice, so
    the summation density starts uniform up to the surface; the reference's
    layers along the inward normal (domain.rs:351-402) crowd together inside
    a body only a few spacings in radius."""
    dx = f32(dx)
    n = [_axis_count(domain_min[k], domain_max[k], dx) for k in range(3)]
    ax = [_lattice(domain_min[k], n[k], dx) for k in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1)
    d = sdf_sample(sdf, pts)
    p = pts[(d < f32(0)) & (d >= -f32(n_layers) * dx)]
    nrm = sdf_gradient(sdf, p) if len(p) else np.zeros((0, 3), np.float32)
    return BoundaryParticles.from_arrays(p[:, 0], p[:, 1], p[:, 2], np.full(len(p), f32(mass)),
                                         nrm[:, 0], nrm[:, 1], nrm[:, 2])


def geometry_boundary_particles(sdf: GridSDF, domain_min, domain_max, dx, mass,
                                n_layers: int = 3) -> BoundaryParticles:
    """``domain.rs:351-402``: 3 layers along the inward normal at lattice points
    within half a spacing outside the surface (i, j, k loop order kept)."""
    dx = f32(dx)
    n = [_axis_count(domain_min[k], domain_max[k], dx) for k in range(3)]
    ax = [_lattice(domain_min[k], n[k], dx) for k in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1)
    d = sdf_sample(sdf, pts)
    sel = (d > f32(0)) & (d < f32(dx * f32(0.5)))
    p = pts[sel]
    nrm = sdf_gradient(sdf, p)
    cols = {k: [] for k in ("x", "y", "z", "nx", "ny", "nz")}
    # interleave layers per lattice point, as the reference pushes them
    offs = [f32(f32(f32(layer) + f32(0.5)) * dx) for layer in range(n_layers)]
    xs = np.stack([(p[:, 0] - nrm[:, 0] * o).astype(np.float32) for o in offs], axis=1).ravel()
    ys = np.stack([(p[:, 1] - nrm[:, 1] * o).astype(np.float32) for o in offs], axis=1).ravel()
    zs = np.stack([(p[:, 2] - nrm[:, 2] * o).astype(np.float32) for o in offs], axis=1).ravel()
    rep = lambda a: np.repeat(a, n_layers).astype(np.float32)
    cols = dict(x=xs, y=ys, z=zs, nx=rep(nrm[:, 0]), ny=rep(nrm[:, 1]), nz=rep(nrm[:, 2]))
    m = np.full(xs.shape[0], f32(mass), np.float32)
    return BoundaryParticles.from_arrays(cols["x"], cols["y"], cols["z"], m,
                                         cols["nx"], cols["ny"], cols["nz"])


# ---------------------------------------------------------------------------
# Scenarios
# ---------------------------------------------------------------------------

@dataclass
class Scenario:
    """Everything ``CpuKernel::new`` (lib.rs:138-148) takes, plus extras."""

    name: str
    particles: ParticleArrays
    boundary: BoundaryParticles
    h: float
    gravity: tuple
    speed_of_sound: float
    cfl_number: float
    viscosity: float
    domain_min: tuple
    domain_max: tuple
    alpha: float = 1.0
    beta: float = 2.0
    sdf: GridSDF | None = None
    extras: dict = field(default_factory=dict)

    def kernel_args(self):
        return (self.particles, self.boundary, self.h, self.gravity, self.speed_of_sound,
                self.cfl_number, self.viscosity, self.domain_min, self.domain_max)

    @property
    def obstacle_sdf(self) -> GridSDF | None:
        """The obstacle's own SDF (the SDF wall mode's ``sdf``: the domain
        box faces are walls of their own), or None without one."""
        return self.extras.get("sphere_sdf")


def dam_break_c0(height: float = 0.2, g: float = 9.81) -> float:
    """``c0 = 10 sqrt(2 g H)`` (19.81 m/s at H = 0.2 m), no auto-tune."""
    return float(f32(10.0 * math.sqrt(2.0 * g * height)))


def block_particles(origin, counts, dx, seed: int | None, jitter: float = 0.01) -> ParticleArrays:
    """Lattice block ``origin + (i + 0.5) dx`` in i (outer), j, k (inner) order,
    jittered by U(-jitter dx, +jitter dx) per coordinate from ``seed``."""
    dx = f32(dx)
    axes = [_lattice(origin[k], counts[k], dx) for k in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1).astype(np.float32)
    if seed is not None and jitter > 0:
        rng = np.random.default_rng(seed)
        pos = (pos.astype(np.float64) + rng.uniform(-jitter * float(dx), jitter * float(dx),
                                                    size=pos.shape)).astype(np.float32)
    return ParticleArrays.from_positions(pos[:, 0], pos[:, 1], pos[:, 2], particle_mass(dx))


def dam_break(dx: float, seed: int = 1234, sphere: bool = False, alpha: float = 0.02,
              block=(0.1, 0.2, 0.1), domain_max=(0.4, 0.2, 0.1), sdf_cell: float = 0.002,
              with_sdf: bool = True) -> Scenario:
    """The 3D dam break: domain [0, 0.4] x [0, 0.2] x [0, 0.1] m, water block
    0.1 x 0.2 x 0.1 m in the corner, g = -9.81 z, c0 = 19.81 m/s, CFL 0.25,
    walls on all six faces. ``sphere`` adds the fixed obstacle of radius
    0.02 m at (0.25, 0.1, 0.03) as geometry boundary particles and merges it
    into the SDF."""
    dmin = (0.0, 0.0, 0.0)
    dmax = tuple(float(v) for v in domain_max)
    dx32 = f32(dx)
    counts = tuple(_axis_count(0.0, block[k], dx32) for k in range(3))
    parts = block_particles(dmin, counts, dx32, seed)
    m = particle_mass(dx32)
    walls = wall_boundary_particles(dmin, dmax, dx32, m)
    sdf = None
    extras = {"block": block, "counts": counts}
    boundary = walls
    if with_sdf or sphere:
        sdf = box_sdf(dmin, dmax, sdf_cell)
    if sphere:
        center, radius = (0.25, 0.1, 0.03), 0.02
        sph = sphere_sdf(dmin, dmax, sdf_cell, center, radius)
        geo = geometry_boundary_particles(sph, dmin, dmax, dx32, m)
        boundary = concat_boundary(walls, geo)
        sdf = merge_sdf(sdf, sph)
        extras.update(sphere_center=center, sphere_radius=radius, sphere_sdf=sph,
                      n_geometry_boundary=len(geo))
    return Scenario(
        name=f"dam_break_dx{dx*1e3:g}mm" + ("_sphere" if sphere else ""),
        particles=parts, boundary=boundary, h=float(smoothing_length(dx32)),
        gravity=(0.0, 0.0, -9.81), speed_of_sound=dam_break_c0(), cfl_number=0.25,
        viscosity=0.0, domain_min=dmin, domain_max=dmax, alpha=alpha, beta=2.0,
        sdf=sdf, extras=extras)


def lattice_kernel_sum(h: float, dx: float) -> float:
    """S = sum over the cubic lattice of W_C2(|x_ijk|, h) dx^3, self included:
    the summation density of an undisturbed lattice of mass rho0 dx^3 is
    S rho0 (1.0096 at h = 1.3 dx)."""
    m = int(math.ceil(2.0 * h / dx)) + 1
    r = np.arange(-m, m + 1, dtype=np.float64) * dx
    X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
    q = np.sqrt(X * X + Y * Y + Z * Z) / h
    w = np.where(q < 2.0, (1.0 - 0.5 * q) ** 4 * (1.0 + 2.0 * q), 0.0)
    return float(21.0 / (16.0 * math.pi * h ** 3) * w.sum() * dx ** 3)


def tank_with_sphere(dx: float, domain_max=(0.12, 0.08, 0.08), center=(0.06, 0.04, 0.035),
                     radius: float = 0.02, fill_height: float | None = None, seed: int = 5,
                     alpha: float = 0.02, sdf_cell: float = 0.002, velocity=(0.0, 0.0, 0.0),
                     hydrostatic: bool = False, solid_gap: float = 0.0,
                     geometry: str = "offset") -> Scenario:
    """A closed tank filled with water up to ``fill_height`` around a fixed
    sphere. Lattice points inside the solid (sphere SDF < 0) are skipped as
    ``place_fluid_particles`` does (domain.rs:127-130); the sphere becomes
    geometry boundary particles (domain.rs:351-402) and is merged into the
    SDF. ``velocity`` is an initial uniform fluid velocity. ``solid_gap``
    (in units of dx) also skips lattice points closer than that to the
    sphere: 0.5 gives the sphere the half-spacing gap the lattice keeps
    from the flat walls. ``geometry`` "offset" builds the boundary particles
    as the reference does; "lattice" puts the box walls and the sphere on the
    fluid lattice's own sites (``lattice_box_walls``,
    ``lattice_solid_particles``) and splits fluid from solid on the bare
    lattice, before jitter and compression.

    ``hydrostatic`` starts the water at rest in its hydrostatic state. The
    particle (and wall) mass is rho0 dx^3 / S with S = sum W(|x_ijk|) dx^3
    over the full lattice (1.0096 at h = 1.3 dx), so the undisturbed
    lattice sums to rho0 instead of S rho0; then, as the summation density
    follows the spacing, the lattice is compressed vertically to the Tait
    density of p = rho0 g (H - z): dz'/dz = rho0 / rho(z) = 1 - p / (7 B)
    to first order, i.e. z' = z - rho0 g (H z - z^2 / 2) / (7 B) with
    B = rho0 c0^2 / 7. Without it the column starts about 3 kPa above its
    hydrostatic pressure, expands and rings for tenths of a second."""
    dmin = (0.0, 0.0, 0.0)
    dmax = tuple(float(v) for v in domain_max)
    dx32 = f32(dx)
    fill = dmax[2] if fill_height is None else fill_height
    counts = (_axis_count(0.0, dmax[0], dx32), _axis_count(0.0, dmax[1], dx32), _axis_count(0.0, fill, dx32))
    sph = sphere_sdf(dmin, dmax, sdf_cell, center, radius)
    parts = block_particles(dmin, counts, dx32, seed)
    c0 = dam_break_c0(fill)
    top = counts[2] * float(dx32)
    kz = 1000.0 * 9.81 / (7.0 * (1000.0 * c0 * c0 / 7.0))

    def zmap(z):  # hydrostatic compression, a constant shift above the fill
        z = np.minimum(z.astype(np.float64), top) + np.maximum(z.astype(np.float64) - top, 0.0)
        zc = np.minimum(z, top)
        return (z - kz * (top * zc - 0.5 * zc * zc)).astype(np.float32)

    if hydrostatic:
        parts.z[:] = zmap(parts.z)
    pts = np.stack([parts.x, parts.y, parts.z], axis=-1)
    if geometry == "lattice":  # fluid and solid split on the bare lattice
        bare = block_particles(dmin, counts, dx32, None)
        pts = np.stack([bare.x, bare.y, bare.z], axis=-1)
    keep = sdf_sample(sph, pts) >= f32(solid_gap * float(dx32))
    m = particle_mass(dx32)
    if hydrostatic:
        m = f32(float(m) / lattice_kernel_sum(float(smoothing_length(dx32)), float(dx32)))
    p = ParticleArrays.from_positions(parts.x[keep], parts.y[keep], parts.z[keep], m)
    p.vx[:], p.vy[:], p.vz[:] = (f32(v) for v in velocity)
    if geometry == "lattice":
        walls = lattice_box_walls(dmin, dmax, dx32, m)
        geo = lattice_solid_particles(sph, dmin, dmax, dx32, m)
    else:
        walls = wall_boundary_particles(dmin, dmax, dx32, m)
        geo = geometry_boundary_particles(sph, dmin, dmax, dx32, m)
    if hydrostatic and geometry == "lattice":  # keep fluid and wall on one lattice
        walls.z[:] = zmap(walls.z)
        geo.z[:] = zmap(geo.z)
    sdf = merge_sdf(box_sdf(dmin, dmax, sdf_cell), sph)
    return Scenario(f"tank_sphere_dx{dx*1e3:g}mm", p, concat_boundary(walls, geo), float(smoothing_length(dx32)),
                    (0.0, 0.0, -9.81), c0, 0.25, 0.0, dmin, dmax, alpha=alpha, sdf=sdf,
                    extras=dict(sphere_center=center, sphere_radius=radius, sphere_sdf=sph,
                                n_geometry_boundary=len(geo), n_wall_boundary=len(walls)))


def two_particles(h: float = 0.05) -> Scenario:
    """``kernel/tests/two_particle.rs:11-24``: two particles h apart on x."""
    p = ParticleArrays.from_positions([0.0, h], [0.0, 0.0], [0.0, 0.0], 0.001)
    return Scenario("two_particles", p, BoundaryParticles(), h, (0.0, 0.0, 0.0), 20.0, 0.3, 1.0,
                    (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))


def hydrostatic_column() -> Scenario:
    """``kernel/tests/hydrostatic.rs:21-78``: 4x4x4 water column on 3 layers."""
    h = f32(0.02)
    spacing = f32(h / f32(1.3))
    mass = f32(f32(1000.0) * spacing * spacing * spacing)
    xs, ys, zs = [], [], []
    for iy in range(4):
        for iz in range(4):
            for ix in range(4):
                xs.append(f32(f32(ix + 0.5) * spacing))
                ys.append(f32(f32(iy + 1.0) * spacing))
                zs.append(f32(f32(iz + 0.5) * spacing))
    p = ParticleArrays.from_positions(xs, ys, zs, mass)
    b = BoundaryParticles()
    bx, by, bz = [], [], []
    for layer in range(3):
        yb = f32(-f32(layer) * spacing)
        for iz in range(-1, 4 + 2):
            for ix in range(-1, 4 + 2):
                bx.append(f32(f32(ix + 0.5) * spacing))
                by.append(yb)
                bz.append(f32(f32(iz + 0.5) * spacing))
    nb = len(bx)
    b = BoundaryParticles.from_arrays(bx, by, bz, np.full(nb, mass), np.zeros(nb), np.ones(nb), np.zeros(nb))
    margin = f32(f32(6.0) * h)
    dmin = (float(-margin),) * 3
    dmax = (float(f32(f32(7) * spacing + margin)), float(f32(f32(14) * spacing + margin)),
            float(f32(f32(7) * spacing + margin)))
    return Scenario("hydrostatic_column", p, b, float(h), (0.0, -9.81, 0.0), 20.0, 0.2, 1.0, dmin, dmax)


def water_box_2mm() -> Scenario:
    """``kernel/tests/gpu_cpu_parity.rs:17-68``: 5x5x5 water box, bottom boundary."""
    spacing = f32(0.002)
    h = f32(f32(1.3) * spacing)
    mass = f32(f32(1000.0) * f32(f32(spacing * spacing) * spacing))
    xs, ys, zs = [], [], []
    x = f32(f32(0.0) + f32(0.5) * spacing)
    while x < f32(0.01):
        y = f32(f32(0.5) * spacing)
        while y < f32(0.01):
            z = f32(f32(0.5) * spacing)
            while z < f32(0.01):
                xs.append(x); ys.append(y); zs.append(z)
                z = f32(z + spacing)
            y = f32(y + spacing)
        x = f32(x + spacing)
    p = ParticleArrays.from_positions(xs, ys, zs, mass)
    bx, bz = [], []
    xb = f32(0.0)
    while xb <= f32(0.01):
        zb = f32(0.0)
        while zb <= f32(0.01):
            bx.append(xb); bz.append(zb)
            zb = f32(zb + spacing)
        xb = f32(xb + spacing)
    nb = len(bx)
    b = BoundaryParticles.from_arrays(bx, np.zeros(nb), bz, np.full(nb, mass), np.zeros(nb),
                                      np.ones(nb), np.zeros(nb))
    return Scenario("water_box_2mm", p, b, float(h), (0.0, -9.81, 0.0), 10.0, 0.4, 0.001,
                    (0.0, 0.0, 0.0), (0.01, 0.01, 0.01))


def batch_boxes(n_instances: int = 256, seed: int = 7, dx: float = 0.002, lo: int = 2000,
                hi: int = 400_000, alpha: float = 0.02, dims_range=(0.05, 0.3),
                fill_range=(0.3, 0.8), draw: str = "stated") -> list:
    """Independent hydrostatic / dam-break boxes for a batch.

    Per instance, drawn from ``seed``: box dims uniform in ``dims_range`` per
    axis and a fill fraction uniform in ``fill_range``; even instances are
    hydrostatic tanks (water fills the bottom ``fill`` of the height), odd
    ones dam breaks (a full-height column over the first ``fill`` of the
    length). Draws whose particle count falls outside [lo, hi] are redrawn
    (the stated ranges alone give about 368k particles per instance at 2 mm,
    far above the 2k-400k the workload names). With ``draw="loguniform"`` a
    target count is drawn log-uniformly in [lo, hi] instead and the drawn box
    is scaled to hold it (box edges may then leave ``dims_range``); that
    matches the workload's stated total of about 20M for 256 instances.
    Walls on all six faces, h = 1.3 dx, c0 = 10 sqrt(2 g H) with H the water
    height."""
    rng = np.random.default_rng(seed)
    out = []
    dx32 = f32(dx)
    q = 0
    while len(out) < n_instances:
        L = rng.uniform(*dims_range, size=3)
        fill = rng.uniform(*fill_range)
        if draw == "loguniform":
            target = math.exp(rng.uniform(math.log(lo), math.log(hi)))
            L = L * (target * dx ** 3 / (fill * L[0] * L[1] * L[2])) ** (1.0 / 3.0)
        dam = (len(out) % 2) == 1
        block = (L[0] * fill, L[1], L[2]) if dam else (L[0], L[1], L[2] * fill)
        counts = tuple(_axis_count(0.0, block[k], dx32) for k in range(3))
        npart = counts[0] * counts[1] * counts[2]
        q += 1
        if not (lo <= npart <= hi):
            continue
        dmax = tuple(float(f32(v)) for v in L)
        parts = block_particles((0.0, 0.0, 0.0), counts, dx32, seed=int(rng.integers(1 << 31)))
        walls = wall_boundary_particles((0.0, 0.0, 0.0), dmax, dx32, particle_mass(dx32))
        height = float(block[2])
        out.append(Scenario(f"box{len(out)}", parts, walls, float(smoothing_length(dx32)),
                            (0.0, 0.0, -9.81), dam_break_c0(height), 0.25, 0.0, (0.0, 0.0, 0.0), dmax,
                            alpha=alpha, extras=dict(kind="dam_break" if dam else "hydrostatic",
                                                     fill=float(fill), dims=tuple(L), draws=q)))
    return out


def size_histogram(scenarios) -> dict:
    """Instance particle counts in log2 bins (the autotuner's cache key)."""
    counts = np.array([len(s.particles) for s in scenarios])
    bins = np.floor(np.log2(np.maximum(counts, 1))).astype(int)
    return {int(b): int(np.sum(bins == b)) for b in np.unique(bins)}
