"""Parity of the CUDA step against the CPU oracle, through the C ABI.

The CUDA step is compared bit for bit with the oracle in pow_mode 1 (the
correctly rounded Tait power it implements) and within 1e-6 relative on
positions with the oracle in pow_mode 0 (libm powf, the reference on Linux).
Grid keys, cell counts/starts, the Morton permutation and neighbour lists
must be identical.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from ultraballpit_b200 import domain
from ultraballpit_b200.kernel import CELL_ORDER_LINEAR, CELL_ORDER_MORTON, CELL_ORDER_ROWS, CudaKernel, SphError
from ultraballpit_b200.particles import BoundaryParticles, ParticleArrays

pytestmark = pytest.mark.gpu
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure", "mass")
POS_RTOL = 1e-6  # positions vs the libm-powf oracle, relative to the domain extent


def make_pair(sc, pow_mode=1, threads=8, **kw):
    args = sc.kernel_args()
    gpu = CudaKernel(*args, alpha=sc.alpha, beta=sc.beta, **kw)
    cpu = orc.OracleKernel(*args, alpha=sc.alpha, beta=sc.beta, tier=1, threads=threads,
                           pow_mode=pow_mode)
    return gpu, cpu


def assert_same(a: ParticleArrays, b: ParticleArrays, fields=FIELDS):
    for f in fields:
        x, y = getattr(a, f), getattr(b, f)
        bad = np.nonzero(~((x == y) | (np.isnan(x) & np.isnan(y))))[0]
        assert bad.size == 0, f"{f}: {bad.size} differ, first id {bad[0]}: {x[bad[0]]!r} vs {y[bad[0]]!r}"
    np.testing.assert_array_equal(a.fluid_type, b.fluid_type)
    np.testing.assert_array_equal(a.temperature, b.temperature)


def small_dam_break(seed=3):
    return domain.dam_break(0.004, seed=seed, block=(0.04, 0.04, 0.04),
                            domain_max=(0.08, 0.04, 0.04), with_sdf=False)


# ---- grid / sort -------------------------------------------------------------

def _grid_vs_oracle(sc, order):
    gpu = CudaKernel(*sc.kernel_args(), cell_order=order)
    g = gpu.read_grid()
    p = sc.particles
    o = orc.grid_build(p.x, p.y, p.z, 2 * sc.h, sc.domain_min, sc.domain_max)
    assert tuple(g["dims"]) == o["dims"]
    np.testing.assert_array_equal(g["cell_linear"], o["cell_idx"])
    np.testing.assert_array_equal(g["morton_key"], o["morton_key"])
    np.testing.assert_array_equal(g["cell_count"], o["counts"])
    if order == CELL_ORDER_LINEAR:
        np.testing.assert_array_equal(g["cell_start"], o["offsets"])
        np.testing.assert_array_equal(g["slot_id"], o["sorted"])
    elif order == CELL_ORDER_ROWS:
        # cells ranked by (Morton code of (cy, cz)) * nx + cx; slots by (rank, id)
        nx, ny, nz = o["dims"]
        lin = np.arange(nx * ny * nz, dtype=np.int64)
        cx, cy, cz = lin % nx, (lin // nx) % ny, lin // (nx * ny)
        spread = lambda v: sum(((v >> b) & 1) << (2 * b) for b in range(21))
        key = (spread(cy) | (spread(cz) << 1)) * nx + cx
        rank_of_lin = np.empty_like(lin)
        rank_of_lin[np.argsort(key, kind="stable")] = lin.copy()  # rank of each linear cell (lin is 0..N-1)
        counts_by_rank = np.zeros(len(lin), np.int64)
        counts_by_rank[rank_of_lin] = o["counts"]
        start_by_rank = np.cumsum(counts_by_rank) - counts_by_rank
        np.testing.assert_array_equal(g["cell_start"], start_by_rank[rank_of_lin].astype(np.uint32))
        prank = rank_of_lin[o["cell_idx"].astype(np.int64)]
        np.testing.assert_array_equal(g["slot_id"], np.lexsort((np.arange(len(prank)), prank)).astype(np.uint32))
    else:
        np.testing.assert_array_equal(g["cell_start"], o["morton_offsets"])
        np.testing.assert_array_equal(g["slot_id"], o["morton_perm"])
    return gpu, o


@pytest.mark.parametrize("order", [CELL_ORDER_MORTON, CELL_ORDER_LINEAR, CELL_ORDER_ROWS])
def test_grid_bit_exact_dam_break(order):
    _grid_vs_oracle(domain.dam_break(0.004, seed=11, with_sdf=False), order)


def _custom(x, y, z, dmin=(0, 0, 0), dmax=(1, 1, 1), h=0.05):
    p = ParticleArrays.from_positions(x, y, z, 1e-3)
    return domain.Scenario("custom", p, BoundaryParticles(), h, (0, 0, -9.81), 20.0, 0.25, 0.0, dmin, dmax)


@pytest.mark.parametrize("order", [CELL_ORDER_MORTON, CELL_ORDER_LINEAR, CELL_ORDER_ROWS])
def test_grid_adversarial(order):
    rng = np.random.default_rng(5)
    cell = np.float32(0.1)
    # on cell faces, outside the domain (clamped), and a crowded cell
    faces = (rng.integers(0, 11, size=(600, 3)).astype(np.float32) * cell).astype(np.float32)
    outside = rng.uniform(-0.5, 1.5, size=(400, 3)).astype(np.float32)
    crowd = (np.float32(0.55) + rng.uniform(-0.01, 0.01, size=(700, 3))).astype(np.float32)
    pts = np.concatenate([faces, outside, crowd])
    sc = _custom(pts[:, 0], pts[:, 1], pts[:, 2])
    gpu, o = _grid_vs_oracle(sc, order)
    for i in (0, 5, 600, 1000, 1500, 1699):
        np.testing.assert_array_equal(gpu.neighbors(i), orc.neighbors(
            sc.particles.x, sc.particles.y, sc.particles.z, sc.h, sc.domain_min, sc.domain_max, i))


def test_grid_all_in_one_cell_and_single_particle():
    pts = np.full((1000, 3), 0.5, np.float32) + np.random.default_rng(1).uniform(
        -0.02, 0.02, size=(1000, 3)).astype(np.float32)
    _grid_vs_oracle(_custom(pts[:, 0], pts[:, 1], pts[:, 2]), CELL_ORDER_MORTON)
    _grid_vs_oracle(_custom([0.5], [0.5], [0.5]), CELL_ORDER_MORTON)


def test_neighbor_lists_reference_order():
    sc = domain.dam_break(0.004, seed=12, with_sdf=False)
    gpu = CudaKernel(*sc.kernel_args())
    p = sc.particles
    for i in np.random.default_rng(0).integers(0, len(p), 64):
        np.testing.assert_array_equal(
            gpu.neighbors(int(i)), orc.neighbors(p.x, p.y, p.z, sc.h, sc.domain_min, sc.domain_max, int(i)))


# ---- one step and short runs, bit for bit ---------------------------------------

@pytest.mark.parametrize("make", [domain.two_particles, domain.hydrostatic_column,
                                  domain.water_box_2mm, small_dam_break])
def test_steps_bit_exact(make):
    sc = make()
    gpu, cpu = make_pair(sc)
    assert_same(gpu.particles(), cpu.particles())
    for s in range(5):
        dt = 1e-4 if sc.name in ("two_particles", "hydrostatic_column") else cpu.compute_timestep(sc.cfl_number)
        gpu.step(dt)
        cpu.step(dt)
        assert_same(gpu.particles(), cpu.particles())
    np.testing.assert_array_equal(gpu.boundary_pressure(), cpu.boundary_pressure())


def test_two_particle_newton3_on_gpu():
    sc = domain.two_particles()
    gpu = CudaKernel(*sc.kernel_args())
    gpu.step(0.0001)
    p = gpu.particles()
    for a in ("ax", "ay", "az"):
        assert abs(getattr(p, a)[0] + getattr(p, a)[1]) < 1e-6


def test_dam_break_100_steps_bit_exact_and_within_tolerance_of_powf():
    """The 4 mm dam break: 31,250 particles, 52,500 wall particles."""
    sc = domain.dam_break(0.004, seed=1234, with_sdf=False)
    gpu, cpu = make_pair(sc, pow_mode=1)
    ref = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, tier=1, threads=8, pow_mode=0)
    for s in range(100):
        dt = cpu.compute_timestep(sc.cfl_number)
        assert gpu.compute_timestep() == dt
        gpu.step(dt)
        cpu.step(dt)
        ref.step(dt)
    g, c, r = gpu.particles(), cpu.particles(), ref.particles()
    assert_same(g, c)
    np.testing.assert_array_equal(gpu.boundary_pressure(), cpu.boundary_pressure())
    extent = max(b - a for a, b in zip(sc.domain_min, sc.domain_max))
    for f in ("x", "y", "z"):
        err = np.max(np.abs(getattr(g, f).astype(np.float64) - getattr(r, f)))
        assert err <= POS_RTOL * extent, (f, err)
    em_g, em_c = gpu.error_metrics(), cpu.error_metrics()
    assert em_g.max_density_variation == em_c.max_density_variation
    assert abs(em_g.energy_conservation - em_c.energy_conservation) <= 1e-6 * max(1e-3, em_c.energy_conservation)
    assert abs(em_g.mass_conservation - em_c.mass_conservation) <= 1e-9


def test_step_auto_matches_host_loop():
    sc = small_dam_break(seed=9)
    a = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    b = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    for _ in range(20):
        b.step(b.compute_timestep())
    dt_last = a.step_auto(20)
    assert_same(a.particles(), b.particles())
    assert dt_last > 0


def test_checkpoint_restore_matches_oracle():
    sc = small_dam_break(seed=4)
    gpu, cpu = make_pair(sc)
    for k in (gpu, cpu):
        k.step(1e-4)
        assert k.save_checkpoint()
        k.step(2e-4)
        k.step(2e-4)
        assert k.restore_checkpoint()
        assert not k.restore_checkpoint()
        k.step(1e-4)  # steps on the stale grid, as the reference does
    assert_same(gpu.particles(), cpu.particles())


def test_cell_orders_give_identical_physics():
    """Morton, linear and row orders (the latter two scan a row's cells as one
    range) give the same steps bit for bit, also against the oracle."""
    sc = small_dam_break(seed=6)
    ks = [CudaKernel(*sc.kernel_args(), alpha=sc.alpha, cell_order=o)
          for o in (CELL_ORDER_MORTON, CELL_ORDER_LINEAR, CELL_ORDER_ROWS)]
    cpu = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=1, threads=8, pow_mode=1)
    for _ in range(10):
        dt = ks[0].compute_timestep()
        for k in ks:
            k.step(dt)
        cpu.step(dt)
    for k in ks[1:]:
        assert_same(ks[0].particles(), k.particles())
    assert_same(ks[2].particles(), cpu.particles())
    with pytest.raises(SphError):
        CudaKernel(*sc.kernel_args(), alpha=sc.alpha, cell_order=3)


def test_profiled_step_equals_graph_step():
    sc = small_dam_break(seed=8)
    a = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    b = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    for _ in range(3):
        prof = a.step_profiled(1e-4)
        b.step(1e-4)
        assert prof["total_us"] > 0
    assert_same(a.particles(), b.particles())


def test_empty_and_no_boundary():
    p = ParticleArrays.empty(0)
    k = CudaKernel(p, None, 0.01, (0, 0, -9.81), 20.0, 0.25, 0.0, (0, 0, 0), (1, 1, 1))
    k.step(1e-4)
    assert k.particle_count() == 0
    assert len(k.particles()) == 0


def test_invalid_arguments_raise():
    sc = domain.two_particles()
    with pytest.raises(SphError):
        CudaKernel(sc.particles, None, -1.0, (0, 0, 0), 20.0, 0.3, 1.0, (-1, -1, -1), (1, 1, 1))
    k = CudaKernel(*sc.kernel_args())
    with pytest.raises(SphError):
        k.step(float("nan"))
    assert not k.restore_checkpoint()


def test_health_counts_nonfinite():
    sc = domain.two_particles()
    p = sc.particles.copy()
    p.vx[0] = np.float32("inf")
    k = CudaKernel(p, None, sc.h, sc.gravity, sc.speed_of_sound, sc.cfl_number, sc.viscosity,
                   sc.domain_min, sc.domain_max)
    assert k.health() == 1


# ---- the 1 mm dam break with the sphere: 2,000,000 particles ----------------------

def test_dam_break_sphere_2m_particles_one_step_bit_exact_and_invariants():
    """The 1 mm dam break with the sphere: 2,000,000 particles."""
    sc = domain.dam_break(0.001, seed=2024, sphere=True)
    assert len(sc.particles) == 2_000_000
    gpu, cpu = make_pair(sc, threads=16)
    g = gpu.read_grid()
    assert int(g["cell_count"].sum()) == len(sc.particles)
    assert np.array_equal(np.sort(g["slot_id"]), np.arange(len(sc.particles), dtype=np.uint32))
    dt = cpu.compute_timestep(sc.cfl_number)
    assert gpu.compute_timestep() == dt
    gpu.step(dt)
    cpu.step(dt)
    assert_same(gpu.particles(), cpu.particles())
    np.testing.assert_array_equal(gpu.boundary_pressure(), cpu.boundary_pressure())
    # size-independent invariants over further steps
    m0 = gpu.particles().mass.copy()
    dt_last = gpu.step_auto(20)
    p = gpu.particles()
    assert dt_last > 0 and gpu.health() == 0
    np.testing.assert_array_equal(p.mass, m0)
    for k, f in enumerate(("x", "y", "z")):
        v = getattr(p, f)
        assert v.min() >= sc.domain_min[k] and v.max() <= sc.domain_max[k]
    assert gpu.error_metrics().mass_conservation == 0.0


# ---- SDF wall mode -------------------------------------------------------------------

def test_sdf_mode_bit_exact_with_sphere():
    from ultraballpit_b200.kernel import BOUNDARY_SDF
    sc = domain.dam_break(0.004, seed=31, sphere=True)
    args = sc.kernel_args()
    gpu = CudaKernel(*args, alpha=sc.alpha, boundary_mode=BOUNDARY_SDF, sdf=sc.obstacle_sdf)
    cpu = orc.OracleKernel(*args, alpha=sc.alpha, tier=1, threads=8, pow_mode=1, boundary_mode=1,
                           sdf=sc.obstacle_sdf)
    for _ in range(20):
        dt = cpu.compute_timestep(sc.cfl_number)
        assert gpu.compute_timestep() == dt
        gpu.step(dt)
        cpu.step(dt)
    assert_same(gpu.particles(), cpu.particles())


# ---- force extraction on the sphere of the 1 mm dam break ----------------------

def test_surface_and_body_forces_on_sphere():
    sc = domain.tank_with_sphere(0.004, seed=41, velocity=(0.3, 0.0, 0.0))
    sph = sc.extras["sphere_sdf"]
    nb_geo = sc.extras["n_geometry_boundary"]
    first = len(sc.boundary) - nb_geo
    gpu, cpu = make_pair(sc)
    gpu.set_geometry_sdf(sph)
    for _ in range(10):
        dt = cpu.compute_timestep(sc.cfl_number)
        gpu.step(dt)
        cpu.step(dt)
    assert_same(gpu.particles(), cpu.particles())
    g = gpu.surface_forces()
    assert g["active_nodes"] > 0
    c = cpu.surface_forces(sph)
    assert g["nodes"] == c["nodes"] > 0
    np.testing.assert_array_equal(g["force_f32"], c["force_f32"])
    np.testing.assert_array_equal(g["moment_f32"], c["moment_f32"])
    np.testing.assert_allclose(g["force"], c["force"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(g["moment"], c["moment"], rtol=1e-12, atol=1e-12)
    gb, cb = gpu.body_force(first, nb_geo), cpu.body_force(first, nb_geo)
    for key in gb:
        np.testing.assert_allclose(gb[key], cb[key], rtol=1e-9, atol=1e-15, err_msg=key)


def test_scale_velocities_scales_the_state_the_next_step_starts_from():
    sc = domain.dam_break(0.004, seed=7, block=(0.04, 0.04, 0.04), domain_max=(0.08, 0.04, 0.04), with_sdf=False)
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    for _ in range(5):
        k.step(k.compute_timestep())
    p0 = k.particles()
    k.scale_velocities(2.0)
    p1 = k.particles()
    for f in ("vx", "vy", "vz"):
        np.testing.assert_array_equal(getattr(p1, f), getattr(p0, f) * np.float32(2.0))
    np.testing.assert_array_equal(p1.x, p0.x)
    k.scale_velocities(0.0)
    p2 = k.particles()
    assert not np.any(p2.vx) and not np.any(p2.vy) and not np.any(p2.vz)
    k.step(k.compute_timestep())
    assert k.health() == 0
    k.close()


def test_sdf_mode_tank_at_rest_stays_quiet_at_edges_and_corners():
    """A closed tank at rest in SDF wall mode: the box faces' slabs, edges and
    corners, and the energy-consistent wall force, keep the water near the
    edges and corners as quiet as the rest (no relaxation first)."""
    from ultraballpit_b200 import closure
    from ultraballpit_b200.kernel import BOUNDARY_SDF
    sc = domain.tank_with_sphere(0.004, domain_max=closure.TANK, center=(0.05, 0.05, -1.0), radius=0.01,
                                 fill_height=closure.FILL, seed=3, hydrostatic=True, geometry="lattice")
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, boundary_mode=BOUNDARY_SDF)
    for _ in range(600):
        k.step(5e-5)
    assert k.health() == 0
    p = k.particles()
    pos = np.stack([p.x, p.y, p.z], 1).astype(np.float64)
    v = np.sqrt(p.vx.astype(np.float64) ** 2 + p.vy ** 2 + p.vz ** 2)
    dw = np.sort(np.stack([pos[:, 0], 0.1 - pos[:, 0], pos[:, 1], 0.1 - pos[:, 1], pos[:, 2]], 1), 1)
    h = sc.h
    for name, m in (("wall", (dw[:, 0] < 2 * h) & (dw[:, 1] >= 2 * h)),
                    ("edge", (dw[:, 1] < 2 * h) & (dw[:, 2] >= 2 * h)), ("corner", dw[:, 2] < 2 * h)):
        assert v[m].mean() < 0.12, (name, v[m].mean())
    assert p.z.max() < closure.FILL + 0.01
    k.close()


def test_device_capacity_bounds_are_reported_not_exceeded():
    """The kernels' own bounds end in an error status, never in an access
    past a buffer: more than 4096 particles in one cell (the id ranking of
    the sort) fails the creation, and a boundary particle with more than 256
    fluid particles in support (the Adami term buffer) fails the next call
    that reads the device flags."""
    h = 0.01
    n = 4097
    p = ParticleArrays.from_positions(np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5), 1e-6)
    with pytest.raises(SphError) as e:
        CudaKernel(p, None, h, (0, 0, -9.81), 20.0, 0.25, 0.0, (0, 0, 0), (1, 1, 1))
    assert e.value.status == 6
    rng = np.random.default_rng(3)
    q = rng.uniform(0.497, 0.503, size=(300, 3)).astype(np.float32)
    p = ParticleArrays.from_positions(q[:, 0], q[:, 1], q[:, 2], 1e-6)
    b = BoundaryParticles.from_arrays([0.5], [0.5], [0.49], [1e-6], [0.0], [0.0], [1.0])
    k = CudaKernel(p, b, h, (0, 0, -9.81), 20.0, 0.25, 0.0, (0, 0, 0), (1, 1, 1))
    k.step(1e-6)
    with pytest.raises(SphError) as e:
        k.compute_timestep()
    assert e.value.status == 6
    k.close()


def test_dense_block_takes_the_per_thread_scans_bit_exact(monkeypatch):
    """A fluid block packed so densely (spacing 0.45 h, about 88 particles
    per cell) that the warp scans' masks cannot hold a neighbourhood: many
    fluid particles' 27 cells hold up to some 1,600 candidates (the density
    kernel's warp scan hands them to its per-thread scan) and up to ~360
    neighbours (past the stored list's 128: density, forces and XSPH visit
    the cells again), and the boundary plane under it sees over 1,024
    candidates per cell group (the cell-wise Adami pass takes its
    per-particle search) with under 256 terms each. The warp-cooperative
    forms are forced (the block is below the sizes at which the library
    picks them). Three steps against the oracle, bit for bit, with the
    boundary pressures."""
    monkeypatch.setenv("SPH_WARP_SCAN_MIN", "0")
    monkeypatch.setenv("SPH_ADAMI_CELLS_MIN", "0")
    h, s = 0.01, 0.0045
    g = (np.arange(12, dtype=np.float32) * np.float32(s) + np.float32(0.03)).astype(np.float32)
    x, y, z = (a.ravel() for a in np.meshgrid(g, g, g + np.float32(0.0045), indexing="ij"))
    p = ParticleArrays.from_positions(x, y, z, np.float32(1000.0 * s ** 3))
    bg = (np.arange(14, dtype=np.float32) * np.float32(s) + np.float32(0.03 - s)).astype(np.float32)
    bx, by = (a.ravel() for a in np.meshgrid(bg, bg, indexing="ij"))
    nbp = bx.size
    b = BoundaryParticles.from_arrays(bx, by, np.full(nbp, 0.03, np.float32), np.full(nbp, 1000.0 * s ** 3),
                                      np.zeros(nbp), np.zeros(nbp), np.ones(nbp))
    sc = domain.Scenario("dense_block", p, b, h, (0, 0, -9.81), 20.0, 0.25, 0.0, (0, 0, 0), (0.12, 0.12, 0.12))
    gpu, cpu = make_pair(sc)
    for _ in range(3):
        gpu.step(1e-5)
        cpu.step(1e-5)
        assert_same(gpu.particles(), cpu.particles())
        np.testing.assert_array_equal(gpu.boundary_pressure(), cpu.boundary_pressure())
    assert np.count_nonzero(gpu.boundary_pressure()) > 0
    gpu.close()
