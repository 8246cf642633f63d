"""setup_domain (orchestrator domain.rs:36-402): the literal restatement in
the oracle against the reference's own test scenarios and hand-computed
lattices, and against the package's vectorised builders; on the GPU,
``sph_setup_domain`` against the oracle bit for bit (host and device output
arrays, face subsets, ragged boxes, a grid smaller than the box, a sphere
obstacle at two million lattice points)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as orc
from ultraballpit_b200 import domain
from ultraballpit_b200.particles import (BOUNDARY_FIELDS, FLUID_AIR, FLUID_MIXED, FLUID_WATER, PARTICLE_FIELDS,
                                         DomainSpec, GridSDF)

f32 = np.float32


def _flat_sdf(dims, value=1.0, cell=0.005, origin=(0.0, 0.0, 0.0)):
    return GridSDF(origin, cell, dims, np.full(int(np.prod(dims)), value, np.float32))


def _sphere_case(dx, dmax=(0.12, 0.08, 0.08), center=(0.06, 0.04, 0.035), radius=0.012):
    dmin = (0.0, 0.0, 0.0)
    sdf = domain.sphere_sdf(dmin, dmax, dx, center, radius)
    return DomainSpec(dx, dmin, dmax), sdf


def _cases():
    """(name, spec, sdf) of the parity cases."""
    out = [("reference_basic", DomainSpec(0.005, (0, 0, 0), (0.01, 0.01, 0.01)), _flat_sdf((3, 3, 3))),
           ("reference_mixed", DomainSpec(0.005, (0, 0, 0), (0.01, 0.02, 0.01), FLUID_MIXED),
            _flat_sdf((3, 5, 3)))]
    spec, sdf = _sphere_case(0.002)
    out.append(("sphere_2mm", spec, sdf))
    out.append(("sphere_2mm_air_open_top", DomainSpec(0.002, spec.domain_min, spec.domain_max, FLUID_AIR, 300.0,
                                                      DomainSpec.faces_mask(("x_min", "x_max", "y_min", "y_max",
                                                                             "z_min"))), sdf))
    # a box that is no whole number of spacings, offset from the origin: the
    # last lattice layer of each axis lies outside and is skipped; the SDF grid
    # covers only part of the box (f32::MAX beyond it counts as outside)
    lo, hi = (-0.0113, 0.0021, 0.0), (0.0291, 0.0317, 0.0253)
    small = domain.sphere_sdf(lo, (0.01, 0.02, 0.02), 0.0015, (0.0, 0.01, 0.01), 0.006)
    out.append(("ragged_partial_grid", DomainSpec(0.0017, lo, hi, FLUID_MIXED, 280.0, 0b101101), small))
    out.append(("no_walls", DomainSpec(0.002, spec.domain_min, spec.domain_max, FLUID_WATER, 293.15, 0), sdf))
    return out


def test_oracle_reference_basic_scenario():
    """domain.rs:879-922 (test_setup_domain_basic), with the values spelled out:
    a 2 x 2 x 2 lattice at (i + 0.5) * 5 mm and 6 walls x 3 layers x 4."""
    spec = DomainSpec(0.005, (0.0, 0.0, 0.0), (0.01, 0.01, 0.01))
    p, b = orc.setup_domain(spec, _flat_sdf((3, 3, 3)))
    assert len(p) == 8 and len(b) == 72
    c = [f32(f32(f32(i) + f32(0.5)) * f32(0.005)) for i in range(2)]
    want = [(x, y, z) for x in c for y in c for z in c]           # x outermost, z innermost
    np.testing.assert_array_equal(np.stack([p.x, p.y, p.z], 1), np.asarray(want, np.float32))
    m = f32(f32(1000.0) * f32(f32(0.005) * f32(f32(0.005) * f32(0.005))))
    assert np.all(p.mass == m) and np.all(p.density == f32(1000.0)) and np.all(p.fluid_type == 0)
    assert np.all(p.temperature == f32(293.15))
    for f in ("vx", "vy", "vz", "ax", "ay", "az", "pressure"):
        assert not getattr(p, f).any()
    # x_min first: layer 0 at -0.5 dx with normal +x, y outer, z inner
    assert (b.x[0], b.y[0], b.z[0], b.nx[0]) == (f32(-0.0025), c[0], c[0], f32(1.0))
    assert (b.y[1], b.z[1]) == (c[0], c[1])
    assert b.x[4] == f32(0.0) - f32(f32(1.5) * f32(0.005))
    assert np.all(b.mass == m)
    np.testing.assert_array_equal(b.nz[60:72], np.full(12, -1.0, np.float32))   # z_max last


def test_oracle_reference_mixed_scenario():
    """domain.rs:924-958: water below the box's middle in y, air above."""
    spec = DomainSpec(0.005, (0.0, 0.0, 0.0), (0.01, 0.02, 0.01), FLUID_MIXED)
    p, b = orc.setup_domain(spec, _flat_sdf((3, 5, 3)))
    water = p.y < f32(0.01)
    assert water.any() and (~water).any()
    np.testing.assert_array_equal(p.fluid_type, np.where(water, 0, 1).astype(np.uint8))
    vol = f32(f32(0.005) * f32(f32(0.005) * f32(0.005)))
    np.testing.assert_array_equal(p.mass, np.where(water, f32(1000.0) * vol, f32(1.2) * vol).astype(np.float32))
    np.testing.assert_array_equal(p.density, np.where(water, f32(1000.0), f32(1.2)).astype(np.float32))
    assert np.all(b.mass == f32(1000.0) * vol)                     # mixed: water mass on the walls


def test_oracle_matches_vectorised_builders():
    """The literal loops against the package's numpy restatements of the wall
    and geometry layers (written independently, same reference lines)."""
    spec, sdf = _sphere_case(0.002)
    p, b = orc.setup_domain(spec, sdf)
    m = domain.particle_mass(0.002)
    walls = domain.wall_boundary_particles(spec.domain_min, spec.domain_max, 0.002, m)
    geo = domain.geometry_boundary_particles(sdf, spec.domain_min, spec.domain_max, 0.002, m)
    want = domain.concat_boundary(walls, geo)
    assert len(geo) > 0
    for f in BOUNDARY_FIELDS:
        np.testing.assert_array_equal(getattr(b, f), getattr(want, f), err_msg=f)
    # fluid: every lattice point in the box and outside the sphere
    inside = (np.sqrt((p.x.astype(np.float64) - 0.06) ** 2 + (p.y - 0.04) ** 2 + (p.z - 0.035) ** 2) < 0.012 - 0.002)
    assert not inside.any()
    in_box = 1
    for a in range(3):
        n = domain._axis_count(spec.domain_min[a], spec.domain_max[a], 0.002)
        in_box *= int(np.count_nonzero(domain._lattice(spec.domain_min[a], n, 0.002) <= f32(spec.domain_max[a])))
    removed, ball = in_box - len(p), 4.0 / 3.0 * np.pi * (0.012 / 0.002) ** 3
    assert 0.9 * ball < removed < 1.1 * ball


def test_oracle_face_mask():
    spec = DomainSpec(0.005, (0.0, 0.0, 0.0), (0.01, 0.01, 0.01), wall_faces=DomainSpec.faces_mask(["y_max"]))
    _, b = orc.setup_domain(spec, _flat_sdf((3, 3, 3)))
    assert len(b) == 12 and np.all(b.ny == -1.0) and np.all(b.y > f32(0.01))


# ---------------------------------------------------------------------------
def _same(a, b, fields):
    for f in fields:
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(6))
def test_device_setup_matches_oracle(case):
    from ultraballpit_b200.kernel import setup_domain
    name, spec, sdf = _cases()[case]
    p, b = setup_domain(spec, sdf)
    q, c = orc.setup_domain(spec, sdf)
    assert len(p) == len(q) and len(b) == len(c), name
    _same(p, q, PARTICLE_FIELDS + ("fluid_type",))
    _same(b, c, BOUNDARY_FIELDS)


@pytest.mark.gpu
def test_device_setup_two_million_lattice_points():
    """The default bench geometry's scale: 200 x 100 x 100 lattice points at
    1 mm around a sphere, bit for bit."""
    from ultraballpit_b200.kernel import setup_domain
    spec, sdf = _sphere_case(0.001, dmax=(0.2, 0.1, 0.1), center=(0.1, 0.05, 0.05), radius=0.02)
    p, b = setup_domain(spec, sdf)
    q, c = orc.setup_domain(spec, sdf)
    assert len(p) > 1_900_000 and len(c) > 3 * 60_000
    _same(p, q, PARTICLE_FIELDS + ("fluid_type",))
    _same(b, c, BOUNDARY_FIELDS)


@pytest.mark.gpu
def test_device_outputs_and_capacity():
    """Output arrays in device memory give the same particles as host arrays;
    a capacity below the count is refused."""
    import torch
    from ultraballpit_b200 import kernel as K
    name, spec, sdf = _cases()[4]
    p, b = K.setup_domain(spec, sdf)
    L = K.load_library()
    s = K.SphDomainSpec(spec.particle_spacing, (C.c_float * 3)(*spec.domain_min), (C.c_float * 3)(*spec.domain_max),
                        spec.fluid_type, spec.initial_temperature, spec.wall_faces)
    keep = []
    sv = K.CudaKernel._sdf_view(sdf, keep)
    n, nb = len(p), len(b)
    dev = {f: torch.empty(n, dtype=torch.float32, device="cuda") for f in PARTICLE_FIELDS}
    ft = torch.empty(n, dtype=torch.uint8, device="cuda")
    bdev = {f: torch.empty(nb, dtype=torch.float32, device="cuda") for f in BOUNDARY_FIELDS}
    fp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float))
    pm = K.SphParticlesMut(n, *[fp(dev[f]) for f in PARTICLE_FIELDS], C.cast(C.c_void_p(ft.data_ptr()),
                                                                            C.POINTER(C.c_uint8)))
    bm = K.SphBoundaryMut(nb, *[fp(bdev[f]) for f in BOUNDARY_FIELDS])
    nf_, nb_ = C.c_size_t(), C.c_size_t()
    assert L.sph_setup_domain(0, C.byref(s), C.byref(sv), C.byref(pm), C.byref(bm), C.byref(nf_), C.byref(nb_)) == 0
    torch.cuda.synchronize()
    for f in PARTICLE_FIELDS:
        np.testing.assert_array_equal(dev[f].cpu().numpy(), getattr(p, f), err_msg=f)
    np.testing.assert_array_equal(ft.cpu().numpy(), p.fluid_type)
    for f in BOUNDARY_FIELDS:
        np.testing.assert_array_equal(bdev[f].cpu().numpy(), getattr(b, f), err_msg=f)
    small = K.SphBoundaryMut(nb - 1, *[fp(bdev[f]) for f in BOUNDARY_FIELDS])
    assert L.sph_setup_domain(0, C.byref(s), C.byref(sv), None, C.byref(small), C.byref(nf_),
                              C.byref(nb_)) == 6  # SPH_ERR_CAPACITY
    assert (nf_.value, nb_.value) == (n, nb)
