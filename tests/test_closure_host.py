"""Host logic of the closure pipeline and its tank builders (CPU only)."""
import numpy as np
from scipy.spatial import cKDTree

from ultraballpit_b200 import closure, closure_batch, domain


def test_lattice_tank_tiles_one_lattice():
    """Fluid, walls and sphere sit on one lattice: no fluid particle closer
    than about a spacing to a boundary particle, edge and corner columns
    filled, particle mass rho0 dx^3 / S."""
    dx = 0.004
    sc = domain.tank_with_sphere(dx, domain_max=closure.TANK, center=(0.05, 0.05, 0.06), radius=0.02,
                                 fill_height=closure.FILL, seed=3, hydrostatic=True, geometry="lattice")
    p, b = sc.particles, sc.boundary
    fl = np.stack([p.x, p.y, p.z], 1).astype(np.float64)
    bd = np.stack([b.x, b.y, b.z], 1).astype(np.float64)
    d, _ = cKDTree(bd).query(fl)
    assert d.min() > 0.9 * dx
    s = domain.lattice_kernel_sum(float(sc.h), dx)
    assert abs(s - 1.0095) < 1e-3
    assert abs(float(p.mass[0]) - 1000.0 * dx ** 3 / s) < 1e-9
    # a wall particle in every edge column beside the floor
    for x, y in ((-0.5 * dx, -0.5 * dx), (0.1 + 0.5 * dx, -0.5 * dx)):
        near = (np.abs(bd[:, 0] - x) < 1e-6) & (np.abs(bd[:, 1] - y) < 1e-6)
        assert near.sum() > 0


def test_hydrostatic_compression_of_the_lattice():
    """Without jitter the layers are exact: spacing grows with height and
    stays below dx, and the column shrinks by rho0 g H^2 / (14 B)."""
    dx = 0.004
    sc = domain.tank_with_sphere(dx, domain_max=closure.TANK, center=(0.05, 0.05, -1.0), radius=0.01,
                                 fill_height=closure.FILL, seed=None, hydrostatic=True, geometry="lattice")
    z = np.unique(sc.particles.z.astype(np.float64))
    assert len(z) == round(closure.FILL / dx)
    gaps = np.diff(z)
    assert np.all(gaps < dx) and gaps[0] < gaps[-1]
    b = 1000.0 * sc.speed_of_sound ** 2 / 7.0
    shrink = (closure.FILL - 0.5 * dx) - z[-1]
    top = closure.FILL - 0.5 * dx
    assert abs(shrink - 1000.0 * 9.81 * (closure.FILL * top - 0.5 * top * top) / (7.0 * b)) < 1e-6


def test_config5_instances_in_whole_spacings():
    inst = closure_batch.draw_instances(64, 5)
    assert len(inst) == 64
    for q in inst:
        for dx in (0.004, 0.002):
            for v in q["dims"] + (q["fill"],):
                assert domain._axis_count(0.0, v, dx) == round(v / dx)
        assert 0.01 <= q["radius"] <= 0.04 and 0.0 <= q["speed"] <= 0.5
        c, r = np.asarray(q["center"]), q["radius"]
        assert np.all(c - r > 0) and c[0] + r < q["dims"][0] and c[1] + r < q["dims"][1] and c[2] + r < q["fill"]


def test_targets_units_clamps_and_holdout():
    rng = np.random.default_rng(0)
    raw = np.stack([rng.normal(0, 30, 10000), rng.normal(0, 3, 10000), rng.normal(0, 3, 10000),
                    rng.normal(0, 50, 10000)], 1)
    c = 17.0
    t = closure.to_units(raw, c)
    np.testing.assert_allclose(t[:, 0], raw[:, 0] / (c * c * 1000.0 * closure.DRHO_UNIT), rtol=1e-6)
    np.testing.assert_allclose(t[:, 1:], raw[:, 1:] / closure.G, rtol=1e-6)
    tp = closure.prepare_targets(t)
    assert np.all(np.abs(tp[:, 0]) <= closure.CLAMP_DRHO) and np.all(np.abs(tp[:, 1:]) <= closure.CLAMP_ACC_G)
    assert np.abs(tp[:, 3]).max() == closure.CLAMP_ACC_G  # the wide column is clipped
    own = np.repeat(np.arange(20), 50)
    hold = closure.split_by_tank(own, 0.1, seed=0)
    assert len(np.unique(own[hold])) == 2 and not set(own[hold]) & set(own[~hold])


def test_probes_sit_one_h_from_the_geometry():
    geo = dict(center=(0.05, 0.05, 0.07), radius=0.02)
    h = 0.0052
    sph, walls = closure.probe_points(geo, h)
    ds = np.linalg.norm(sph.astype(np.float64) - np.asarray(geo["center"]), axis=1) - geo["radius"]
    np.testing.assert_allclose(ds, h, atol=1e-6)
    w = walls.astype(np.float64)
    dw = np.minimum.reduce([w[:, 0], 0.1 - w[:, 0], w[:, 1], 0.1 - w[:, 1], w[:, 2]])
    np.testing.assert_allclose(dw, h, atol=1e-6)
    assert np.all(np.linalg.norm(w - np.asarray(geo["center"]), axis=1) - geo["radius"] >= 2 * h - 1e-9)
    assert np.all(w[:, 2] <= closure.FILL - 3 * h)
