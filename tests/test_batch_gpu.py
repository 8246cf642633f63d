"""Batches of independent simulations (one launch per stage for all of them).

Every instance of a batch must evolve bit for bit like the same simulation
run alone through sph_create, with its own device dt; launch shapes chosen
by the autotuner must not change any result."""
import numpy as np
import pytest

from ultraballpit_b200 import domain
from ultraballpit_b200.kernel import CudaBatch, CudaKernel

pytestmark = pytest.mark.gpu
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure", "mass")


def small_batch(n=6, seed=3):
    return domain.batch_boxes(n, seed=seed, dx=0.004, lo=200, hi=20000, dims_range=(0.03, 0.09))


def _same(a, b):
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


def test_batch_instances_match_single_runs():
    scs = small_batch()
    batch = CudaBatch(scs)
    singles = [CudaKernel(*sc.kernel_args(), alpha=sc.alpha) for sc in scs]
    np.testing.assert_array_equal(batch.timesteps(),
                                  np.array([k.compute_timestep() for k in singles], np.float32))
    batch.step_auto(15, want_dt=False)
    for k in singles:
        k.step_auto(15, want_dt=False)
    np.testing.assert_array_equal(batch.timesteps(),
                                  np.array([k.compute_timestep() for k in singles], np.float32))
    for q, k in enumerate(singles):
        _same(batch.instance(q), k.particles())


def test_batch_host_dt_and_launch_shapes():
    scs = small_batch(4, seed=8)
    a = CudaBatch(scs)
    b = CudaBatch(scs)
    b.set_launch(64, 512, 128)
    for _ in range(5):
        a.step(1e-4)
        b.step(1e-4)
    _same(a.particles(), b.particles())


def test_autotune_returns_valid_shapes_and_caches():
    scs = small_batch(4, seed=9)
    k = CudaBatch(scs)
    best = k.autotune(2)
    assert all(v in (64, 128, 256, 512) for v in best.values())
    assert k.launch() == best
    k2 = CudaBatch(scs)
    assert k2.autotune(2) == best  # cache hit: same histogram, same device


def test_batch_sdf_mode_matches_single_runs():
    from ultraballpit_b200 import closure
    from ultraballpit_b200.kernel import BOUNDARY_SDF
    scs = [closure.tank_pair(s, dx_coarse=0.008)[0] for s in (21, 22, 23)]
    batch = CudaBatch(scs, boundary_mode=BOUNDARY_SDF)
    singles = [CudaKernel(*sc.kernel_args(), alpha=sc.alpha, boundary_mode=BOUNDARY_SDF, sdf=sc.obstacle_sdf)
               for sc in scs]
    batch.step_auto(10, want_dt=False)
    for k in singles:
        k.step_auto(10, want_dt=False)
    for q, k in enumerate(singles):
        _same(batch.instance(q), k.particles())


def test_batch_closure_with_per_instance_dt_matches_single_runs():
    """Closure mode 2 on a batch stepped with one dt per instance
    (sph_batch_step) == each instance alone with its own dt, bit for bit."""
    from ultraballpit_b200 import closure
    scs = [closure.tank_pair(s)[0] for s in (3, 4)]
    w = closure.ClosureNet(seed=9).params()
    dts = np.array([5e-5, 4e-5], np.float32)
    b = CudaBatch(scs)
    b.set_feature_sdfs([sc.sdf for sc in scs])
    b.set_closure(2, w)
    for _ in range(5):
        b.step_each(dts)
    for q, sc in enumerate(scs):
        k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
        k.set_feature_sdf(sc.sdf)
        k.set_closure(2, w)
        for _ in range(5):
            k.step(float(dts[q]))
        got, ref = b.instance(q), k.particles()
        for f in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure"):
            np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=f"instance {q} {f}")
        k.close()
    b.close()
