"""Long runs of the reference's validation benchmarks on the CUDA path.

Three kinds of evidence, on the loop the reference's harness runs
(``reference-tests/src/benchmarks.rs``; ``ultraballpit_b200/validation.py``):

* bit-exact against the oracle over the whole run: the SHA-256 of the final
  state equals the oracle's (``tests/golden/validation_runs.json``, made by
  ``tests/golden/make_validation.py``): T086 to t = 0.1 s (about 1,960
  steps), T087 to t = 1 s (38,500 steps), the 31,250-particle 3D dam break
  for 1000 steps;
* the reference's own published outputs (``tests/golden/
  reference_benchmarks.json``, from ``specs/001-sph-fluid-sim/
  benchmark-results.md``): that table predates the reference's delta-SPH and
  XSPH stages (its optimisation record O-009/O-010 added them afterwards and
  quotes the table's 9-22 % hydrostatic error as the state before them), so
  the CUDA step with those two stages off must reproduce the printed front
  Z*(T*) to the table's three decimals;
* statistics against the oracle with glibc ``powf`` (the reference on
  Linux), which is not correctly rounded: those runs decorrelate particle by
  particle, so the comparison is on the front position and the band
  pressures, with the tolerances stated below.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from ultraballpit_b200 import domain, validation as V
from ultraballpit_b200.kernel import CudaKernel, setup_domain

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
STATE_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "density", "pressure")


def _golden(name):
    with open(os.path.join(HERE, "golden", name)) as f:
        return json.load(f)


RUNS = _golden("validation_runs.json")
PUBLISHED = _golden("reference_benchmarks.json")


def digest(p) -> str:
    h = hashlib.sha256()
    for f in STATE_FIELDS:
        h.update(np.ascontiguousarray(getattr(p, f), np.float32).tobytes())
    return h.hexdigest()


def cuda(sc, flags):
    return CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, flags=flags)


@pytest.fixture(scope="module")
def dam2d():
    return V.dam_break_2d(setup_domain)


@pytest.mark.parametrize("flags", [0xF, 0xC])
def test_dam_break_2d_bit_exact_with_the_oracle(dam2d, flags):
    sc, a = dam2d
    ref = RUNS["dam_break_2d"]
    assert (len(sc.particles), len(sc.boundary)) == (ref["particles"], ref["boundary"]) == (156, 7950)
    k = cuda(sc, flags)
    run = V.run_to_time(k, V.DAM_BREAK_2D["max_time"], 0.01, stop_time=0.1)
    want = ref[f"flags{flags:x}_pow1"]
    assert run.steps == want["steps"]
    assert digest(k.particles()) == want["digest"]
    front = np.asarray(V.front_positions(run, a))
    np.testing.assert_array_equal(front, np.asarray(want["front"]))
    # glibc powf: the same front to 1e-3 of Z* at every snapshot up to T* = 3.5
    loose = np.asarray(ref[f"flags{flags:x}_pow0"]["front"])
    np.testing.assert_allclose(front[:, 1], loose[:, 1], atol=1e-3)
    k.close()


def test_dam_break_2d_reproduces_the_published_front(dam2d):
    """The reference's printed Z*_sim (3 decimals) at its 8 values of T*,
    from the CUDA step without delta-SPH and XSPH."""
    sc, a = dam2d
    pub = PUBLISHED["dam_break_2d"]
    k = cuda(sc, 0xC)
    run = V.run_to_time(k, V.DAM_BREAK_2D["max_time"], 0.01, stop_time=0.1)
    got = np.asarray(V.front_positions(run, a))
    assert got.shape == (8, 2)
    np.testing.assert_allclose(got[:, 0], pub["t_star"], atol=5e-3)      # printed with 2 decimals
    np.testing.assert_allclose(got[:, 1], pub["z_star_sim"], atol=6e-4)  # printed with 3 decimals
    # the reference's own pass criterion against Martin & Moyce: within 10 %
    err = np.abs(got[:, 1] - np.asarray(pub["z_star_ref"])) / np.asarray(pub["z_star_ref"])
    assert err.max() <= 0.10
    k.close()


@pytest.mark.parametrize("flags", [0xF, 0xC])
def test_hydrostatic_hires_bit_exact_over_38500_steps(flags):
    sc = V.hydrostatic_hires(setup_domain)
    ref = RUNS["hydrostatic_hires"]
    assert (len(sc.particles), len(sc.boundary)) == (ref["particles"], ref["boundary"]) == (1250, 3150)
    k = cuda(sc, flags)
    run = V.run_to_time(k, 1.0, 1.0)
    want = ref[f"flags{flags:x}_pow1"]
    assert run.steps == want["steps"]
    p = k.particles()
    assert digest(p) == want["digest"]
    cfg = V.HYDROSTATIC_HIRES
    bands = V.hydrostatic_bands(p.y, p.pressure, cfg["domain_min"][1], cfg["domain_max"][1])
    assert [b["p_sim"] for b in bands] == [b["p_sim"] for b in want["bands"]]
    if flags == 0xC:
        # the published P_sim at t = 1 s: the closed, full box still rings
        # (its band pressures swing by +-50 % over 0.75-1 s in the oracle's
        # time series), so one instant is phase-sensitive; every band agrees
        # within 10 % (4-7 % measured, the glibc and correctly rounded runs
        # differ by up to 1.6 %)
        pub = PUBLISHED["hydrostatic_hires"]
        for b, ps in zip(bands[1:], pub["p_sim"][1:]):
            assert abs(b["p_sim"] - ps) <= 0.10 * ps
    k.close()


def test_dam_break_4mm_1000_steps_bit_exact_and_statistics():
    ref = RUNS["dam_break_4mm"]
    sc = domain.dam_break(0.004, seed=ref["seed"], sphere=False, with_sdf=False)
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta)
    front = []
    for s in range(ref["steps"]):
        k.step(k.compute_timestep())
        if (s + 1) % ref["every"] == 0:
            front.append(float(k.particles().x.max()))
    p = k.particles()
    assert digest(p) == ref["pow1"]["digest"]
    assert front == ref["pow1"]["front"]
    # glibc powf: the front within 20 um (1/200 of dx) at every sample (4.4 um
    # measured), the height-band pressures within 3 % (+ 1 Pa)
    np.testing.assert_allclose(front, ref["pow0"]["front"], atol=2e-5)
    bands = V.hydrostatic_bands(p.z, p.pressure, 0.0, 0.1)
    for b, c in zip(bands, ref["pow0"]["bands"]):
        if c["p_sim"] is not None:
            assert abs(b["p_sim"] - c["p_sim"]) <= 0.03 * abs(c["p_sim"]) + 1.0
    k.close()
