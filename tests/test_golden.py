"""Committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces every fixture bit for bit (a regression pin
on the checker). GPU: the CUDA step, driven by the fixture's dt sequence,
equals the correctly rounded fixture bit for bit and the libm one within
1e-6 of the domain extent on positions."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

from oracle import mlp_oracle  # noqa: E402

NAMES = ("two_particles", "hydrostatic_column", "water_box_2mm", "dam_break_small")


def _fixture(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(name):
    g = _fixture(name)
    sc = mg.scenarios()[name]
    for pm in (0, 1):
        got = mg.run(sc, pm)
        for f, a in got.items():
            np.testing.assert_array_equal(a, g[f"pow{pm}_{f}"], err_msg=f"{name} pow{pm} {f}")


def test_mlp_oracle_reproduces_fixture():
    g = np.load(os.path.join(HERE, "golden", "mlp.npz"))
    y, _ = mlp_oracle.forward(g["params"], g["x"])
    np.testing.assert_array_equal(np.asarray(y, np.float64), g["y"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_step_matches_fixture(name):
    from ultraballpit_b200.kernel import CudaKernel
    g = _fixture(name)
    sc = mg.scenarios()[name]
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta)
    for dt in g["pow1_dt"]:
        k.step(float(dt))
    p = k.particles()
    for f in mg.FIELDS:
        np.testing.assert_array_equal(getattr(p, f), g[f"pow1_{f}"], err_msg=f"{name} {f}")
    extent = max(b - a for a, b in zip(sc.domain_min, sc.domain_max))
    for f in ("x", "y", "z"):
        assert np.max(np.abs(getattr(p, f).astype(np.float64) - g[f"pow0_{f}"])) <= 1e-6 * extent, (name, f)
    k.close()
