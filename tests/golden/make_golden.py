"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

For each scenario (the reference's own test scenarios and a small dam break)
the literal oracle (tier L: the reference's O(N * N_b) boundary scans) runs
``STEPS`` steps with the reference's dt policy (sph::compute_timestep before
every step) in both pow modes (0: libm powf, the reference on Linux;
1: correctly rounded x^7, what the CUDA kernels compute); the fixture holds
the dt sequence and the final state. ``mlp.npz`` holds the float64 closure
network's outputs on seeded inputs and parameters.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import mlp_oracle  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from ultraballpit_b200 import domain  # noqa: E402

STEPS = 10
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure")


def scenarios():
    return {
        "two_particles": domain.two_particles(),
        "hydrostatic_column": domain.hydrostatic_column(),
        "water_box_2mm": domain.water_box_2mm(),
        "dam_break_small": domain.dam_break(0.004, seed=7, block=(0.04, 0.04, 0.04), domain_max=(0.08, 0.04, 0.04),
                                            with_sdf=False),
    }


def run(sc, pow_mode: int, steps: int = STEPS):
    k = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=0, threads=1, pow_mode=pow_mode)
    dts = []
    for _ in range(steps):
        dt = k.compute_timestep(sc.cfl_number)
        dts.append(dt)
        k.step(dt)
    p = k.particles()
    out = {f: np.asarray(getattr(p, f), np.float32) for f in FIELDS}
    out["dt"] = np.asarray(dts, np.float32)
    return out


def mlp_case():
    rng = np.random.default_rng(123)
    params = (rng.standard_normal(mlp_oracle.N_PARAMS) * 0.2).astype(np.float32)
    x = rng.standard_normal((64, 16)).astype(np.float32)
    y, _ = mlp_oracle.forward(params, x)
    return dict(params=params, x=x, y=np.asarray(y, np.float64))


def main():
    for name, sc in scenarios().items():
        arrs = {}
        for pm in (0, 1):
            for f, a in run(sc, pm).items():
                arrs[f"pow{pm}_{f}"] = a
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrs)
        print(name, len(sc.particles), "particles")
    np.savez_compressed(os.path.join(HERE, "mlp.npz"), **mlp_case())


if __name__ == "__main__":
    main()
