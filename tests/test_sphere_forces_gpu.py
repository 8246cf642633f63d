"""The sphere force series (``ultraballpit_b200.sphere_run``)
against the CPU oracle: the first 10 steps of the 2,000,000-particle dam
break with the sphere, sampled every 5 steps. The states are bit-identical
(correctly rounded x^7 in both; every field of every particle compared after
the 10th step); the FP64 integrals on the sphere (the
fluid's reaction on the sphere's boundary particles, and force.rs's surface
integral) differ only in summation order: within 1e-9 relative. (The
water front reaches the sphere only after several thousand steps, so these
early samples check the plumbing of the series; the integrals themselves are
checked against the oracle on a submerged sphere in test_parity_gpu.)"""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as orc
from ultraballpit_b200 import sphere_run

pytestmark = pytest.mark.gpu


def test_sphere_force_series_matches_the_oracle():
    sc, first, nb = sphere_run.scenario()
    ok = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=1,
                          threads=os.cpu_count() or 1, pow_mode=1)
    want = {}

    def beside(step, dt):
        odt = ok.compute_timestep(sc.cfl_number)
        assert odt == dt, (step, odt, dt)
        ok.step(odt)
        if step % 5 == 0:
            want[step] = sphere_run.record(step, 0.0, ok.body_force(first, nb), ok.surface_forces(sc.obstacle_sdf))

    res = sphere_run.run(steps=10, every=5, on_sample=beside, state_digest=True)
    assert res["health_nonfinite"] == 0 and len(res["samples"]) == 2
    for s in res["samples"]:
        w = want[s["step"]]
        for key in ("pressure_force", "viscous_force", "repulsion_force", "surface_force"):
            a, b = np.asarray(s[key]), np.asarray(w[key])
            assert np.allclose(a, b, rtol=1e-9, atol=1e-12 * max(1.0, np.abs(b).max())), (key, a, b)
        assert s["surface_force_f32"] == w["surface_force_f32"]
    p = ok.particles()
    h = hashlib.sha256()
    for f in sphere_run.STATE_FIELDS:
        h.update(np.ascontiguousarray(getattr(p, f), np.float32).tobytes())
    assert res["state_sha256"] == h.hexdigest()
