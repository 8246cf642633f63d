"""The 2,000,000-particle dam break (dx = 1 mm) with the fixed sphere for
2000 steps, reporting the pressure and viscous force
integrals on the sphere.

    python -m ultraballpit_b200.sphere_run [--steps 2000] [--every 50] [--out FILE]

Every ``--every`` steps it records the simulated time and, in FP64:

* the reaction of the fluid on the sphere's boundary particles
  (``sph_body_force`` over the geometry layers): the pressure force the
  fluid receives from them negated (kernel/src/sph.rs:391-408), the
  repulsion likewise (boundary.rs:161-179), and a Monaghan viscous force
  with the body at rest;
* ``compute_surface_forces`` (orchestrator/src/force.rs:39-129) over the
  sphere's SDF nodes, in FP64 and in the reference's own f32 node order.

``tests/test_sphere_forces_gpu.py`` checks the first samples of this series
against the CPU oracle.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import time

import numpy as np

from . import domain
from .kernel import CudaKernel


STATE_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure")


def record(step, t, body, surf):
    return {"step": step, "time": t,
            "pressure_force": body["pressure_force"].tolist(), "viscous_force": body["viscous_force"].tolist(),
            "repulsion_force": body["repulsion_force"].tolist(), "surface_force": surf["force"].tolist(),
            "surface_force_f32": surf["force_f32"].tolist(), "surface_active_nodes": surf.get("active_nodes")}


def scenario(seed: int = 2024):
    """(scenario, first sphere boundary particle, sphere boundary particles)."""
    sc = domain.dam_break(0.001, seed=seed, sphere=True, with_sdf=True)
    nb_geo = sc.extras["n_geometry_boundary"]
    return sc, len(sc.boundary) - nb_geo, nb_geo


def run(steps: int = 2000, every: int = 50, seed: int = 2024, device: int = 0, on_sample=None,
        state_digest: bool = False) -> dict:
    """The run; ``on_sample(step, dt)`` (optional) is called after every step
    with the step's dt, before that step's sample is taken. ``state_digest``
    adds the SHA-256 of the final state (STATE_FIELDS, original order)."""
    sc, first, nb_geo = scenario(seed)
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, device=device)
    k.set_geometry_sdf(sc.obstacle_sdf)
    out = {"workload": "dam_break_1mm_sphere", "particles": len(sc.particles), "boundary": len(sc.boundary),
           "sphere_boundary_particles": nb_geo, "sphere": {"center": sc.extras["sphere_center"],
                                                           "radius": sc.extras["sphere_radius"]},
           "steps": steps, "every": every, "samples": []}
    t, t0 = 0.0, time.perf_counter()
    for s in range(1, steps + 1):
        dt = k.compute_timestep()
        k.step(dt)
        t += float(np.float32(dt))
        if on_sample is not None:
            on_sample(s, dt)
        if s % every == 0 or s == steps:
            out["samples"].append(record(s, t, k.body_force(first, nb_geo), k.surface_forces()))
    out["wall_s"] = time.perf_counter() - t0
    if state_digest:
        p = k.particles()
        h = hashlib.sha256()
        for f in STATE_FIELDS:
            h.update(np.ascontiguousarray(getattr(p, f), np.float32).tobytes())
        out["state_sha256"] = h.hexdigest()
    k.synchronize()
    out["health_nonfinite"] = k.health()
    k.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--out", default="sphere_run.json")
    a = ap.parse_args()
    res = run(a.steps, a.every)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    last = res["samples"][-1]
    print(json.dumps({"steps": a.steps, "time": last["time"], "pressure_force": last["pressure_force"],
                      "viscous_force": last["viscous_force"], "wall_s": res["wall_s"]}))


if __name__ == "__main__":
    main()
