"""BASELINE config 2 as specified: the 2,000,000-particle dam break with the
fixed sphere for 2000 steps, reporting the pressure and viscous force
integrals on the sphere.

    python -m ultraballpit_b200.sphere_run [--steps 2000] [--every 50] [--oracle-steps 100] [--out FILE]

Every ``--every`` steps it records the simulated time and, in FP64:

* the reaction of the fluid on the sphere's boundary particles
  (``sph_body_force`` over the geometry layers): the pressure force the
  fluid receives from them negated (kernel/src/sph.rs:391-408), the
  repulsion likewise (boundary.rs:161-179), and a Monaghan viscous force
  with the body at rest;
* ``compute_surface_forces`` (orchestrator/src/force.rs:39-129) over the
  sphere's SDF nodes, in FP64 and in the reference's own f32 node order.

With ``--oracle-steps N`` the CPU oracle (tier G, correctly rounded x^7,
all host threads) runs the first N steps beside it and the same integrals
are compared at every sample (the states are bit-identical, the FP64 sums
differ only in summation order).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import domain
from .kernel import CudaKernel


def _record(step, t, body, surf):
    return {"step": step, "time": t,
            "pressure_force": body["pressure_force"].tolist(), "viscous_force": body["viscous_force"].tolist(),
            "repulsion_force": body["repulsion_force"].tolist(), "surface_force": surf["force"].tolist(),
            "surface_force_f32": surf["force_f32"].tolist(), "surface_active_nodes": surf.get("active_nodes")}


def run(steps: int = 2000, every: int = 50, oracle_steps: int = 0, seed: int = 2024, device: int = 0) -> dict:
    sc = domain.dam_break(0.001, seed=seed, sphere=True, with_sdf=True)
    nb_geo = sc.extras["n_geometry_boundary"]
    first = len(sc.boundary) - nb_geo
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, device=device)
    k.set_geometry_sdf(sc.obstacle_sdf)
    orc_k = None
    if oracle_steps > 0:
        from oracle import oracle as orc  # the checker: only with --oracle-steps
        orc_k = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=1,
                                 threads=os.cpu_count() or 1, pow_mode=1)
    out = {"workload": "dam_break_1mm_sphere", "particles": len(sc.particles), "boundary": len(sc.boundary),
           "sphere_boundary_particles": nb_geo, "sphere": {"center": sc.extras["sphere_center"],
                                                           "radius": sc.extras["sphere_radius"]},
           "steps": steps, "every": every, "samples": [], "oracle": []}
    t, t0 = 0.0, time.perf_counter()
    for s in range(1, steps + 1):
        dt = k.compute_timestep()
        k.step(dt)
        t += float(np.float32(dt))
        if orc_k is not None and s <= oracle_steps:
            odt = orc_k.compute_timestep(sc.cfl_number)
            assert odt == dt, (s, odt, dt)
            orc_k.step(odt)
        if s % every == 0 or s == steps:
            rec = _record(s, t, k.body_force(first, nb_geo), k.surface_forces())
            out["samples"].append(rec)
            if orc_k is not None and s <= oracle_steps:
                ob = orc_k.body_force(first, nb_geo)
                osf = orc_k.surface_forces(sc.obstacle_sdf)
                out["oracle"].append(_record(s, t, ob, osf))
    out["wall_s"] = time.perf_counter() - t0
    k.synchronize()
    out["health_nonfinite"] = k.health()
    k.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--oracle-steps", type=int, default=0)
    ap.add_argument("--out", default="sphere_run.json")
    a = ap.parse_args()
    res = run(a.steps, a.every, a.oracle_steps)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    last = res["samples"][-1]
    print(json.dumps({"steps": a.steps, "time": last["time"], "pressure_force": last["pressure_force"],
                      "viscous_force": last["viscous_force"], "wall_s": res["wall_s"]}))


if __name__ == "__main__":
    main()
