"""Long-run oracle fixtures for the validation parity tests.

Runs the CPU oracle (``oracle/``, tier G; correctly rounded x^7, and glibc
``powf`` for the statistics runs) through the reference's benchmark loop
(``ultraballpit_b200/validation.py``) and stores, per run, the statistics the
reference's harness reads plus a SHA-256 of the final state, so that a GPU
test checks the CUDA path bit for bit over thousands of steps without
re-running the oracle on the GPU host:

* ``dam_break_2d`` (T086, ``configs/dam-break-2d.json``) to t = 0.1 s (past
  T* = 3.5) with the reference's stages as they are (flags 0xF) and without
  delta-SPH and XSPH (flags 0xC: the code of the reference's published
  table, which predates those two stages);
* ``hydrostatic_hires`` (T087) to t = 1 s, both flag sets;
* the 3D dam break at dx = 4 mm (31,250 particles) for 1000 steps: the
  water front (max x) every 10 steps and the mean pressure in 10 height
  bands of the initial column at the end.

    python tests/golden/make_validation.py [threads]

writes ``tests/golden/validation_runs.json`` (about 15 minutes on 8 threads).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from ultraballpit_b200 import domain, validation as V  # noqa: E402

STATE_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "density", "pressure")


def state_digest(p) -> str:
    h = hashlib.sha256()
    for f in STATE_FIELDS:
        h.update(np.ascontiguousarray(getattr(p, f), np.float32).tobytes())
    return h.hexdigest()


class OracleRun:
    """The oracle behind the methods ``validation.run_to_time`` calls."""

    def __init__(self, sc, **kw):
        self.k = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, **kw)
        self.cfl = sc.cfl_number

    def compute_timestep(self):
        return self.k.compute_timestep(self.cfl)

    def step(self, dt):
        self.k.step(dt)

    def particles(self):
        return self.k.particles()


def dam_break_2d_runs(threads: int) -> dict:
    out = {}
    sc, a = V.dam_break_2d(orc.setup_domain)
    for flags in (0xF, 0xC):
        for pm in (1, 0):
            k = OracleRun(sc, tier=1, threads=threads, pow_mode=pm, flags=flags)
            run = V.run_to_time(k, V.DAM_BREAK_2D["max_time"], 0.01, stop_time=0.1)
            rec = {"steps": run.steps, "front": V.front_positions(run, a), "final_time": run.times[-1]}
            if pm == 1:
                rec["digest"] = state_digest(k.particles())
            out[f"flags{flags:x}_pow{pm}"] = rec
    out["a"] = a
    out["particles"], out["boundary"] = len(sc.particles), len(sc.boundary)
    return out


def hydrostatic_runs(threads: int) -> dict:
    out = {}
    sc = V.hydrostatic_hires(orc.setup_domain)
    cfg = V.HYDROSTATIC_HIRES
    for flags in (0xF, 0xC):
        for pm in (1, 0):
            k = OracleRun(sc, tier=1, threads=threads, pow_mode=pm, flags=flags)
            run = V.run_to_time(k, 1.0, 1.0)
            p = k.particles()
            rec = {"steps": run.steps,
                   "bands": V.hydrostatic_bands(p.y, p.pressure, cfg["domain_min"][1], cfg["domain_max"][1])}
            if pm == 1:
                rec["digest"] = state_digest(p)
            out[f"flags{flags:x}_pow{pm}"] = rec
    out["particles"], out["boundary"] = len(sc.particles), len(sc.boundary)
    return out


def dam_break_3d_runs(threads: int, steps: int = 1000, every: int = 10) -> dict:
    sc = domain.dam_break(0.004, seed=2024, sphere=False, with_sdf=False)
    out = {"seed": 2024, "steps": steps, "every": every, "particles": len(sc.particles),
           "boundary": len(sc.boundary)}
    for pm in (1, 0):
        k = OracleRun(sc, tier=1, threads=threads, pow_mode=pm)
        front, dts = [], []
        for s in range(steps):
            dt = k.compute_timestep()
            dts.append(float(dt))
            k.step(dt)
            if (s + 1) % every == 0:
                front.append(float(k.particles().x.max()))
        p = k.particles()
        rec = {"front": front, "sim_time": float(np.sum(np.asarray(dts, np.float64))),
               "bands": V.hydrostatic_bands(p.z, p.pressure, 0.0, 0.1)}
        if pm == 1:
            rec["digest"] = state_digest(p)
        out[f"pow{pm}"] = rec
    return out


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    t0 = time.time()
    res = {"generator": "tests/golden/make_validation.py", "oracle": "tier G",
           "dam_break_2d": dam_break_2d_runs(threads)}
    print(f"dam_break_2d {time.time() - t0:.0f} s", flush=True)
    res["dam_break_4mm"] = dam_break_3d_runs(threads)
    print(f"dam_break_4mm {time.time() - t0:.0f} s", flush=True)
    res["hydrostatic_hires"] = hydrostatic_runs(threads)
    print(f"hydrostatic_hires {time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "validation_runs.json"), "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
