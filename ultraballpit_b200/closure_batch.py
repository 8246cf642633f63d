"""Batched sphere-in-tank flows with the learned closure (many coarse
simulations in one launch per stage, closure inference fused into the step).

    python -m ultraballpit_b200.closure_batch --weights W.npy --instances 64 --steps 1000 --compare 4 --out DIR

1. ``draw_instances``: closed tanks with seeded dims in [0.1, 0.4] m (whole
   4 mm spacings), a fill
   giving a log-uniform 4 mm particle count in [50k, 1M], a sphere of radius
   U[0.01, 0.04] m at a seeded submerged position and a start speed
   U[0, 0.5] m/s along +x; fluid, walls and sphere on one lattice with the
   hydrostatic start (``domain.tank_with_sphere``, ``geometry="lattice"``).
   Each instance keeps c0 = 10 sqrt(2 g fill) and steps with
   dt = DT_C_OVER_H h / c0, the dt c / h of the tanks the network was
   trained on.
2. The instances are relaxed together (kinetic damping, one batch), then
   started at their speeds.
3. Timed, 1000 steps each: the batch with the closure (mode 2), the batch
   without it, and the instances one after another without it.
4. For ``--compare`` instances (drawn among those with at most
   ``--compare-max`` particles, which bounds the 2 mm runs' cost): the
   2 mm plain run (dt / 2) is the reference for the 4 mm run without and with the closure
   (``closure.compare_scenarios``: time-averaged near-wall probe pressure
   and the force on the sphere); GPU time of the 2 mm run against the
   instance's share of the batched closure run.

Writes ``DIR/report.json``.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import closure, domain
from .kernel import CudaBatch, CudaKernel

DX = 0.004
# dt c0 / h of the training tanks (dt 5e-5 s, c0 = 10 sqrt(2 g 0.16) m/s, h = 5.2 mm)
DT_C_OVER_H = 5e-5 * float(domain.dam_break_c0(closure.FILL)) / float(domain.smoothing_length(DX))


def draw_instances(n: int, seed: int, counts=(50_000, 1_000_000), dx: float = DX) -> list[dict]:
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        # whole spacings (at dx and dx / 2), so the lattice meets every wall
        # half a spacing from it
        dims = tuple(round(float(v) / dx) * dx for v in rng.uniform(0.1, 0.4, 3))
        target = math.exp(rng.uniform(math.log(counts[0]), math.log(counts[1])))
        fill = round(target * dx ** 3 / (dims[0] * dims[1]) / dx) * dx
        r = float(rng.uniform(0.01, 0.04))
        m = r + 2 * dx
        if fill < 2 * m + 2 * dx or fill > 0.8 * dims[2] or min(dims[0], dims[1]) < 2 * m + 2 * dx:
            continue
        center = (float(rng.uniform(m, dims[0] - m)), float(rng.uniform(m, dims[1] - m)),
                  float(rng.uniform(m, fill - m)))
        out.append(dict(dims=dims, fill=fill, center=center, radius=r, speed=float(rng.uniform(0.0, 0.5)),
                        seed=int(seed * 1000 + len(out))))
    return out


def build(inst: dict, dx: float):
    return domain.tank_with_sphere(dx, domain_max=inst["dims"], center=inst["center"], radius=inst["radius"],
                                   fill_height=inst["fill"], seed=inst["seed"], alpha=closure.ALPHA,
                                   hydrostatic=True, geometry="lattice")


def dt_of(sc) -> float:
    return DT_C_OVER_H * float(sc.h) / float(sc.speed_of_sound)


def settle_batch(scs, seconds: float = closure.SETTLE_S, every: int = 20, device: int = 0):
    """``closure.settle`` for many instances at once (one batch, each
    instance at its own dt); returns relaxed copies at rest."""
    import dataclasses
    b = CudaBatch(scs, device=device)
    dts = np.array([dt_of(sc) for sc in scs], np.float32)
    for s in range(int(math.ceil(seconds / float(dts.min())))):
        b.step_each(dts)
        if (s + 1) % every == 0:
            b.scale_velocities(0.0)
    out = []
    for q, sc in enumerate(scs):
        p = b.instance(q)
        qp = sc.particles.copy()
        qp.x[:], qp.y[:], qp.z[:] = p.x, p.y, p.z
        qp.vx[:] = qp.vy[:] = qp.vz[:] = np.float32(0.0)
        out.append(dataclasses.replace(sc, particles=qp))
    b.health()
    b.close()
    return out


def _timed(fn) -> float:
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--weights", required=True, help="closure weights (5,508 float32, .npy)")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--compare", type=int, default=4)
    ap.add_argument("--compare-max", type=int, default=250_000)
    ap.add_argument("--compare-steps", type=int, default=800)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=".")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    w = np.load(a.weights).astype(np.float32)
    inst = draw_instances(a.instances, a.seed)
    scs = [build(q, DX) for q in inst]
    counts = np.array([len(sc.particles) for sc in scs])
    rep: dict = dict(config=vars(a), particles=int(counts.sum()), boundary=int(sum(len(sc.boundary) for sc in scs)),
                     count_min=int(counts.min()), count_max=int(counts.max()),
                     count_hist_log2=np.bincount(np.log2(counts).astype(int)).tolist())
    t0 = time.perf_counter()
    settled = settle_batch(scs, device=a.device)
    rep["settle_s"] = time.perf_counter() - t0
    for sc, q in zip(settled, inst):
        sc.particles.vx[:] = np.float32(q["speed"])
    dts = np.array([dt_of(sc) for sc in settled], np.float32)

    def batch_run(mode: int) -> float:
        b = CudaBatch(settled, device=a.device)
        if mode:
            b.set_feature_sdfs([sc.sdf for sc in settled])
            b.set_closure(mode, w)
        for _ in range(3):
            b.step_each(dts)
        b.synchronize()
        sec = _timed(lambda: ([b.step_each(dts) for _ in range(a.steps)], b.synchronize()))
        b.health()
        b.close()
        return sec

    rep["batched_closure_s"] = batch_run(2)
    rep["batched_plain_s"] = batch_run(0)
    seq = 0.0
    for sc, dt in zip(settled, dts):
        k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, device=a.device)
        for _ in range(3):
            k.step(float(dt))
        k.synchronize()
        seq += _timed(lambda: ([k.step(float(dt)) for _ in range(a.steps)], k.synchronize()))
        k.close()
    rep["sequential_plain_s"] = seq
    ps = float(counts.sum()) * a.steps
    rep["particle_steps_per_s"] = dict(batched_closure=ps / rep["batched_closure_s"],
                                       batched_plain=ps / rep["batched_plain_s"], sequential_plain=ps / seq)

    rep["compare"] = []
    pick = [q for q in range(len(inst)) if counts[q] <= a.compare_max][: a.compare]
    for q in pick:
        fine = closure.settle(build(inst[q], DX / 2), closure.SETTLE_S, float(dts[q]) / 2, device=a.device)
        fine.particles.vx[:] = np.float32(inst[q]["speed"])
        geo = dict(center=inst[q]["center"], radius=inst[q]["radius"], speed=inst[q]["speed"])
        r = closure.compare_scenarios(settled[q], fine, geo, w, steps=a.compare_steps, dt=float(dts[q]),
                                      device=a.device, fill=inst[q]["fill"], tank=inst[q]["dims"])
        share = rep["batched_closure_s"] * counts[q] / counts.sum() * a.compare_steps / a.steps
        rep["compare"].append(dict(instance=q, particles=int(counts[q]), speed=inst[q]["speed"],
                                   radius=inst[q]["radius"], plain={k: r["plain"][k] for k in ("all", "sphere", "walls", "force")},
                                   closure={k: r["closure"][k] for k in ("all", "sphere", "walls", "force")},
                                   fine_seconds=r["fine_seconds"], batched_share_seconds=float(share),
                                   gpu_time_ratio=float(r["fine_seconds"] / share)))
    with open(os.path.join(a.out, "report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps({k: rep[k] for k in ("particles", "count_min", "count_max", "particle_steps_per_s")}))
    for c in rep["compare"]:
        print(json.dumps(c))
    return rep


if __name__ == "__main__":
    main()
