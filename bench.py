"""Throughput of the WCSPH step in particle-steps/s on B200 (one JSON line).

Workload (default): the 3D dam break at dx = 1 mm, 2,000,000 fluid particles,
with the fixed sphere obstacle (r = 0.02 m at (0.25, 0.1, 0.03)) as geometry
boundary particles plus 3-layer walls, CFL 0.25 with dt computed on the
device each step, alpha = 0.02. Inputs are synthetic (seeded jitter), built
on the host. A "step" is one full SPH step of every particle.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload dam_break_1mm_sphere]

Under torchrun each rank runs its own replica (instances are independent, no
collective on the data path); rank 0 prints the whole-job throughput.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200: plain vs batched+closure at fixed error"
UNIT = "particle-steps/s"
WORKLOADS = {
    "dam_break_1mm_sphere": dict(dx=0.001, sphere=True),   # 2,000,000 particles
    "dam_break_4mm": dict(dx=0.004, sphere=False),          # 31,250 particles
    "dam_break_2mm": dict(dx=0.002, sphere=False),          # 250,000 particles (profiling case)
    "batch_boxes_2mm": dict(batch=256),                     # 256 instances, about 51M particles
    "batch_boxes_2mm_loguniform": dict(batch=256, draw="loguniform"),  # 256 instances, about 20M
    # 64 sphere-in-tank flows at 4 mm with the learned closure (about 8.6M particles)
    "batch_closure_4mm": dict(batch=64, closure=True),
}
CLOSURE_WEIGHTS = os.path.join(ROOT, "ultraballpit_b200", "data", "closure_weights.npy")


def pair_stats(sc, sample: int = 20000, seed: int = 0) -> dict:
    """Mean in-support neighbours (interactions) and mean candidates per
    particle on a seeded sample of the initial state (2h grid cells, as the
    kernels bin): every particle of the 27 cells, as the reference's neighbour
    loop tests them (neighbor.rs:129-182) and as the warp-cooperative density
    scan does, and the fewer left after the per-thread scan's cell culling."""
    from scipy.spatial import cKDTree
    p = sc.particles
    pos = np.stack([p.x, p.y, p.z], axis=1).astype(np.float64)
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(pos), min(sample, len(pos)), replace=False)
    r = 2.0 * sc.h
    inter = cKDTree(pos).query_ball_point(pos[pick], r, return_length=True) - 1
    gmin = np.asarray(sc.domain_min, np.float64)
    cell = 2.0 * sc.h
    dims = np.maximum(np.ceil((np.asarray(sc.domain_max) - gmin) / cell), 1).astype(np.int64)
    c = np.clip(np.floor((pos - gmin) / cell).astype(np.int64), 0, dims - 1)
    lin = (c[:, 2] * dims[1] + c[:, 1]) * dims[0] + c[:, 0]
    counts = np.bincount(lin, minlength=int(np.prod(dims)))
    cq, pq = c[pick], pos[pick]
    face = gmin + cq * cell
    lo2 = np.maximum(pq - face, 0.0) ** 2
    hi2 = np.maximum(face + cell - pq, 0.0) ** 2
    cand = np.zeros(len(pick))
    cand_all = np.zeros(len(pick))
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                d = np.array([dx, dy, dz])
                e = sum(np.where(d[a] < 0, lo2[:, a], np.where(d[a] > 0, hi2[:, a], 0.0)) for a in range(3))
                nc = cq + d
                inside = np.all((nc >= 0) & (nc < dims), axis=1)
                ok = inside & (e <= r * r)
                l2 = (nc[:, 2] * dims[1] + nc[:, 1]) * dims[0] + nc[:, 0]
                cand += np.where(ok, counts[np.where(ok, l2, 0)], 0)
                cand_all += np.where(inside, counts[np.where(inside, l2, 0)], 0)
    return {"interactions_per_particle": float(inter.mean()), "candidates_per_particle": float(cand_all.mean() - 1),
            "candidates_after_culling_per_particle": float(cand.mean() - 1),
            "sample": f"{len(pick)} particles of the initial state"}


def roofline_bytes():
    src = open(os.path.join(ROOT, "include", "sph_roofline.h")).read()
    return {k: int(v) for k, v in re.findall(r"#define (SPH_\w+) (\d+)", src)}


KERNEL_SOURCES = ["ultraballpit_b200/csrc/sph_kernels.cuh", "ultraballpit_b200/csrc/sph_mlp.cuh"]


def strip_source(src: bytes) -> bytes:
    """C++ source without comments and whitespace: what a digest of the
    kernels should see (string literals in these files hold no comment
    markers)."""
    src = re.sub(rb"/\*.*?\*/", b"", src, flags=re.S)
    src = re.sub(rb"//[^\n]*", b"", src)
    return re.sub(rb"\s+", b"", src)


def kernel_sources_digest(read=None) -> str:
    """sha1 over the step's kernel sources (comments and whitespace removed,
    so a change of wording or layout alone keeps it) and the default launch
    shapes: an ncu figure recorded with the same digest was captured on these
    kernels. `read(path)` returns a file's bytes (default: this tree)."""
    import hashlib
    read = read or (lambda f: open(os.path.join(ROOT, f), "rb").read())
    h = hashlib.sha1()
    for f in KERNEL_SOURCES:
        h.update(strip_source(read(f)))
    api = read("ultraballpit_b200/csrc/sph_api.cu").decode()
    h.update(re.search(r"int bs_xsph = \d+, bs_density = \d+, bs_forces = \d+;", api).group(0).encode())
    return h.hexdigest()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.first = threading.Event()
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(timeout=5.0)   # sampling is live before the timed region starts
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append([time.monotonic()] + parts)
                self.first.set()

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        inside = [r[1:] for r in self.rows if self.t0 <= r[0] <= self.t1]
        # a region shorter than the sampling period: the samples next to it
        rows = inside or [r[1:] for r in sorted(self.rows, key=lambda r: min(abs(r[0] - self.t0),
                                                                           abs(r[0] - self.t1)))[:2]]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside), "period_ms": 200}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def build_scenario(name: str, seed: int):
    from ultraballpit_b200 import domain
    w = WORKLOADS[name]
    if "batch" in w:
        raise SystemExit("the batch workload has no CPU reference leg in this script")
    return domain.dam_break(w["dx"], seed=seed, sphere=w["sphere"], with_sdf=w["sphere"])


def cpu_reference_run(sc, steps: int, warmup: int, budget_s: float, threads: int):
    """Time the CPU oracle (the reference algorithm, grid-accelerated boundary
    loops with identical results) on the same workload."""
    from oracle import oracle as orc
    k = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, tier=1, threads=threads, pow_mode=0)
    for _ in range(warmup):
        k.step(k.compute_timestep(sc.cfl_number))
    done, t0 = 0, time.perf_counter()
    while done < steps:
        k.step(k.compute_timestep(sc.cfl_number))
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return len(sc.particles) * done / el, done, el


def measure_batch(scs, steps: int, warmup: int, local: int) -> dict:
    """Batched step of independent simulations (one handle, one launch per
    stage, graph-captured, CFL dt per instance on the device) against the same
    instances solved one after another, each through its own single-simulation
    handle with the same launch shapes: device times of ``steps`` steps."""
    import torch
    from ultraballpit_b200.kernel import CudaBatch, CudaKernel
    b = CudaBatch(scs, device=local)
    stream = torch.cuda.ExternalStream(b.stream())
    tuned = b.autotune(3)
    b.step_auto(warmup, want_dt=True)
    torch.cuda.synchronize()
    l0 = b.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        b.step_auto(steps, want_dt=False)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = b.launch_count() - l0
    b.synchronize()
    if b.health() != 0:
        raise SystemExit("non-finite particle state after the timed steps")
    prof = {}
    for _ in range(3):
        for kk, v in b.step_profiled(float(b.timesteps().min())).items():
            prof[kk] = prof.get(kk, 0.0) + v / 3
    b.close()
    del b
    seq_ms = 0.0
    for sc in scs:
        k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, device=local)
        k.set_launch(**tuned)
        st = torch.cuda.ExternalStream(k.stream())
        k.step_auto(warmup, want_dt=True)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        k.step_auto(steps, want_dt=False)
        a1.record(st)
        a1.synchronize()
        seq_ms += a0.elapsed_time(a1)
        k.synchronize()
        k.close()
    return dict(ms=ms, seq_ms=seq_ms, launches=launches, tuned=tuned, prof=prof, clk=clk.summary())


def run_batch_arm(args):
    """Batched step of independent boxes against the same instances solved
    one after another (each through its own single-simulation handle)."""
    import torch
    from ultraballpit_b200 import domain
    from ultraballpit_b200.replicas import Replicas
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    w = WORKLOADS[args.workload]
    if args.shard:
        # one draw shared by all ranks, instances bin-packed across the GPUs
        from ultraballpit_b200.replicas import partition_lpt
        allscs = domain.batch_boxes(w["batch"], seed=args.seed, draw=w.get("draw", "stated"))
        mine = partition_lpt([len(s.particles) for s in allscs], world)[rank]
        scs = [allscs[i] for i in mine]
    else:
        scs = domain.batch_boxes(w["batch"], seed=args.seed + rank, draw=w.get("draw", "stated"))
    ntot = sum(len(s.particles) for s in scs)
    m = measure_batch(scs, args.steps, args.warmup, local)
    value, ms = rep.whole_job_rate(ntot, args.steps, m["ms"])
    seq_value, seq_ms = rep.whole_job_rate(ntot, args.steps, m["seq_ms"])
    per_rank = rep.gather({"instances": len(scs), "particles": ntot})
    rep.close()
    counts = [len(s.particles) for s in scs]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded boxes, host-built)",
        "config": {"workload": args.workload, "instances": len(scs), "particles": ntot,
                   "sharding": "one draw bin-packed across ranks" if args.shard else "a draw per rank",
                   "per_rank": per_rank,
                   "boundary_particles": sum(len(s.boundary) for s in scs),
                   "instance_particles_min_max": [min(counts), max(counts)],
                   "size_histogram_log2": domain.size_histogram(scs), "launch": m["tuned"],
                   "dt": "device CFL per instance", "l2": "inputs larger than L2"},
        "sequential": {"value": seq_value, "unit": UNIT, "ms_per_step": seq_ms / args.steps,
                       "how": "each instance alone through sph_create, same launch shapes, graph-captured"},
        "batched_over_sequential": value / seq_value,
        "stage_us": {kk: round(v, 1) for kk, v in m["prof"].items()},
        "clocks": m["clk"], "gpu_launches": m["launches"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_subrecord(args, local: int) -> dict:
    """The batched form beside the default line: a seeded draw of
    ``--batch-instances`` boxes at dx = 2 mm with particle counts log-uniform
    in [2k, 400k] (the batch workload's draw, fewer instances so the default
    run stays short), batched against one after another."""
    from ultraballpit_b200 import domain
    scs = domain.batch_boxes(args.batch_instances, seed=args.seed, draw="loguniform")
    ntot = sum(len(s.particles) for s in scs)
    m = measure_batch(scs, args.steps, args.warmup, local)
    counts = [len(s.particles) for s in scs]
    value = ntot * args.steps / (m["ms"] / 1e3)
    seq = ntot * args.steps / (m["seq_ms"] / 1e3)
    return {"workload": "batch_boxes_2mm_loguniform", "instances": len(scs), "particles": ntot,
            "instance_particles_min_max": [min(counts), max(counts)], "value": value, "unit": UNIT,
            "ms_per_step": m["ms"] / args.steps, "sequential_value": seq,
            "sequential_ms_per_step": m["seq_ms"] / args.steps, "batched_over_sequential": value / seq,
            "launch": m["tuned"], "gpu_launches": m["launches"], "clocks": m["clk"],
            "stage_us": {kk: round(v, 1) for kk, v in m["prof"].items()}}


def run_batch_closure_arm(args):
    """Batched sphere-in-tank flows with the closure fused into the step
    against the same instances solved one after another without it."""
    import torch
    from ultraballpit_b200 import closure_batch as cb
    from ultraballpit_b200.kernel import CudaBatch, CudaKernel
    from ultraballpit_b200.replicas import Replicas
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    w = WORKLOADS[args.workload]
    weights = np.load(CLOSURE_WEIGHTS).astype(np.float32)
    inst = cb.draw_instances(w["batch"], args.seed + rank)
    scs = cb.settle_batch([cb.build(q, cb.DX) for q in inst], device=local)
    for sc, q in zip(scs, inst):
        sc.particles.vx[:] = np.float32(q["speed"])
    dts = np.array([cb.dt_of(sc) for sc in scs], np.float32)
    ntot = sum(len(s.particles) for s in scs)
    b = CudaBatch(scs, device=local)
    b.set_feature_sdfs([sc.sdf for sc in scs])
    b.set_closure(2, weights)
    stream = torch.cuda.ExternalStream(b.stream())
    for _ in range(args.warmup):
        b.step_each(dts)
    torch.cuda.synchronize()
    l0 = b.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            b.step_each(dts)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = b.launch_count() - l0
    b.synchronize()
    if b.health() != 0:
        raise SystemExit("non-finite particle state after the timed steps")
    b.close()
    del b
    seq_ms = 0.0
    for sc, dt in zip(scs, dts):
        k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, device=local)
        st = torch.cuda.ExternalStream(k.stream())
        for _ in range(args.warmup):
            k.step(float(dt))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        for _ in range(args.steps):
            k.step(float(dt))
        a1.record(st)
        a1.synchronize()
        seq_ms += a0.elapsed_time(a1)
        k.close()
    value, ms = rep.whole_job_rate(ntot, args.steps, ms)
    seq_value, seq_ms = rep.whole_job_rate(ntot, args.steps, seq_ms)
    rep.close()
    counts = [len(s.particles) for s in scs]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (closure network bf16 operands, f32 accumulation)",
        "data": "synthetic (seeded sphere-in-tank flows, host-built, relaxed on the device)",
        "config": {"workload": args.workload, "instances": len(scs), "particles": ntot,
                   "boundary_particles": sum(len(s.boundary) for s in scs),
                   "instance_particles_min_max": [min(counts), max(counts)],
                   "size_histogram_log2": np.bincount(np.log2(counts).astype(int)).tolist(),
                   "dt": "per instance, dt c0 / h = %.4f" % cb.DT_C_OVER_H, "closure": "mode 2, shipped weights",
                   "l2": "inputs larger than L2"},
        "sequential_plain": {"value": seq_value, "unit": UNIT, "ms_per_step": seq_ms / args.steps,
                             "how": "each instance alone through sph_create, closure off, graph-captured"},
        "batched_closure_over_sequential_plain": value / seq_value,
        "clocks": clk.summary(), "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def plain_config(args, sc, world: int) -> dict:
    """The config block of a single-simulation workload, shared by both arms
    so that the two lines name the same workload with the same keys."""
    n = len(sc.particles)
    state_bytes = n * 4 * (16 * 6 + 8 * 2 + 4 * 6)
    return {"workload": args.workload, "particles_per_gpu": n, "boundary_particles": len(sc.boundary),
            "parallelism": f"replicas{world}", "dt": "device CFL each step",
            "l2": f"inputs larger than L2 (state {state_bytes / 1e6:.0f} MB per GPU)",
            "alpha": sc.alpha, "cell_order": "rows", "seed": args.seed}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sc = build_scenario(args.workload, seed=args.seed)
    threads = os.cpu_count() or 1
    value, done, el = cpu_reference_run(sc, args.steps, args.warmup, args.ref_budget, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": done, "warmup": args.warmup, "ms_per_step": el / done * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dam break, host-built)",
        "config": plain_config(args, sc, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{done} of the {args.steps} requested full steps of {args.workload} "
                                   f"({len(sc.particles)} particles) within {args.ref_budget:.0f} s, after "
                                   f"{args.warmup} warm-up steps; oracle tier G (reference arithmetic, "
                                   f"grid-visited boundary terms)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_cuda_arm(args):
    import torch
    from ultraballpit_b200.replicas import Replicas
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    from ultraballpit_b200.kernel import CudaKernel

    def barrier():
        rep.barrier()
        torch.cuda.synchronize()

    sc = build_scenario(args.workload, seed=args.seed + rank)
    n = len(sc.particles)
    kw = dict(alpha=sc.alpha, beta=sc.beta, device=local)

    # ---- device-resident throughput (value) ------------------------------
    k = CudaKernel(*sc.kernel_args(), **kw)
    stream = torch.cuda.ExternalStream(k.stream())
    k.step_auto(args.warmup, want_dt=True)
    barrier()
    l0 = k.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        k.step_auto(args.steps, want_dt=False)
        e1.record(stream)
        e1.synchronize()
    launches = k.launch_count() - l0
    # every kernel returns at once when the device error word is set, so a
    # tripped capacity bound or a non-finite state would make the timed steps
    # fast and meaningless: the run must end clean
    k.synchronize()
    if k.health() != 0:
        raise SystemExit("non-finite particle state after the timed steps")
    barrier()
    value, ms = rep.whole_job_rate(n, args.steps, e0.elapsed_time(e1))

    # ---- per-kernel durations (profiled steps, events between stages) -----
    prof_steps = max(3, min(args.steps // 4, 50))
    acc = {}
    for _ in range(prof_steps):
        dt = k.compute_timestep()
        p = k.step_profiled(dt)
        for kk, v in p.items():
            acc[kk] = acc.get(kk, 0.0) + v
    avg = {kk: v / prof_steps for kk, v in acc.items()}
    stage_keys = ["xsph_drift_us", "sort_us", "density_us", "boundary_pressure_us", "forces_us"]
    dom = max(stage_keys, key=lambda s: avg[s])
    rb = roofline_bytes()
    bytes_of = {"xsph_drift_us": rb["SPH_BYTES_XSPH_DRIFT"] * n,
                "sort_us": rb["SPH_BYTES_SORT"] * n + rb["SPH_BYTES_PER_CELL"] * k.grid_info()["total_cells"],
                "density_us": rb["SPH_BYTES_DENSITY"] * n,
                "boundary_pressure_us": rb["SPH_BYTES_PER_BOUNDARY"] * len(sc.boundary),
                "forces_us": rb["SPH_BYTES_FORCES"] * n}
    peak, peak_kind = measured_peaks()
    hbm_achieved = bytes_of[dom] / (avg[dom] * 1e-6) / 1e9
    ps = pair_stats(sc)
    cand, inter = ps["candidates_per_particle"], ps["interactions_per_particle"]
    # FP32 operations per particle of each neighbour kernel (sph_roofline.h)
    flops_of = {"density_us": cand * rb["SPH_FLOPS_SCAN_PER_CANDIDATE"]
                + inter * rb["SPH_FLOPS_DENSITY_PER_INTERACTION"],
                "forces_us": inter * rb["SPH_FLOPS_FORCES_PER_INTERACTION"],
                "xsph_drift_us": inter * rb["SPH_FLOPS_XSPH_PER_INTERACTION"]}
    sm_mhz = clk.summary().get("sm_max_mhz") or 1965.0
    fp32_peak = rb["SPH_FP32_LANES_PER_SM"] * rb["SPH_SM_COUNT"] * sm_mhz * 1e6 / 1e12  # TFLOP/s
    prof_ncu, traffic, fresh = {}, None, False
    tfile = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tfile):
        tj = json.load(open(tfile))
        fresh = tj.get("kernel_sources_sha1") == kernel_sources_digest()
        prof_ncu = tj.get(dom.replace("_us", ""), {})
        if "bytes_per_particle" in prof_ncu:
            traffic = prof_ncu["bytes_per_particle"] * n
    hbm = {"achieved": hbm_achieved, "peak": peak, "unit": "GB/s", "frac": hbm_achieved / peak,
           "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_of[dom]}
    if traffic is not None:
        # DRAM rate of the ncu-measured traffic at this run's launch time
        hbm["dram_gbs_of_measured_traffic"] = traffic / (avg[dom] * 1e-6) / 1e9
        hbm["dram_frac_of_measured_traffic"] = hbm["dram_gbs_of_measured_traffic"] / peak
    if dom in flops_of:
        # neighbour kernels: bound by instruction issue (ncu), measured here as
        # FP32 operations per second against the FP32 peak at this run's clock
        achieved = n * flops_of[dom] / (avg[dom] * 1e-6) / 1e12
        roofline = {"bound": "issue", "kernel": dom.replace("_us", ""), "achieved": achieved,
                    "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                    "peak_source": f"FP32 lanes x SMs x {sm_mhz:.0f} MHz (sph_roofline.h)",
                    "flops_per_particle": flops_of[dom]}
    else:
        roofline = {"bound": "hbm", "kernel": dom.replace("_us", ""), "achieved": hbm_achieved, "peak": peak,
                    "unit": "GB/s", "frac": hbm_achieved / peak, "peak_source": peak_kind}
    roofline.update({
        "traffic": traffic,
        "traffic_source": ("profiles/ncu_traffic.json, captured on these kernel sources" if fresh else
                           "profiles/ncu_traffic.json, captured on earlier kernel sources (stale)")
        if traffic is not None else None,
        "issue_active_pct_ncu": prof_ncu.get("issue_active_pct"),
        "threads_active_per_warp_instruction_ncu": prof_ncu.get("threads_per_inst"),
        "l2_pct_of_peak_ncu": prof_ncu.get("l2_pct_of_peak"),
        "hbm": hbm,
        "stage_us": {s.replace("_us", ""): round(avg[s], 2) for s in stage_keys},
        "kernels": {s.replace("_us", ""): {"tflops": n * f / (avg[s] * 1e-6) / 1e12,
                                           "fp32_frac": n * f / (avg[s] * 1e-6) / 1e12 / fp32_peak}
                    for s, f in flops_of.items()},
    })
    roofline["pairs"] = dict(ps, **{
        "density_candidate_tests_per_s": n * ps["candidates_per_particle"] / (avg["density_us"] * 1e-6),
        "density_interactions_per_s": n * ps["interactions_per_particle"] / (avg["density_us"] * 1e-6),
        "forces_interactions_per_s": n * ps["interactions_per_particle"] / (avg["forces_us"] * 1e-6),
        "xsph_interactions_per_s": n * ps["interactions_per_particle"] / (avg["xsph_drift_us"] * 1e-6)})
    k.close()
    del k

    # ---- end to end through the public API from host arrays ---------------
    barrier()
    t0 = time.perf_counter()
    k2 = CudaKernel(*sc.kernel_args(), **kw)
    for _ in range(args.steps):
        dt = k2.compute_timestep()
        k2.step(dt)
        k2.error_metrics()
    final = k2.particles()
    torch.cuda.synchronize()
    e2e_s = rep.max(time.perf_counter() - t0)
    n_all = rep.sum(n)
    assert len(final) == n
    k2.close()
    h2d_init = n * (13 * 4 + 1) + len(sc.boundary) * 7 * 4
    d2h_final = n * (13 * 4 + 1)
    e2e = {"value": n_all * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": h2d_init / args.steps + 4,
           "d2h_bytes_per_step": d2h_final / args.steps + 4 + 12 + 4,
           "includes": "handle creation from host arrays, per step compute_timestep + step + "
                       "error_metrics, final particles() readback"}

    # ---- setup_domain (domain.rs:36-402) of this box and obstacle --------
    setup = None
    if sc.obstacle_sdf is not None:
        from ultraballpit_b200.kernel import setup_domain
        from ultraballpit_b200.particles import DomainSpec
        spec = DomainSpec(float(np.float32(WORKLOADS[args.workload]["dx"])), sc.domain_min, sc.domain_max)
        setup_domain(spec, sc.obstacle_sdf, device=local)          # warm-up
        t0 = time.perf_counter()
        sp, sb = setup_domain(spec, sc.obstacle_sdf, device=local)
        setup_s = time.perf_counter() - t0
        setup = {"fluid": len(sp), "boundary": len(sb), "device_call_ms": setup_s * 1e3,
                 "includes": "SDF upload, count + scan + emit kernels, both particle sets read back into "
                             "pageable host arrays (two calls: count, then fill)"}
        del sp, sb

    batched = None
    if world == 1 and args.batch_instances > 0:
        batched = batched_subrecord(args, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, done, el = cpu_reference_run(sc, 3, 0, args.cpu_budget, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{done} full steps of {args.workload} ({n} particles) on {threads} host threads, "
                         f"oracle tier G ({el:.1f} s)"}
        if setup is not None:
            from oracle import oracle as orc
            t0 = time.perf_counter()
            orc.setup_domain(spec, sc.obstacle_sdf)
            setup["oracle_ms"] = (time.perf_counter() - t0) * 1e3
            setup["oracle"] = "literal restatement of domain.rs:36-402, one host thread"

    rep.barrier()
    rep.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded dam break, host-built)",
            "config": plain_config(args, sc, world),
            "clocks": clk.summary(), "gpu_launches": launches, "e2e": e2e,
            "roofline": roofline, "cpu_baseline": cpu, "domain_setup": setup, "batched": batched,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="dam_break_1mm_sphere", choices=sorted(WORKLOADS))
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-budget", type=float, default=25.0)
    ap.add_argument("--ref-budget", type=float, default=150.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=64,
                    help="default workload: instances of the batched sub-record (0: none)")
    ap.add_argument("--shard", action="store_true",
                    help="batch workloads: bin-pack one draw of instances across the ranks (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif WORKLOADS[args.workload].get("closure"):
        run_batch_closure_arm(args)
    elif "batch" in WORKLOADS[args.workload]:
        run_batch_arm(args)
    else:
        run_cuda_arm(args)


if __name__ == "__main__":
    main()
