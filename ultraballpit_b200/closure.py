"""Learned near-wall closure: the network handle (``sph_mlp_*`` in the C ABI).

``ClosureNet`` wraps the device network (16 -> 64 -> 64 -> 4, SiLU, BF16
tensor-core training and inference with FP32 accumulation, FP32 master
weights and Adam). Training data come from paired coarse / fine runs of the
WCSPH step (``closure_data``); the trained parameters are handed to a
``CudaKernel`` with ``set_closure`` for inference in the force stage.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .kernel import SPH_OK, SphError, _fp, load_library

N_IN, N_OUT, N_PARAMS = 16, 4, 5508


def _lib():
    L = load_library()
    if not getattr(L, "_mlp_bound", False):
        vp = C.c_void_p
        L.sph_mlp_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(vp)]
        L.sph_mlp_destroy.argtypes = [vp]
        L.sph_mlp_destroy.restype = None
        L.sph_mlp_set_params.argtypes = [vp, C.POINTER(C.c_float)]
        L.sph_mlp_get_params.argtypes = [vp, C.POINTER(C.c_float)]
        L.sph_mlp_forward.argtypes = [vp, C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_float)]
        L.sph_mlp_loss_grad.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t,
                                        C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.sph_mlp_train.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t, C.c_int,
                                    C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float)]
        for f in ("sph_mlp_create", "sph_mlp_set_params", "sph_mlp_get_params", "sph_mlp_forward",
                  "sph_mlp_loss_grad", "sph_mlp_train"):
            getattr(L, f).restype = C.c_int
        L._mlp_bound = True
    return L


def _chk(st, what):
    if st != SPH_OK:
        raise SphError(st, what)


class ClosureNet:
    """The closure network on one device."""

    def __init__(self, seed: int = 0, device: int = 0):
        self._lib = _lib()
        h = C.c_void_p()
        _chk(self._lib.sph_mlp_create(device, seed, C.byref(h)), "sph_mlp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.sph_mlp_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        _chk(self._lib.sph_mlp_get_params(self._h, _fp(p)), "sph_mlp_get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.shape == (N_PARAMS,)
        _chk(self._lib.sph_mlp_set_params(self._h, _fp(p)), "sph_mlp_set_params")

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], N_OUT), np.float32)
        _chk(self._lib.sph_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)), "sph_mlp_forward")
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_float()
        g = np.zeros(N_PARAMS, np.float32)
        _chk(self._lib.sph_mlp_loss_grad(self._h, _fp(x), _fp(t), x.shape[0], C.byref(loss), _fp(g)),
             "sph_mlp_loss_grad")
        return float(loss.value), g

    def train(self, x, t, batch: int = 1024, epochs: int = 20, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(epochs, np.float32)
        _chk(self._lib.sph_mlp_train(self._h, _fp(x), _fp(t), x.shape[0], batch, epochs, lr, seed, _fp(losses)),
             "sph_mlp_train")
        return losses


# ---------------------------------------------------------------------------
# Paired coarse / fine runs -> training samples
# ---------------------------------------------------------------------------

RHO0, G = 1000.0, 9.81
FILL = 0.16  # 40 layers at 4 mm, 80 at 2 mm
SETTLE_S = 0.05  # kinetic-damping relaxation before every paired run
TANK = (0.1, 0.1, 0.2)
ALPHA = 0.02


def tank_pair(seed: int, dx_coarse: float = 0.004, fill: float = FILL, alpha: float = ALPHA):
    """Hydrostatic tank 0.1 x 0.1 x 0.2 m filled to ``fill`` (a multiple of
    both spacings, so both runs hold the same water) around a fixed sphere
    of seeded radius in [0.01, 0.03] m at a seeded submerged position, at dx
    and dx / 2; fluid, walls and sphere on one lattice (``tank_with_sphere``
    with ``geometry="lattice"``). The seed also draws the speed U in
    [0, 0.5] m/s the moving variant starts with (``settled_pair``)."""
    from . import domain
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.01, 0.03)
    m = r + 0.008
    c = (rng.uniform(m, TANK[0] - m), rng.uniform(m, TANK[1] - m), rng.uniform(m, fill - m))
    speed = rng.uniform(0.0, 0.5)
    out = []
    for dx in (dx_coarse, dx_coarse / 2):
        sc = domain.tank_with_sphere(dx, domain_max=TANK, center=c, radius=r, fill_height=fill, seed=seed,
                                     alpha=alpha, hydrostatic=True, geometry="lattice")
        out.append(sc)
    return out[0], out[1], dict(center=c, radius=r, speed=speed)


def settle(sc, seconds: float = 0.05, dt: float = 5e-5, every: int = 20, device: int = 0):
    """Kinetic-damping relaxation of the initial lattice: ``seconds`` of
    steps of ``dt`` with every velocity zeroed after each ``every`` steps.
    The Cartesian lattice does not conform to the sphere, so its first shell
    sits anywhere in [0, dx) from the surface and starts tens of kPa off
    equilibrium; the relaxation lets it find the equilibrium of the wall
    model before the run. Returns a copy of ``sc`` with the relaxed
    positions and zero velocity."""
    import dataclasses
    k = _kernel(sc, device)
    for s in range(int(round(seconds / dt))):
        k.step(dt)
        if (s + 1) % every == 0:
            k.scale_velocities(0.0)
    p = k.particles()
    k.health()
    k.close()
    q = sc.particles.copy()
    q.x[:], q.y[:], q.z[:] = p.x, p.y, p.z
    q.vx[:] = q.vy[:] = q.vz[:] = np.float32(0.0)
    q.density[:], q.pressure[:] = p.density, p.pressure
    return dataclasses.replace(sc, particles=q)


# Wall treatment of the closure tanks: "particles" (the reference's wall and
# geometry boundary particles with Adami pressure) or "sdf" (the homogenised
# SDF wall layers). The merged SDF gives the closure features either way.
WALLS = "particles"


def _kernel(sc, device=0, walls=None):
    from .kernel import BOUNDARY_SDF, CudaKernel
    if (walls or WALLS) == "sdf":
        return CudaKernel(*sc.kernel_args(), alpha=sc.alpha, device=device, boundary_mode=BOUNDARY_SDF,
                          sdf=sc.obstacle_sdf)
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, device=device)
    k.set_feature_sdf(sc.sdf)
    return k


def settled_pair(seed: int, dx_coarse: float = 0.004, dt_coarse: float = 5e-5, settle_s: float = SETTLE_S,
                 device: int = 0, moving: bool = False):
    """tank_pair with both tanks relaxed (``settle``) for ``settle_s``; with
    ``moving`` the water then starts at the seed's speed along +x."""
    coarse_sc, fine_sc, geo = tank_pair(seed, dx_coarse)
    if settle_s > 0:
        coarse_sc = settle(coarse_sc, settle_s, dt_coarse, device=device)
        fine_sc = settle(fine_sc, settle_s, dt_coarse / 2, device=device)
    if moving:
        for sc in (coarse_sc, fine_sc):
            sc.particles.vx[:] = np.float32(geo["speed"])
    return coarse_sc, fine_sc, geo


def run_pair(seed: int, t_snap=(0.02, 0.03, 0.04, 0.05), dt_coarse: float = 5e-5, device: int = 0,
             dx_coarse: float = 0.004, settle_s: float = SETTLE_S, moving: bool = False):
    """Samples (features, targets) of one settled tank pair at the snapshot
    times (seconds after the relaxation).

    Targets in physical units: (p_f(x) - p_c(x), a_f(x) - a_c(x)), Pa and
    m/s^2, with both runs Shepard-interpolated at the coarse sample
    positions x at the same time (the fine run at dx / 2, dt / 2):
    smoothing the coarse side too removes the sample particle's own noise,
    which no feature can predict. Returned in network units (``to_units``)."""
    coarse_sc, fine_sc, geo = settled_pair(seed, dx_coarse, dt_coarse, settle_s, device, moving)
    kc, kf = _kernel(coarse_sc, device), _kernel(fine_sc, device)
    kc.set_closure(1)
    X, T, step = [], [], 0
    for t in t_snap:
        n = int(round(t / dt_coarse))
        while step < n:
            kc.step(dt_coarse)
            kf.step(dt_coarse / 2)
            kf.step(dt_coarse / 2)
            step += 1
        ids, feat, rho_pre = kc.closure_samples()
        pc = kc.particles()
        pts = np.stack([pc.x[ids], pc.y[ids], pc.z[ids]], axis=1)
        fine = kf.interpolate(pts)
        crs = kc.interpolate(pts)
        ok = (fine[:, 6] > 0) & (crs[:, 6] > 0)
        tgt = np.concatenate([(fine[:, 1] - crs[:, 1])[:, None], fine[:, 2:5] - crs[:, 2:5]], axis=1)
        X.append(feat[ok])
        T.append(to_units(tgt[ok], coarse_sc.speed_of_sound))
    kc.close()
    kf.close()
    return np.concatenate(X), np.concatenate(T)


def generate(seeds, moving=False, **kw):
    """Samples of ``run_pair`` over ``seeds``; ``moving`` is a bool or a
    function of the seed (True: the tank starts at the seed's speed)."""
    xs, ts, owners = [], [], []
    for s in seeds:
        x, t = run_pair(s, moving=bool(moving(s) if callable(moving) else moving), **kw)
        xs.append(x)
        ts.append(t)
        owners.append(np.full(len(x), s))
    return np.concatenate(xs), np.concatenate(ts), np.concatenate(owners)


# Output units and clamps of the step: y0 in SPH_CLOSURE_DRHO_UNIT rho0
# (clamped to SPH_CLOSURE_MAX_DRHO), y1..3 in |g| (SPH_CLOSURE_MAX_ACC_G).
DRHO_UNIT, CLAMP_DRHO, CLAMP_ACC_G = 1e-4, 30.0, 2.5


def to_units(raw, c: float) -> np.ndarray:
    """(dp [Pa], da [m/s^2]) -> network outputs: a density change of
    dp / c^2 (the Tait slope at rest) in units of DRHO_UNIT rho0, and
    accelerations in units of |g|."""
    raw = np.asarray(raw, np.float64)
    out = np.empty_like(raw)
    out[:, 0] = raw[:, 0] / (c * c * RHO0 * DRHO_UNIT)
    out[:, 1:] = raw[:, 1:] / G
    return out.astype(np.float32)


def prepare_targets(t, lo: float = 1.0, hi: float = 99.0) -> np.ndarray:
    """Winsorise each target column at its [lo, hi] percentiles, then clip it
    to the clamp the step applies to the network's outputs. Per-particle
    accelerations carry heavy-tailed particle noise; the fit wants the
    conditional mean, which the tails only disturb."""
    t = np.array(t, np.float32, copy=True)
    for j in range(t.shape[1]):
        a, b = np.percentile(t[:, j], [lo, hi])
        np.clip(t[:, j], a, b, out=t[:, j])
    np.clip(t[:, 0], -CLAMP_DRHO, CLAMP_DRHO, out=t[:, 0])
    np.clip(t[:, 1:], -CLAMP_ACC_G, CLAMP_ACC_G, out=t[:, 1:])
    return t


def split_by_tank(owners, frac: float = 0.1, seed: int = 0):
    """Boolean mask of the held-out samples: whole tanks (seeds), about
    ``frac`` of them, so the held-out loss measures unseen geometry."""
    tanks = np.unique(owners)
    rng = np.random.default_rng(seed)
    n_out = max(1, int(round(frac * len(tanks))))
    out = rng.choice(tanks, n_out, replace=False)
    return np.isin(owners, out)


def probe_points(geo, h: float, fill: float = FILL, tank=TANK, n_sphere: int = 256):
    """Fixed near-wall pressure probes at distance h from the geometry:
    a Fibonacci lattice on the sphere (radius r + h) and grids on the floor
    and the four side walls, each at least 2h from the other surfaces and
    below fill - 3h. Returns (sphere probes, wall probes)."""
    c = np.asarray(geo["center"], np.float64)
    r = float(geo["radius"])
    q = np.arange(n_sphere) + 0.5
    phi = np.arccos(1.0 - 2.0 * q / n_sphere)
    th = np.pi * (1.0 + 5.0 ** 0.5) * q
    dirs = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    sph = c + (r + h) * dirs
    lo = np.array([2 * h, 2 * h, 2 * h])
    hi = np.array([tank[0] - 2 * h, tank[1] - 2 * h, fill - 3 * h])
    sph = sph[np.all((sph >= lo) & (sph <= hi), axis=1)]
    gx = np.linspace(3 * h, tank[0] - 3 * h, 8)
    gy = np.linspace(3 * h, tank[1] - 3 * h, 8)
    gz = np.linspace(3 * h, fill - 4 * h, 5)
    pts = [np.array([(x, y, h) for x in gx for y in gy])]
    pts += [np.array([(h, y, z) for y in gy for z in gz]), np.array([(tank[0] - h, y, z) for y in gy for z in gz])]
    pts += [np.array([(x, h, z) for x in gx for z in gz]), np.array([(x, tank[1] - h, z) for x in gx for z in gz])]
    walls = np.concatenate(pts)
    walls = walls[np.linalg.norm(walls - c, axis=1) - r >= 2 * h]
    return sph.astype(np.float32), walls.astype(np.float32)


def _sphere_force(k, sc) -> np.ndarray:
    """Fluid force on the sphere: with boundary particles the FP64 reaction
    (pressure + repulsion) on the sphere's particles, which is a pairwise
    sum and so comparable across resolutions; in SDF wall mode the surface
    integral of force.rs, whose 2h node shell makes it scale with h."""
    ex = sc.extras
    if (WALLS == "particles") and ex.get("n_geometry_boundary", 0):
        f = k.body_force(ex["n_wall_boundary"], ex["n_geometry_boundary"])
        return np.asarray(f["pressure_force"]) + np.asarray(f["repulsion_force"])
    return k.surface_forces()["force"]


def run_probes(sc, probes, steps: int, dt: float, every: int, start: int, mode: int = 0, params=None,
               device: int = 0, substeps: int = 1):
    """Run ``sc`` for ``steps`` x ``substeps`` steps of dt / substeps and
    average the Shepard-interpolated pressure at ``probes`` and the surface
    force on the sphere over the snapshots start, start + every, ... (in
    units of dt). Returns (mean pressure, snapshot count per probe, mean
    force on the sphere, seconds spent stepping with the device synchronised
    on both sides)."""
    import time
    k = _kernel(sc, device)
    if mode:
        k.set_closure(mode, params)
    k.set_geometry_sdf(sc.extras["sphere_sdf"])
    acc = np.zeros(len(probes))
    cnt = np.zeros(len(probes), np.int64)
    forces, secs, s = [], 0.0, 0
    for target in range(start, steps + 1, every):
        k.synchronize()
        t0 = time.perf_counter()
        while s < target * substeps:
            k.step(dt / substeps)
            s += 1
        k.synchronize()
        secs += time.perf_counter() - t0
        out = k.interpolate(probes)
        ok = out[:, 6] > 0
        acc[ok] += out[ok, 1]
        cnt[ok] += 1
        forces.append(_sphere_force(k, sc))
    k.health()
    k.close()
    return acc / np.maximum(cnt, 1), cnt, np.mean(forces, axis=0), secs


def compare(seed: int, params=None, steps: int = 800, dt: float = 5e-5, every: int = 20, start: int | None = None,
            dx_coarse: float = 0.004, device: int = 0, settle_s: float = SETTLE_S, moving: bool = False) -> dict:
    """``compare_scenarios`` on the settled tank pair of ``seed``."""
    coarse, fine, geo = settled_pair(seed, dx_coarse, dt, settle_s, device, moving)
    out = compare_scenarios(coarse, fine, geo, params, steps, dt, every, start, device)
    out["seed"] = seed
    return out


def compare_scenarios(coarse, fine, geo, params=None, steps: int = 800, dt: float = 5e-5, every: int = 20,
                      start: int | None = None, device: int = 0, fill: float = FILL, tank=TANK) -> dict:
    """The fine tank (dx / 2, dt / 2) is the reference for the coarse tank without
    (``plain``) and, when ``params`` is given, with the closure
    (``closure``): near-wall pressure error = mean |p_c - p_f| / mean |p_f|
    over the probes on the sphere and on the walls, each pressure averaged
    over the snapshots of the second half of the run; force error =
    |F_c - F_f| / |F_f| for the time-averaged force on the sphere;
    ``speedup`` = fine stepping time / coarse stepping time."""
    start = steps // 2 if start is None else start
    sph, walls = probe_points(geo, coarse.h, fill=fill, tank=tank)
    probes = np.concatenate([sph, walls])
    ns = len(sph)
    pf, nf, ff, tf = run_probes(fine, probes, steps, dt, every, start, device=device, substeps=2)
    out = dict(geo=geo, fine_seconds=tf, fine_force=ff, probes=(ns, len(walls)))
    runs = [("plain", 1, None)] + ([("closure", 2, params)] if params is not None else [])
    for name, mode, prm in runs:
        pc, nc, fc, tc = run_probes(coarse, probes, steps, dt, every, start, mode=mode, params=prm, device=device)
        ok = (nc == nc.max()) & (nf == nf.max())
        res = {}
        for part, sel in (("sphere", slice(0, ns)), ("walls", slice(ns, None)), ("all", slice(None))):
            m = ok[sel]
            a, b = pc[sel][m], pf[sel][m]
            res[part] = float(np.mean(np.abs(a - b)) / max(np.mean(np.abs(b)), 1e-12)) if len(b) else float("nan")
        res["force"] = float(np.linalg.norm(fc - ff) / max(np.linalg.norm(ff), 1e-12))
        res["seconds"] = tc
        res["speedup"] = tf / max(tc, 1e-12)
        res["mean_p_coarse"], res["mean_p_fine"] = float(np.mean(pc[ok])), float(np.mean(pf[ok]))
        out[name] = res
    return out
