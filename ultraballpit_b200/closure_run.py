"""Train the near-wall closure on paired tank runs and evaluate it.

    python -m ultraballpit_b200.closure_run --seeds 64 --epochs 20 --out DIR

1. ``closure.generate``: for each seed a settled hydrostatic tank
   0.1 x 0.1 x 0.2 m (fill 0.16 m) around a sphere of seeded radius
   (0.01-0.03 m) and position, run at dx = 4 mm and 2 mm; features of the
   coarse particles within 2h of the geometry and the smoothed fine - coarse
   pressure / acceleration offsets at ``--snapshots`` times. Odd seeds start
   moving at the seed's speed (0-0.5 m/s), so the inputs span the flows the
   closure is applied to (``--static-only`` trains on tanks at rest).
2. About ``--holdout`` of the tanks (whole seeds) are held out; the network
   (16-64-64-4 SiLU, BF16 tensor-core kernels, FP32 master weights) is
   trained with Adam at ``--lr`` for ``--epochs`` epochs on the rest.
3. A priori: held-out loss of the network, of the zero correction (the
   plain method) and of the best constant.
4. A posteriori: ``closure.compare`` on unseen tanks, static and moving
   (the seed's speed along +x), with and without the closure.

Writes ``DIR/closure_weights.npy`` (5,508 float32) and ``DIR/report.json``.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import closure


def _round(d):
    return {k: (round(v, 5) if isinstance(v, float) else v) for k, v in d.items()}


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--seeds", type=int, default=64)
    ap.add_argument("--first-seed", type=int, default=0)
    ap.add_argument("--snapshots", type=int, default=6, help="snapshots 0.01 s apart after the relaxation")
    ap.add_argument("--static-only", action="store_true",
                    help="train on tanks at rest only (default: odd seeds start moving)")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--holdout", type=float, default=0.1)
    ap.add_argument("--eval-seeds", type=int, default=4, help="unseen tanks per a-posteriori case")
    ap.add_argument("--eval-steps", type=int, default=800)
    ap.add_argument("--dt", type=float, default=5e-5)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=".")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    rep: dict = dict(config=vars(a))

    t0 = time.perf_counter()
    snaps = tuple(0.01 * (q + 1) for q in range(a.snapshots))
    x, t, own = closure.generate(range(a.first_seed, a.first_seed + a.seeds), dx_coarse=0.004, dt_coarse=a.dt,
                                 t_snap=snaps, device=a.device,
                                 moving=(lambda s: False) if a.static_only else (lambda s: s % 2 == 1))
    rep["generate_s"] = time.perf_counter() - t0
    rep["samples"] = int(len(x))
    tp = closure.prepare_targets(t)
    hold = closure.split_by_tank(own, a.holdout, seed=0)
    rep["held_out_tanks"] = sorted(int(s) for s in np.unique(own[hold]))
    rep["train_samples"], rep["held_out_samples"] = int((~hold).sum()), int(hold.sum())
    rep["target_mean"] = tp[~hold].mean(0).tolist()
    rep["target_std"] = tp[~hold].std(0).tolist()

    net = closure.ClosureNet(seed=1, device=a.device)
    t0 = time.perf_counter()
    losses = net.train(x[~hold], tp[~hold], batch=a.batch, epochs=a.epochs, lr=a.lr, seed=2)
    rep["train_s"] = time.perf_counter() - t0
    rep["epoch_loss"] = [float(v) for v in losses]
    l_net, _ = net.loss_grad(x[hold], tp[hold])
    th = tp[hold].astype(np.float64)
    rep["held_out_loss"] = dict(network=float(l_net), zero=float(np.mean(th ** 2)),
                                constant=float(np.mean((th - tp[~hold].mean(0)) ** 2)))
    np.save(os.path.join(a.out, "closure_weights.npy"), net.params())

    rep["a_posteriori"] = []
    base = a.first_seed + a.seeds + 1000
    for moving in (False, True):
        for s in range(base, base + a.eval_seeds):
            r = closure.compare(s, net.params(), steps=a.eval_steps, dt=a.dt, moving=moving, device=a.device)
            rep["a_posteriori"].append(dict(seed=s, moving=moving, speed=float(r["geo"]["speed"]),
                                            radius=float(r["geo"]["radius"]), plain=_round(r["plain"]),
                                            closure=_round(r["closure"]), fine_seconds=r["fine_seconds"]))
    for moving in (False, True):
        rows = [q for q in rep["a_posteriori"] if q["moving"] == moving]
        key = "moving" if moving else "static"
        rep[key] = {arm: {m: float(np.mean([q[arm][m] for q in rows])) for m in ("all", "sphere", "walls", "force")}
                    for arm in ("plain", "closure")}
    with open(os.path.join(a.out, "report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps({k: rep[k] for k in ("samples", "held_out_loss", "static", "moving", "generate_s", "train_s")}))
    return rep


if __name__ == "__main__":
    main()
