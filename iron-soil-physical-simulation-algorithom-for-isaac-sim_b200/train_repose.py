"""Train the learned repose proposal on config-3 pairs, on the GPU.

    python -m soilb200.train_repose --patches 20000 --steps 8000 --out weights.npz

Pairs (config 3): 20k seeded 128^2 patches of the reference's fractal
gradient noise (``workloads.fractal_perlin_noise``, seeds 0..19999) steepened
to 45-60 deg (``workloads.config3_patch``), each relaxed to the repose angle
by the plain sweep on the GPU (FP64: the reference's own arithmetic).  The network learns the height change of that relaxation in flux
form; forward and backward passes run in the library's tensor-core kernels,
PyTorch only keeps the Adam state.  The package ships the weights trained this
way as ``data/repose_net_c3.npz``.
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "repose_net_c3.npz"


def make_pairs(n: int, size: int = 128, seed0: int = 0, critical_angle_deg: float = 35.0,
               tolerance_m: float = 1e-8, dx: float = 0.05):
    """n (pre, post) pairs: config-3 patches (seeds seed0 .. seed0+n-1) and
    their plain-sweep relaxation (FP64, the reference's arithmetic), all
    relaxed on one resident grid (upload, sb_relax_full, download)."""
    from . import _lib, workloads
    from .grid import DeviceGrid
    pre = np.empty((n, size, size))
    post = np.empty((n, size, size))
    grid = DeviceGrid((size, size), dx, dx, precision="fp64")
    crit = float(np.tan(np.deg2rad(critical_angle_deg)))
    params = _lib.RelaxParams(float(dx), float(dx), crit, float(tolerance_m), 20000, 0)
    lib = _lib.load()
    try:
        for i in range(n):
            pre[i] = workloads.config3_patch(seed0 + i, n=size, dx=dx)
            grid.upload("b_eff", pre[i])
            st = _lib.RelaxStats()
            _lib.check(grid.ctx, lib.sb_relax_full(grid.ctx, params, st), "relax")
            if not st.converged:
                raise RuntimeError(f"training patch {seed0 + i} did not relax")
            post[i] = grid.download("b_eff")
    finally:
        grid.close()
    return pre, post


def train_schedule(net, pre, post, *, steps: int, batch: int, lr: float, dx: float,
                   critical_angle_deg: float, chunks: int = 4):
    """Adam with the learning rate stepped down over `chunks` equal phases."""
    from .learned import train
    stats = []
    for c in range(chunks):
        st = train(net, pre, post, dx=dx, dy=dx, critical_angle_deg=critical_angle_deg,
                   steps=max(1, steps // chunks), batch=batch, lr=lr * (0.5 ** c), seed=c)
        stats.append(st)
    return stats


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--patches", type=int, default=20000)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--angle", type=float, default=35.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", type=Path, default=DEFAULT_WEIGHTS)
    args = ap.parse_args(argv)
    from .learned import ReposeNet
    t0 = time.perf_counter()
    pre, post = make_pairs(args.patches, critical_angle_deg=args.angle)
    t1 = time.perf_counter()
    net = ReposeNet(seed=args.seed)
    stats = train_schedule(net, pre, post, steps=args.steps, batch=args.batch, lr=args.lr,
                           dx=0.05, critical_angle_deg=args.angle)
    t2 = time.perf_counter()
    args.out.parent.mkdir(parents=True, exist_ok=True)
    net.save(args.out)
    print(json.dumps({"patches": args.patches, "steps": args.steps, "batch": args.batch,
                      "pairs_s": t1 - t0, "train_s": t2 - t1,
                      "loss_first": stats[0].first_loss, "loss_last": stats[-1].last_loss,
                      "out": str(args.out)}))


if __name__ == "__main__":
    main()
