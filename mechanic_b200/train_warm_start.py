"""Trains the learned contact warm start and writes its parameters.

  python -m mechanic_b200.train_warm_start --out mechanic_b200/data/warm_start.npy

Samples: every active contact of the plain contact solve run to a 1e-5
relative residual along the trajectories of the 1,000-cube config (seeds
given by --seeds, never seed 0, which the benchmark and tests measure);
inputs at the start of each tick's solve, targets the converged impulses.
The 100,000-body config is not used: its overlapping start makes the
relaxed-Jacobi solve diverge when it is iterated to a residual.  Training
runs on the GPU (bf16 tcgen05 kernels, Adam).
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import learned, scenes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "data", "warm_start.npy"))
    ap.add_argument("--seeds", default="1,2,3,4,5,6,7,8")
    ap.add_argument("--ticks", type=int, default=60)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--max-samples", type=int, default=4_000_000)
    args = ap.parse_args()
    rng = np.random.default_rng(0)
    xs, ys = [], []
    t0 = time.time()
    for seed in (int(s) for s in args.seeds.split(",")):
        for scene, caps in ((scenes.falling_cubes(1000, seed=seed), None),):
            x, y, passes = learned.collect_samples(scene, args.ticks, capacities=caps)
            if len(x) > args.max_samples // 4:
                keep = rng.choice(len(x), args.max_samples // 4, replace=False)
                x, y = x[keep], y[keep]
            xs.append(x)
            ys.append(y)
            print(f"{scene.name} seed {seed}: {len(x)} samples, plain passes/tick {passes.mean():.1f} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    params, losses = learned.train(x, y, steps=args.steps, batch=8192, lr=2e-3)
    print(f"trained on {len(x)} samples: loss {losses[:20].mean():.4f} -> {losses[-200:].mean():.4f}", flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.save(args.out, params.astype(np.float32))
    print("wrote", args.out)


if __name__ == "__main__":
    main()
