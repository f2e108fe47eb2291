"""Training of the learned warm start (no counterpart in the reference).

The plain contact solve, run to a relative residual, generates the data: for
every active contact of every tick, the 16 network inputs recorded at the
start of the solve and the converged impulse x D (D the impulse denominator
along the normal) as the target.  The network (mk_op_mlp_*: bf16 tcgen05
kernels, f32 accumulation) is trained on the GPU with Adam on the mean
squared error of output 0.  The result is a parameter array for
GpuPhysics.set_warm_start_network.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .physics import GpuPhysics, GpuPhysicsConfig


def residual_config(tolerance: float = 1e-5, max_iterations: int = 512, learned: bool = False,
                    **kw) -> GpuPhysicsConfig:
    return GpuPhysicsConfig(contact_tolerance=tolerance, contact_max_iterations=max_iterations,
                            warm_start=abi.WARM_LEARNED if learned else abi.WARM_CACHED, **kw)


def collect_samples(scene, ticks: int, config: GpuPhysicsConfig | None = None, capacities=None,
                    params: np.ndarray | None = None):
    """Steps `scene` for `ticks` ticks with the plain (or, with params, the learned) solve to
    a residual and returns (inputs (n, 16) float32, targets (n,) float32, passes per tick)."""
    cfg = config or residual_config(learned=params is not None)
    feats, targs, passes = [], [], []
    with GpuPhysics(scene, cfg, capacities=capacities) as gpu:
        if params is not None:
            gpu.set_warm_start_network(params)
        for t in range(1, ticks + 1):
            gpu.dispatch_tick(t)
            rb = gpu.read_last_tick()
            passes.append(rb.contact_iterations)
            f, y = gpu.warm_start_samples()
            feats.append(f)
            targs.append(y)
    return np.concatenate(feats), np.concatenate(targs), np.asarray(passes)


def train(inputs: np.ndarray, targets: np.ndarray, steps: int = 3000, batch: int = 8192, lr: float = 2e-3,
          seed: int = 0, params: np.ndarray | None = None):
    """Trains the warm-start network on the GPU; returns (params, per-step losses)."""
    import torch

    from . import ops
    from .net_init import init_params

    rng = np.random.default_rng(seed)
    order = rng.permutation(len(inputs))
    x = np.zeros((len(inputs), 16), np.float32)
    x[:] = inputs[order]
    t = np.zeros((len(inputs), 16), np.float32)
    t[:, 0] = targets[order]
    w = np.zeros(16, np.float32)
    w[0] = 1.0
    p = torch.from_numpy(params if params is not None else init_params(seed)).cuda()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    xs, ts, ws = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    losses = ops.mlp_train(p, m, v, xs, ts, ws, steps=steps, batch=min(batch, len(x)), lr=lr)
    return p.cpu().numpy(), losses.cpu().numpy()
