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


# ------------------------------------------------------- closure preconditioner
def closure_config(learned: bool = False, tolerance: float = 1e-5, max_iterations: int = 256,
                   preconditioner: int | None = None, **kw) -> GpuPhysicsConfig:
    """Closure PCG to a residual; the default preconditioner is per-loop block Jacobi, `learned`
    selects the network-corrected 2 x 2 blocks (whose own baseline is PRECOND_PAIR_BLOCKS)."""
    if preconditioner is None:
        preconditioner = abi.PRECOND_LEARNED if learned else abi.PRECOND_BLOCK_JACOBI
    return GpuPhysicsConfig(closure_mode=abi.CLOSURE_PCG_RESIDUAL, closure_tolerance=tolerance,
                            closure_max_iterations=max_iterations, preconditioner=preconditioner, **kw)


def block_targets(pd: np.ndarray, ad: np.ndarray, coord: np.ndarray, closure: np.ndarray, max_abs: float = 1e3):
    """Training targets of the preconditioner network from one Newton step's Jacobian columns:
    for each 2 x 2 block of consecutive closure coordinates, (t11, t12, t22) of S (A^-1)_bb S,
    A = J^T J of the block's loop component and S = diag(sqrt(diag A)).  Returns (targets
    (blocks, 3), valid mask); blocks of singular or badly scaled components are masked out."""
    coords = np.unique(coord)
    index = {int(c): i for i, c in enumerate(coords)}
    nq = len(coords)
    a = np.zeros((nq, nq))
    parent = list(range(nq))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for k in np.unique(closure):
        sl = np.nonzero(closure == k)[0]
        v = np.concatenate([pd[sl], ad[sl]], axis=1).astype(np.float64)
        ids = [index[int(c)] for c in coord[sl]]
        g = v @ v.T
        for x, i in enumerate(ids):
            for y, j in enumerate(ids):
                a[i, j] += g[x, y]
            parent[find(ids[0])] = find(i)
    comps: dict[int, list[int]] = {}
    for i in range(nq):
        comps.setdefault(find(i), []).append(i)
    inv = np.zeros((nq, nq))
    ok = np.zeros(nq, bool)
    for members in comps.values():
        sub = a[np.ix_(members, members)]
        dg = np.sqrt(np.maximum(np.diag(sub), 1e-300))
        nrm = sub / np.outer(dg, dg)
        if np.any(np.diag(sub) <= 1e-12) or np.linalg.cond(nrm) > 1e8:
            continue
        inv[np.ix_(members, members)] = np.linalg.inv(nrm)
        ok[members] = True
    nb = (nq + 1) // 2
    t = np.zeros((nb, 3), np.float32)
    valid = np.zeros(nb, bool)
    for b in range(nb):
        i, j = 2 * b, 2 * b + 1
        if j < nq:
            blk = (inv[i, i], inv[i, j], inv[j, j])
            valid[b] = ok[i] and ok[j] and inv[i, i] > 0 and inv[j, j] > 0
        else:
            blk = (inv[i, i], 0.0, 0.0)
            valid[b] = ok[i] and inv[i, i] > 0
        t[b] = blk
        if valid[b] and np.max(np.abs(blk)) > max_abs:
            valid[b] = False
    return t, valid


def output_targets(blocks: np.ndarray) -> np.ndarray:
    """(t11, t12, t22) -> the network's outputs (log t11, log t22, atanh(t12 / 0.999 sqrt(t11 t22)))."""
    t11 = np.maximum(blocks[:, 0], 1e-30)
    t22 = np.maximum(blocks[:, 2], 1e-30)
    c = np.clip(blocks[:, 1] / (0.999 * np.sqrt(t11 * t22)), -0.999, 0.999)
    return np.stack([np.log(t11), np.log(t22), np.arctanh(c)], 1).astype(np.float32)


def collect_closure_samples(scene, ticks: int, config: GpuPhysicsConfig | None = None, params=None):
    """(inputs (n, 16), targets (n, 3), PCG iterations per tick) from `ticks` ticks."""
    cfg = config or closure_config(learned=params is not None,
                                   preconditioner=None if params is not None else abi.PRECOND_PAIR_BLOCKS)
    xs, ts, its = [], [], []
    with GpuPhysics(scene, cfg) as gpu:
        if params is not None:
            gpu.set_preconditioner_network(params)
        for t in range(1, ticks + 1):
            gpu.dispatch_tick(t)
            its.append(gpu.read_last_tick().closure_iterations)
            pd, ad, coord, closure = gpu.closure_slots()
            feats = gpu.closure_blocks()
            targ, valid = block_targets(pd, ad, coord, closure)
            valid &= feats[:, 7] > 0   # pair blocks with a partner
            xs.append(feats[valid])
            ts.append(targ[valid])
    return np.concatenate(xs), np.concatenate(ts), np.asarray(its)


def train_preconditioner(inputs: np.ndarray, targets: np.ndarray, steps: int = 4000, batch: int = 8192,
                         lr: float = 2e-3, seed: int = 0):
    """Trains the preconditioner network on the GPU; returns (params, losses)."""
    import torch

    from . import ops
    from .net_init import init_params

    rng = np.random.default_rng(seed)
    order = rng.permutation(len(inputs))
    x = np.ascontiguousarray(inputs[order], np.float32)
    t = np.zeros((len(inputs), 16), np.float32)
    t[:, :3] = output_targets(targets[order])
    w = np.zeros(16, np.float32)
    w[:3] = 1.0
    p = torch.from_numpy(init_params(seed)).cuda()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    losses = ops.mlp_train(p, m, v, torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda(),
                           steps=steps, batch=min(batch, len(x)), lr=lr)
    return p.cpu().numpy(), losses.cpu().numpy()
