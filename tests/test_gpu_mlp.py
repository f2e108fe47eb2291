"""The tcgen05 network kernels against the CPU restatement (oracle/mlp.py).

Both sides round weights, inputs and activations to bf16 at the same points
and accumulate in f32, so they differ only in the f32 summation order of the
tensor cores: outputs agree to a relative 1e-3 of their scale, gradients to a
relative 1e-2 per parameter block (a bf16 rounding flip of one activation is
one part in 256 of that activation).
"""
import numpy as np
import pytest
import torch

from mechanic_b200 import ops
from oracle import mlp

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 16)).astype(np.float32)
    t = np.zeros((n, 16), np.float32)
    t[:, 0] = np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2]
    t[:, 1] = np.abs(x[:, 3]) - 0.3
    t[:, 2] = np.tanh(x[:, 4] + x[:, 5])
    w = np.zeros(16, np.float32)
    w[:3] = [1.0, 0.5, 2.0]
    return x, t, w


def _params(seed=0):
    p = mlp.init_params(seed, out_scale=1.0)
    rng = np.random.default_rng(seed + 100)
    p[mlp.B2:mlp.B3] = rng.normal(0, 0.1, 64)
    p[mlp.B3:mlp.PARAMS] = rng.normal(0, 0.1, 16)
    return p


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40000])
def test_forward_matches_oracle(cuda_lib, n):
    x, _, _ = _data(n)
    p = _params()
    y = ops.mlp_forward(torch.from_numpy(p).cuda(), torch.from_numpy(x).cuda(), y_cols=16).cpu().numpy()
    ref, _ = mlp.forward(p, x)
    scale = np.abs(ref).max() + 1e-6
    assert np.abs(y - ref).max() <= 1e-3 * scale


@pytest.mark.parametrize("n", [128, 1000, 50000])
def test_gradient_matches_oracle(cuda_lib, n):
    x, t, w = _data(n, seed=1)
    p = _params(1)
    g, loss = ops.mlp_gradient(torch.from_numpy(p).cuda(), torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(),
                               torch.from_numpy(w).cuda())
    g = g.cpu().numpy().astype(np.float64)
    ref, ref_loss = mlp.gradient(p, x, t, w)
    assert float(loss) == pytest.approx(ref_loss, rel=1e-4)
    for lo, hi, name in ((mlp.W1, mlp.W2, "W1"), (mlp.W2, mlp.W3, "W2"), (mlp.W3, mlp.B2, "W3"),
                         (mlp.B2, mlp.B3, "b2"), (mlp.B3, mlp.PARAMS, "b3")):
        err = np.linalg.norm(g[lo:hi] - ref[lo:hi]) / (np.linalg.norm(ref[lo:hi]) + 1e-12)
        assert err <= 1e-2, (name, err)


def test_gradient_is_deterministic(cuda_lib):
    x, t, w = _data(30000, seed=2)
    p = torch.from_numpy(_params(2)).cuda()
    args = (torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda())
    g1, _ = ops.mlp_gradient(p, *args)
    g2, _ = ops.mlp_gradient(p, *args)
    assert torch.equal(g1, g2)


def test_training_reduces_the_loss(cuda_lib):
    x, t, w = _data(65536, seed=3)
    p = torch.from_numpy(mlp.init_params(3)).cuda()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    xs, ts, ws = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda()
    _, before = ops.mlp_gradient(p, xs, ts, ws)
    losses = ops.mlp_train(p, m, v, xs, ts, ws, steps=400, batch=8192, lr=3e-3)
    _, after = ops.mlp_gradient(p, xs, ts, ws)
    assert float(after) < 0.2 * float(before), (float(before), float(after), losses[-5:].tolist())
    assert int(ops.MlpWorkspace(1).flags.item()) == 0
