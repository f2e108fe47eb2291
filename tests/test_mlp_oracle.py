"""The network restatement (oracle/mlp.py) pinned by finite differences.

The learned parts have no reference counterpart, so the oracle's backward
pass is checked against central differences of its own float64 loss; the
GPU kernels are then checked against this oracle (tests/test_gpu_mlp.py).
"""
import numpy as np

from oracle import mlp


def _problem(seed=0, n=40):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 16))
    t = rng.normal(size=(n, 16))
    w = np.zeros(16)
    w[:3] = [1.0, 0.5, 2.0]
    p = mlp.init_params(seed, out_scale=1.0).astype(np.float64)
    p[mlp.B2:mlp.B3] = rng.normal(0, 0.1, 64)
    p[mlp.B3:mlp.PARAMS] = rng.normal(0, 0.1, 16)
    p[mlp.W1:mlp.W2].reshape(64, 16)[:, 15] = rng.normal(0, 0.1, 64)
    return p, x, t, w


def test_backward_matches_central_differences():
    p, x, t, w = _problem()
    g, loss = mlp.gradient(p, x, t, w, bf16_round=False)
    assert abs(loss - mlp.loss_only(p, x, t, w)) < 1e-12
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(0, 1024), 12), rng.choice(np.arange(1024, 5120), 12),
                          rng.choice(np.arange(5120, 6144), 12), rng.choice(np.arange(6144, 6224), 8),
                          np.arange(15, 1024, 16)[:6]])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp = mlp.loss_only(q, x, t, w)
        q[i] -= 2 * h
        lm = mlp.loss_only(q, x, t, w)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_unused_outputs_carry_no_gradient():
    p, x, t, w = _problem(1)
    g, _ = mlp.gradient(p, x, t, w, bf16_round=False)
    w3 = g[mlp.W3:mlp.B2].reshape(16, 64)
    assert np.all(w3[3:] == 0) and np.all(g[mlp.B3 + 3:mlp.PARAMS] == 0)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], np.float32)
    r = mlp.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -6)
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
