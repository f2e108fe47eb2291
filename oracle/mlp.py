"""CPU restatement of the learned parts' network (test infrastructure only).

The network of mechanic_b200/csrc/mk_mlp.cu: 16 inputs (slot 15 replaced by
the constant 1 that carries the first layer's bias), two ReLU layers of 64,
16 outputs,

    h1 = relu(W1 x),  h2 = relu(W2 h1 + b2),  y = W3 h2 + b3,

with the loss L = (1/n) sum_s sum_o w_o (y_so - t_so)^2.  The reference has
no learned parts, so this restatement is pinned by finite differences (in
float64 without rounding) and used as the checker of the GPU kernels, whose
arithmetic it mirrors: with `bf16=True` the weights, the inputs, h1, h2, dY,
dH2 and dH1 are rounded to bf16 (nearest even) at the same points as the
kernels, and products are accumulated in float32.
"""
from __future__ import annotations

import numpy as np

W1, W2, W3, B2, B3, PARAMS = 0, 1024, 5120, 6144, 6208, 6224


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bf16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    return (p[W1:W2].reshape(64, 16), p[W2:W3].reshape(64, 64), p[W3:B2].reshape(16, 64), p[B2:B3], p[B3:PARAMS])


def init_params(seed: int = 0, out_scale: float = 0.1) -> np.ndarray:
    """He-style initialisation; the first-layer bias (W1 column 15) and b2 start at 0."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    w1 = rng.normal(0, np.sqrt(2.0 / 15), (64, 16)).astype(np.float32)
    w1[:, 15] = 0.0
    p[W1:W2] = w1.ravel()
    p[W2:W3] = rng.normal(0, np.sqrt(2.0 / 64), (64, 64)).astype(np.float32).ravel()
    p[W3:B2] = (rng.normal(0, np.sqrt(1.0 / 64), (16, 64)) * out_scale).astype(np.float32).ravel()
    return p


def _inputs(x, dtype):
    x = np.array(x, dtype=dtype, copy=True)
    x[:, 15] = 1.0
    return x


def forward(p, x, bf16_round: bool = True):
    w1, w2, w3, b2, b3 = unpack(p)
    f = bf16 if bf16_round else (lambda a: a)
    dt = np.float32 if bf16_round else np.float64
    xs = f(_inputs(x, dt))
    w1, w2, w3 = f(w1.astype(dt)), f(w2.astype(dt)), f(w3.astype(dt))
    a1 = xs @ w1.T
    h1 = f(np.maximum(a1, 0))
    a2 = h1 @ w2.T + b2.astype(dt)
    h2 = f(np.maximum(a2, 0))
    y = h2 @ w3.T + b3.astype(dt)
    return y, (xs, w1, w2, w3, a1, h1, a2, h2)


def gradient(p, x, t, w_out, bf16_round: bool = True):
    """Returns (gradient with the parameter layout, loss)."""
    f = bf16 if bf16_round else (lambda a: a)
    dt = np.float32 if bf16_round else np.float64
    y, (xs, w1, w2, w3, a1, h1, a2, h2) = forward(p, x, bf16_round)
    n = len(x)
    t = np.asarray(t, dt)
    w_out = np.asarray(w_out, dt)
    e = y - t
    loss = float((w_out * e * e).sum() / n)
    dy = f((dt(2.0) / dt(n)) * w_out * e) if bf16_round else 2.0 / n * w_out * e
    dh2 = f((dy @ w3) * (a2 > 0))
    dh1 = f((dh2 @ w2) * (a1 > 0))
    g = np.zeros(PARAMS, np.float64)
    g[W1:W2] = (dh1.T @ xs).ravel()
    g[W2:W3] = (dh2.T @ h1).ravel()
    g[W3:B2] = (dy.T @ h2).ravel()
    g[B2:B3] = dh2.sum(0)
    g[B3:PARAMS] = dy.sum(0)
    return g, loss


def loss_only(p, x, t, w_out):
    y, _ = forward(p, x, bf16_round=False)
    return float((np.asarray(w_out) * (y - t) ** 2).sum() / len(x))
