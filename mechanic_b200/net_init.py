"""Initial parameters of the learned parts' network (layout of mk_mlp_param_count)."""
from __future__ import annotations

import numpy as np

W1, W2, W3, B2, B3, PARAMS = 0, 1024, 5120, 6144, 6208, 6224


def init_params(seed: int = 0, out_scale: float = 0.1) -> np.ndarray:
    """He-normal weights; the first-layer bias (W1 column 15), b2 and b3 start at 0."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    w1 = rng.normal(0, np.sqrt(2.0 / 15), (64, 16)).astype(np.float32)
    w1[:, 15] = 0.0
    p[W1:W2] = w1.ravel()
    p[W2:W3] = rng.normal(0, np.sqrt(2.0 / 64), (64, 64)).astype(np.float32).ravel()
    p[W3:B2] = (rng.normal(0, np.sqrt(1.0 / 64), (16, 64)) * out_scale).astype(np.float32).ravel()
    return p
