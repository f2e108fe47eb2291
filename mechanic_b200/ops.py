"""Stream-ordered device operations of libmechanic_b200 on torch CUDA tensors.

torch is used only for device memory and the current stream; the work runs
in the library's own kernels (mk_op_* in include/mechanic_b200.h).
"""
from __future__ import annotations

import torch

from .physics import _raise, library


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def sort_keys(keys: torch.Tensor, values: torch.Tensor, key_bits: int = 63):
    """Stable radix sort of int64-stored unsigned keys with int32-stored values
    (the LBVH sort of lbvh.wgsl:132-217).  Returns (sorted_keys, sorted_values)."""
    assert keys.is_cuda and values.is_cuda and keys.dtype == torch.int64 and values.dtype == torch.int32
    n = keys.numel()
    keys = keys.contiguous()
    values = values.contiguous()
    k_out = torch.empty_like(keys)
    v_out = torch.empty_like(values)
    if n == 0:
        return k_out, v_out
    L = library()
    need = int(L.mk_op_sort_scratch_bytes(n))   # sized for the widest (64-bit) keys, so any key_bits fits
    scratch = torch.empty(need + 256, dtype=torch.uint8, device=keys.device)
    base = scratch.data_ptr()
    aligned = (base + 255) & ~255
    _raise(L.mk_op_sort_keys(keys.data_ptr(), values.data_ptr(), k_out.data_ptr(), v_out.data_ptr(), n,
                             key_bits, aligned, need, _stream()))
    return k_out, v_out


def obb_sat(boxes_a: torch.Tensor, boxes_b: torch.Tensor):
    """Batched 15-axis OBB SAT (collision.wgsl:393-486).  Boxes are (N, 4, 4)
    float32: {center, hx}, {axis_x, hy}, {axis_y, hz}, {axis_z, -}.
    Returns (normal+penetration (N, 4) float32, feature words (N,) int32)."""
    assert boxes_a.shape == boxes_b.shape and boxes_a.shape[1:] == (4, 4)
    a = boxes_a.contiguous().float()
    b = boxes_b.contiguous().float()
    n = a.shape[0]
    out = torch.empty((n, 4), dtype=torch.float32, device=a.device)
    feat = torch.empty((n,), dtype=torch.int32, device=a.device)
    _raise(library().mk_op_obb_sat(a.data_ptr(), b.data_ptr(), n, out.data_ptr(), feat.data_ptr(), _stream()))
    return out, feat


# ----------------------------------------------------------- learned parts
MLP_INPUTS = 16
MLP_OUTPUTS = 16


def mlp_param_count() -> int:
    return int(library().mk_mlp_param_count())


class MlpWorkspace:
    """Scratch and error word for the network kernels on one device."""

    def __init__(self, max_samples: int, device="cuda"):
        L = library()
        need = int(L.mk_op_mlp_scratch_bytes(max(1, int(max_samples))))
        if need == 0:
            raise RuntimeError("mk_op_mlp_scratch_bytes failed: " + (L.mk_last_error() or b"").decode())
        self._buf = torch.empty(need + 256, dtype=torch.uint8, device=device)
        self.scratch = (self._buf.data_ptr() + 255) & ~255
        self.bytes = need
        self.flags = torch.zeros(1, dtype=torch.int32, device=device)


def _rows16(a: torch.Tensor) -> torch.Tensor:
    assert a.is_cuda and a.dtype == torch.float32 and a.dim() == 2 and a.shape[1] == 16
    return a.contiguous()


def mlp_forward(params: torch.Tensor, x: torch.Tensor, y_cols: int = 16, ws: MlpWorkspace | None = None):
    """net(x) for x (n, 16) float32 on the GPU; returns (n, y_cols)."""
    x = _rows16(x)
    n = x.shape[0]
    ws = ws or MlpWorkspace(n, x.device)
    y = torch.empty((n, y_cols), dtype=torch.float32, device=x.device)
    _raise(library().mk_op_mlp_forward(params.data_ptr(), x.data_ptr(), n, y.data_ptr(), y_cols, ws.scratch,
                                        ws.bytes, ws.flags.data_ptr(), _stream()))
    return y


def mlp_gradient(params: torch.Tensor, x: torch.Tensor, targets: torch.Tensor, out_weights: torch.Tensor,
                 ws: MlpWorkspace | None = None):
    """(gradient of the weighted mean squared error w.r.t. params, loss)."""
    x = _rows16(x)
    targets = _rows16(targets)
    n = x.shape[0]
    ws = ws or MlpWorkspace(n, x.device)
    grad = torch.empty(params.numel() + 1, dtype=torch.float32, device=x.device)
    _raise(library().mk_op_mlp_gradient(params.data_ptr(), x.data_ptr(), targets.data_ptr(),
                                         out_weights.contiguous().data_ptr(), n, grad.data_ptr(), ws.scratch,
                                         ws.bytes, ws.flags.data_ptr(), _stream()))
    return grad[:-1], grad[-1]


def mlp_train(params: torch.Tensor, adam_m: torch.Tensor, adam_v: torch.Tensor, x: torch.Tensor,
              targets: torch.Tensor, out_weights: torch.Tensor, steps: int, batch: int, lr: float,
              first_step: int = 0, ws: MlpWorkspace | None = None) -> torch.Tensor:
    """`steps` Adam steps in place on params (and its moments); returns the per-step batch losses."""
    x = _rows16(x)
    targets = _rows16(targets)
    n = x.shape[0]
    ws = ws or MlpWorkspace(min(n, batch), x.device)
    losses = torch.zeros(steps, dtype=torch.float32, device=x.device)
    _raise(library().mk_op_mlp_train(params.data_ptr(), adam_m.data_ptr(), adam_v.data_ptr(), x.data_ptr(),
                                      targets.data_ptr(), out_weights.contiguous().data_ptr(), n, batch, steps,
                                      float(lr), first_step, losses.data_ptr(), ws.scratch, ws.bytes,
                                      ws.flags.data_ptr(), _stream()))
    return losses
