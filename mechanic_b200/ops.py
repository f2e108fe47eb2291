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
    need = int(L.mk_op_sort_scratch_bytes(n)) if key_bits == 63 else None
    if need is None:
        need = int(L.mk_op_sort_scratch_bytes(n))
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
