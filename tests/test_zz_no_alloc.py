"""The allocation-free sort entry point against the allocating one.

Callers that cannot allocate device memory when they need a sort (allocator
and memory-pool hooks that must not recurse into the allocator, embedders
with a fixed memory budget) use mk_op_sort_keys_static, whose scratch is a
static device array inside the library.  This file checks it through the C ABI against mk_op_sort_keys,
which takes scratch from the caller, on calls in a row: the static array
keeps whatever the previous call left in it, so each call must clear what it
needs.  Integer keys and indices: the tolerance is exact equality.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from mechanic_b200 import abi

pytestmark = pytest.mark.gpu

MAX_KEYS = 524288   # MK_STATIC_SORT_MAX_KEYS in include/mechanic_b200.h


def _keys(rng, n):
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    keys[: n // 4] = keys[0]                 # a long run of equal keys: order must follow the values
    keys[n // 2: n // 2 + 100] = 7
    return keys


# (keys, key bits) of consecutive calls.  Each call inherits the array the one
# before it left: larger-to-smaller runs on the onesweep path (more than 4,096
# keys) leave stale look-back words and histograms behind, a 24-bit call (three
# digit passes) after 63-bit ones (eight) leaves stale words of passes it does
# not run, and the last, small call takes the one-block path.
CALLS = ((300_001, 63), (MAX_KEYS, 63), (20_001, 63), (MAX_KEYS, 24), (20_001, 24), (1_000, 63))


def test_static_sort_matches_allocating_sort_on_calls_in_a_row(cuda_lib):
    import torch
    from mechanic_b200 import ops, physics
    lib = physics.library()
    rng = np.random.default_rng(12)
    stream = torch.cuda.current_stream().cuda_stream
    for n, bits in CALLS:
        keys_np = _keys(rng, n) & np.uint64((1 << bits) - 1)
        vals_np = rng.permutation(n).astype(np.uint32)
        keys = torch.from_numpy(keys_np.view(np.int64)).cuda()
        vals = torch.from_numpy(vals_np.view(np.int32)).cuda()
        k_static = torch.full_like(keys, -1)
        v_static = torch.full_like(vals, -1)
        rc = lib.mk_op_sort_keys_static(keys.data_ptr(), vals.data_ptr(), k_static.data_ptr(), v_static.data_ptr(),
                                        n, bits, stream)
        assert rc == abi.MK_OK, lib.mk_last_error()
        k_alloc, v_alloc = ops.sort_keys(keys, vals, key_bits=bits)
        torch.cuda.synchronize()
        assert torch.equal(k_static, k_alloc), f"keys differ for n={n}, {bits} bits"
        assert torch.equal(v_static, v_alloc), f"values differ for n={n}, {bits} bits"
        order = np.argsort(keys_np, kind="stable")
        assert np.array_equal(k_static.cpu().numpy().view(np.uint64), keys_np[order])
        assert np.array_equal(v_static.cpu().numpy().view(np.uint32), vals_np[order])


def test_static_sort_rejects_more_keys_than_its_array_holds(cuda_lib):
    import torch
    from mechanic_b200 import physics
    lib = physics.library()
    n = MAX_KEYS + 1
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    vals = torch.zeros(n, dtype=torch.int32, device="cuda")
    out_k = torch.full_like(keys, 5)
    out_v = torch.full_like(vals, 5)
    rc = lib.mk_op_sort_keys_static(keys.data_ptr(), vals.data_ptr(), out_k.data_ptr(), out_v.data_ptr(), n, 63,
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == abi.MK_ERR_INVALID_ARGUMENT
    assert b"exceed" in lib.mk_last_error()
    assert bool((out_k == 5).all()) and bool((out_v == 5).all())   # nothing was written


def test_static_sort_rejects_overlapping_input_and_output(cuda_lib):
    import torch
    from mechanic_b200 import physics
    lib = physics.library()
    n = 10_000
    keys = torch.arange(n, 0, -1, dtype=torch.int64, device="cuda")
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    out_v = torch.full_like(vals, 5)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.mk_op_sort_keys_static(keys.data_ptr(), vals.data_ptr(), keys.data_ptr(), out_v.data_ptr(), n, 24,
                                    stream)
    torch.cuda.synchronize()
    assert rc == abi.MK_ERR_INVALID_ARGUMENT
    assert b"overlap" in lib.mk_last_error()
    assert bool((out_v == 5).all())
