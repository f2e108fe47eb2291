"""Published snapshot pair and the device interpolation between its slots.

mk_published_state mirrors PublishedGpuState (runtime.rs:60-75) as
publish_tick (runtime.rs:222-237) advances it; mk_interpolate_snapshot
writes the render hand-off at the scheduler's fraction alpha
(scheduler.rs:69-73).  Checked against a CPU lerp / shortest-arc slerp of
the two slots read back through the C ABI, within 2e-6 (FP32 arithmetic of
a few operations on unit quaternions and metre-scale positions).
"""
import numpy as np
import pytest

from mechanic_b200 import scenes
from mechanic_b200.physics import GpuPhysics, InvalidArgument
from mechanic_b200.scheduler import FixedStepScheduler

pytestmark = pytest.mark.gpu


def _slerp(q0, q1, a):
    q0 = q0.astype(np.float64)
    q1 = q1.astype(np.float64).copy()
    d = np.sum(q0 * q1, axis=1)
    q1[d < 0] *= -1
    d = np.abs(d)
    theta = np.arccos(np.clip(d, -1, 1))
    small = d > 0.9995
    st = np.where(small, 1.0, np.sin(theta))
    s0 = np.where(small, 1 - a, np.sin((1 - a) * theta) / st)
    s1 = np.where(small, a, np.sin(a * theta) / st)
    q = q0 * s0[:, None] + q1 * s1[:, None]
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def test_published_pair_and_interpolation(cuda_lib):
    import torch
    scene = scenes.falling_cubes(1000, seed=0)
    gpu = GpuPhysics(scene)
    st = gpu.published_state()
    assert st.ticks_published == 0 and st.body_count == 1000
    clock = FixedStepScheduler()
    for tick in clock.advance(3 * 16_666_667 + 5_000_000):   # three ticks and 0.3 of the next
        gpu.dispatch_tick(tick)
    alpha = clock.interpolation_alpha()
    assert 0.29 < alpha < 0.31
    st = gpu.published_state()
    assert (st.previous_tick, st.current_tick) == (2, 3)
    assert (st.previous_slot, st.current_slot) == (2, 0)
    assert st.ticks_published == 2
    pos = torch.empty((1000, 4), dtype=torch.float32, device="cuda")
    rot = torch.empty((1000, 4), dtype=torch.float32, device="cuda")
    gpu.interpolate_snapshot(alpha, pos.data_ptr(), rot.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    prev = gpu.read_snapshot_transforms(st.previous_slot)
    cur = gpu.read_snapshot_transforms(st.current_slot)
    p0, p1 = prev["position"][:, :3].astype(np.float64), cur["position"][:, :3].astype(np.float64)
    want_p = p0 + (p1 - p0) * alpha
    want_q = _slerp(prev["rotation"], cur["rotation"], alpha)
    got_p = pos.cpu().numpy()[:, :3]
    got_q = rot.cpu().numpy()
    np.testing.assert_allclose(got_p, want_p, atol=2e-6 * max(1.0, np.abs(want_p).max()))
    # q and -q are the same rotation
    sign = np.sign(np.sum(got_q * want_q, axis=1))[:, None]
    np.testing.assert_allclose(got_q * sign, want_q, atol=2e-6)
    # the next tick rewrites the previous slot only after the interpolation read it
    gpu.dispatch_tick(4)
    assert (gpu.published_state().previous_tick, gpu.published_state().current_tick) == (3, 4)
    with pytest.raises(InvalidArgument):
        gpu.interpolate_snapshot(1.5, pos.data_ptr(), rot.data_ptr())
    gpu.close()
