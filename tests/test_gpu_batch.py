"""Batched scenes through mk_create_batch against the oracle and against
single-scene handles.  Integer outputs and the state are compared bit for
bit: the batch's scene keys, pair list, contacts and body rows equal the
oracle's, and with the fixed passes each scene's slice equals that scene
stepped alone on the GPU."""
import numpy as np
import pytest

import oracle
from mechanic_b200 import scenes
from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def _lst():
    return [scenes.mixed_scene(400, seed=1), scenes.falling_cubes(100, seed=2),
            scenes.mixed_scene(700, seed=3, bearing_fraction=0.0), scenes.mixed_scene(90, seed=4),
            scenes.falling_cubes(300, seed=5)]


def test_batch_bitexact_against_oracle(cuda_lib):
    lst = _lst()
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics.batch(lst, cfg, capacities={"pair_capacity": 1 << 20, "max_bodies": 1 << 20,
                                                 "max_colliders": 1 << 22, "max_bearings": 1 << 20})
    orc = oracle.OracleWorld.batch(lst, cfg.to_c(), pair_capacity=1 << 20)
    bo, co = gpu.scene_offsets()
    assert list(bo) == list(np.cumsum([0] + [s.body_count for s in lst]))
    for tick in range(1, 9):
        gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        orc.step(tick)
        d = orc.diagnostics()
        assert rb.error_flags == int(d["error_flags"]) and rb.pair_count == int(d["pair_count"])
        assert rb.contact_count == int(d["contact_count"]), tick
        assert np.array_equal(gpu.collider_keys(), orc.collider_keys())
        gk, gv = gpu.sorted_entries()
        ok, ov = orc.sorted_entries()
        assert np.array_equal(gk, ok) and np.array_equal(gv, ov)
        assert np.array_equal(gpu.pairs(), orc.pairs())
        assert_bitwise(gpu.contacts(), orc.contacts(), f"tick {tick} contacts")
        st = gpu.save_state(manifold_capacity=0)
        tr, vel = orc.state()
        assert_bitwise(st["transforms"], tr, f"tick {tick} transforms")
        assert_bitwise(st["velocities"], vel, f"tick {tick} velocities")


def test_batch_tiny_scenes_against_oracle(cuda_lib):
    """Scenes of one, two and three colliders beside a larger one: a one-collider scene has no
    subtree of its own (its walk is skipped), the others are walked from their own subtree roots."""
    lst = [scenes.falling_cubes(1, seed=7), scenes.falling_cubes(2, seed=8, box=0.2), scenes.mixed_scene(90, seed=4),
           scenes.falling_cubes(3, seed=9, box=0.3), scenes.falling_cubes(1, seed=10)]
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics.batch(lst, cfg, capacities={"pair_capacity": 1 << 16})
    orc = oracle.OracleWorld.batch(lst, cfg.to_c(), pair_capacity=1 << 16)
    seen = 0
    for tick in range(1, 5):
        gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        orc.step(tick)
        d = orc.diagnostics()
        assert rb.error_flags == int(d["error_flags"]) and rb.pair_count == int(d["pair_count"]), tick
        assert np.array_equal(gpu.pairs(), orc.pairs()), tick
        assert_bitwise(gpu.contacts(), orc.contacts(), f"tick {tick} contacts")
        seen += rb.pair_count
    assert seen > 0


def test_batch_slices_equal_single_scenes(cuda_lib):
    # plain scenes only: a batch holding a mechanism takes the reference's mechanism
    # contact path (device.rs:1370-1417) for all of its contacts
    lst = [scenes.falling_cubes(100, seed=2), scenes.mixed_scene(700, seed=3, bearing_fraction=0.0),
           scenes.falling_cubes(300, seed=5), scenes.mixed_scene(250, seed=6, bearing_fraction=0.0)]
    caps = {"pair_capacity": 1 << 20}
    gpu = GpuPhysics.batch(lst, GpuPhysicsConfig(), capacities=caps)
    singles = [GpuPhysics(s, GpuPhysicsConfig(), capacities=caps) for s in lst]
    for tick in range(1, 31):
        gpu.dispatch_tick(tick)
        for h in singles:
            h.dispatch_tick(tick)
    st = gpu.save_state(manifold_capacity=0)
    bo, _ = gpu.scene_offsets()
    for i, h in enumerate(singles):
        one = h.save_state(manifold_capacity=0)
        assert_bitwise(st["transforms"][bo[i]:bo[i + 1]], one["transforms"], f"scene {i} transforms")
        assert_bitwise(st["velocities"][bo[i]:bo[i + 1]], one["velocities"], f"scene {i} velocities")


def test_batched_config_runs(cuda_lib):
    lst = scenes.batched_uneven(256, seed=0)
    nb = sum(s.body_count for s in lst)
    nc = sum(s.collider_count for s in lst)
    gpu = GpuPhysics.batch(lst, GpuPhysicsConfig(), capacities={
        "max_bodies": nb, "max_colliders": nc, "max_bearings": 1 << 20, "pair_capacity": 1 << 26})
    for tick in range(1, 4):
        gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        assert rb.error_flags & 1 == 0, rb.pair_count     # (bit 4: the drives keep some loops open)
        assert rb.pair_count > 0 and rb.contact_count > 0
    bo, co = gpu.scene_offsets()
    assert bo[-1] == nb and co[-1] == nc
