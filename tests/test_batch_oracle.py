"""Batched independent scenes on the CPU oracle (no reference counterpart).

A batch is the scenes' rows concatenated with offset indices; colliders of
different scenes never pair.  With the reference's fixed solver passes the
scenes do not interact at all, so a batch must reproduce, bit for bit, each
scene stepped on its own.
"""
import numpy as np

import oracle
from mechanic_b200 import abi, scenes


def _cfg():
    c = abi.MkConfig()
    c.collisions_enabled = 1
    c.mechanism_self_collisions = 1
    c.solver_iterations = 8
    return c


def _small_batch():
    return [scenes.falling_cubes(60, seed=1), scenes.mixed_scene(150, seed=2, bearing_fraction=0.0),
            scenes.falling_cubes(90, seed=3), scenes.mixed_scene(120, seed=4, bearing_fraction=0.0)]


def test_concatenation_offsets():
    lst = [scenes.mixed_scene(300, seed=5), scenes.falling_cubes(40, seed=6), scenes.mixed_scene(500, seed=7)]
    comb, col_scene = scenes.concatenate(lst)
    assert comb.body_count == sum(s.body_count for s in lst)
    assert np.array_equal(np.bincount(col_scene), [s.collider_count for s in lst])
    bo = np.cumsum([0] + [s.body_count for s in lst])
    body = comb.colliders["metadata"][:, 0]
    for i in range(3):
        sel = col_scene == i
        assert body[sel].min() >= bo[i] and body[sel].max() < bo[i + 1]
    jo = np.cumsum([0] + [s.bearing_count for s in lst])
    qo = np.cumsum([0] + [s.coordinate_count for s in lst])
    for i in range(3):
        br = comb.bearings[jo[i]:jo[i + 1]]
        if len(br):
            assert br["metadata"][:, :2].min() >= bo[i] and br["metadata"][:, :2].max() < bo[i + 1]
            coord = br["metadata"][:, 2][br["metadata"][:, 2] != abi.INVALID_INDEX]
            assert coord.min() >= qo[i] and coord.max() < qo[i + 1]
    assert comb.max_depth == max(s.max_depth for s in lst)


def test_batch_has_no_cross_scene_pairs_and_matches_single_scenes():
    lst = _small_batch()
    batch = oracle.OracleWorld.batch(lst, _cfg())
    singles = [oracle.OracleWorld(s, _cfg()) for s in lst]
    comb, col_scene = scenes.concatenate(lst)
    bo = np.cumsum([0] + [s.body_count for s in lst])
    co = np.cumsum([0] + [s.collider_count for s in lst])
    for tick in range(1, 31):
        batch.step(tick)
        for w in singles:
            w.step(tick)
        pairs = batch.pairs()
        if len(pairs):
            assert np.all(col_scene[pairs["collider_a"]] == col_scene[pairs["collider_b"]])
        assert batch.pair_count == sum(w.pair_count for w in singles)
    tr, vel = batch.state()
    for i, w in enumerate(singles):
        t1, v1 = w.state()
        assert tr[bo[i]:bo[i + 1]].tobytes() == t1.tobytes()
        assert vel[bo[i]:bo[i + 1]].tobytes() == v1.tobytes()
        mine = batch.pairs()
        sel = (mine["collider_a"] >= co[i]) & (mine["collider_a"] < co[i + 1])
        got = np.stack([mine["collider_a"][sel] - co[i], mine["collider_b"][sel] - co[i]], 1)
        ref = np.stack([w.pairs()["collider_a"], w.pairs()["collider_b"]], 1)
        assert np.array_equal(got, ref)


def test_batched_config_sizes():
    lst = scenes.batched_uneven(256, seed=0)
    sizes = np.array([s.body_count for s in lst])
    assert sizes.min() >= 64 and sizes.max() <= 8192
    assert 300_000 < sizes.sum() < 700_000
    frac = sum(s.bearing_count for s in lst) / sizes.sum()
    assert 0.005 < frac < 0.03


def test_full_scale_scene_layout():
    """The full form's generator at a small size: the lattice and the chain field are one
    creation, the chain field beside the lattice (no overlap), 10% of the chains closed."""
    lattice = scenes.stack_grid(6, 6, 6, seed=0)
    full = scenes.config_full(0, grid=6, chains=40)
    assert full.body_count == lattice.body_count + 40 * 5
    assert full.collider_count == lattice.collider_count + 40 * 5
    x = full.transforms["position"][:, 0]
    assert x[: lattice.body_count].max() < 10.0 and x[lattice.body_count:].min() > 50.0
    assert full.bearing_count > 0 and full.max_depth > 0
