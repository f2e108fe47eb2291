"""GPU parity: libmechanic_b200 (through the C ABI) against the CPU oracle.

Bit-exact targets: collider Morton keys, the sort permutation, Karras
topology, AABBs, the canonical pair list, contact rows (points, depths,
normals, impulses), SAT feature words, the active list and the body state
after each tick.  The oracle's FP32 build and the CUDA build both evaluate
every float operation as one IEEE-754 operation in the reference's order, so
the tolerance for all of these is zero ULP.
"""
import numpy as np
import pytest

import oracle
from mechanic_b200 import abi, scenes
from mechanic_b200.physics import (BodyIndexOutOfRange, GpuPhysics, GpuPhysicsConfig,
                                   InvalidSnapshotSlot, NonFinite)

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def assert_bitwise(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    if not np.array_equal(_bits(a), _bits(b)):
        fa = a.view(np.float32).reshape(len(a), -1) if a.dtype.names else a
        fb = b.view(np.float32).reshape(len(b), -1) if b.dtype.names else b
        bad = np.nonzero((_bits(a).reshape(len(a), -1) != _bits(b).reshape(len(b), -1)).any(axis=1))[0]
        raise AssertionError(f"{what}: {len(bad)} rows differ, first {bad[:5]}: {fa[bad[:2]]} vs {fb[bad[:2]]}")


def make_pair(scene, config=None, pair_capacity=1 << 22):
    cfg = config or GpuPhysicsConfig()
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": pair_capacity})
    orc = oracle.OracleWorld(scene, cfg.to_c(), precision=32, pair_capacity=pair_capacity)
    return gpu, orc


def compare_tick(gpu, orc, tick, check_tree=True):
    gpu.dispatch_tick(tick)
    rb = gpu.read_last_tick()
    orc.step(tick)
    d = orc.diagnostics()
    assert rb.error_flags == int(d["error_flags"]), f"tick {tick} flags"
    assert rb.pair_count == int(d["pair_count"]), f"tick {tick} pair count"
    assert rb.contact_count == int(d["contact_count"]), f"tick {tick} contact count"
    assert rb.active_contact_count == int(d["active_contact_count"]), f"tick {tick} active count"
    if check_tree:
        assert np.array_equal(gpu.collider_keys(), orc.collider_keys()), "Morton keys"
        gk, gv = gpu.sorted_entries()
        ok, ov = orc.sorted_entries()
        assert np.array_equal(gk, ok) and np.array_equal(gv, ov), "sort permutation"
        assert np.array_equal(gpu.node_children(), orc.karras()), "Karras topology"
        assert_bitwise(gpu.aabbs(), orc.aabbs(), "collider AABBs")
        assert_bitwise(gpu.world_masses(), orc.world_masses(), "world inverse inertia")
    assert np.array_equal(gpu.pairs(), orc.pairs()), f"tick {tick} canonical pair list"
    assert_bitwise(gpu.contacts(), orc.contacts(), f"tick {tick} contacts")
    assert np.array_equal(gpu.features() & 0xFFFFFF, orc.features()), f"tick {tick} SAT features"
    assert np.array_equal(gpu.active(), orc.active()), f"tick {tick} active list"
    st = gpu.save_state(manifold_capacity=0)
    tr, vel = orc.state()
    assert_bitwise(st["transforms"], tr, f"tick {tick} transforms")
    assert_bitwise(st["velocities"], vel, f"tick {tick} velocities")


def test_falling_cubes_one_tick_bitexact(cuda_lib):
    scene = scenes.falling_cubes(1000, seed=0)
    gpu, orc = make_pair(scene)
    compare_tick(gpu, orc, 1)


def test_falling_cubes_sixty_ticks_bitexact(cuda_lib):
    """Config 1 (1,000 cubes, 8 iterations, 60 steps) with warm starting."""
    scene = scenes.falling_cubes(1000, seed=0)
    gpu, orc = make_pair(scene)
    for tick in range(1, 61):
        compare_tick(gpu, orc, tick, check_tree=(tick % 20 == 0))
    slot = 60 % 3
    snap = gpu.read_snapshot_transforms(slot)
    assert_bitwise(snap, orc.snapshot(slot), "snapshot ring slot")


def test_stack_grid_small_bitexact(cuda_lib):
    """Config 2's mix (cubes + 16-segment cylinders) on a 12x8x12 grid."""
    scene = scenes.stack_grid(12, 8, 12, seed=3)
    gpu, orc = make_pair(scene)
    for tick in range(1, 6):
        compare_tick(gpu, orc, tick)


def test_reference_morton_mode_same_pairs(cuda_lib):
    """30-bit keys of lbvh.wgsl:93-98 build another tree; the pair set is the same."""
    scene = scenes.stack_grid(10, 6, 10, seed=5)
    cfg = GpuPhysicsConfig(morton_mode=abi.MORTON_REFERENCE_30)
    gpu, orc = make_pair(scene, cfg)
    for tick in range(1, 4):
        compare_tick(gpu, orc, tick)


@pytest.mark.parametrize("mode", [abi.MORTON_63, abi.MORTON_48, abi.MORTON_30_ADAPTIVE],
                         ids=["63-bit", "48-bit", "30-bit-adaptive"])
def test_other_morton_modes_bitexact(cuda_lib, mode):
    """21, 16 and 10 bits per axis (the default has 13): the same bit-exact path (keys,
    permutation, topology, pairs, contacts, state)."""
    scene = scenes.stack_grid(10, 6, 10, seed=5)
    gpu, orc = make_pair(scene, GpuPhysicsConfig(morton_mode=mode))
    for tick in range(1, 4):
        compare_tick(gpu, orc, tick)


@pytest.mark.parametrize("grid,ticks", [((14, 9, 14), (1, 3, 6)), ((30, 30, 30), (2,))],
                         ids=["7k-colliders", "100k-colliders"])
def test_node_boxes_are_leaf_range_unions(cuda_lib, grid, ticks):
    """Every LBVH node box equals the min/max over the AABBs of its leaf range
    (exact: unions are min/max), over ticks with dense and sparse contact; the
    larger scene spans about a hundred 1,024-leaf super-chunks, so its long
    ranges go through every level of the super-chunk sparse table."""
    scene = scenes.stack_grid(*grid, seed=11)
    gpu = GpuPhysics(scene, GpuPhysicsConfig(), capacities={"pair_capacity": 1 << 24})
    for tick in range(1, max(ticks) + 1):
        gpu.dispatch_tick(tick)
        gpu.wait()
        if tick not in ticks:
            continue
        ch = gpu.node_children().astype(np.int64)
        nodes = gpu.node_aabbs()
        _, vals = gpu.sorted_entries()
        ab = gpu.aabbs()
        C = len(vals)
        I = C - 1
        leaf_min, leaf_max = ab[vals, 0:3], ab[vals, 4:7]
        assert np.array_equal(nodes[I:, 0:3], leaf_min) and np.array_equal(nodes[I:, 4:7], leaf_max)
        first = np.zeros(I, np.int64)
        last = np.zeros(I, np.int64)
        order, stack = [], [0]
        while stack:
            x = stack.pop()
            order.append(x)
            stack.extend(int(c) for c in ch[x] if c < I)
        for x in reversed(order):   # children before parents
            lo = [c - I if c >= I else first[c] for c in ch[x]]
            hi = [c - I if c >= I else last[c] for c in ch[x]]
            first[x], last[x] = min(lo), max(hi)
        for x in range(I):
            want_min = leaf_min[first[x]:last[x] + 1].min(axis=0)
            want_max = leaf_max[first[x]:last[x] + 1].max(axis=0)
            assert np.array_equal(nodes[x, 0:3], want_min), f"tick {tick} node {x} min"
            assert np.array_equal(nodes[x, 4:7], want_max), f"tick {tick} node {x} max"
            assert nodes[x, 3:4].view(np.uint32)[0] == last[x]


def _expected_records(ch, nodes, vals):
    """Traversal records rebuilt from the topology and node boxes: per internal node its
    grandchildren in leaf order (a leaf child is one entry), {min.xyz, code} {max.xyz, last}."""
    I = len(ch)
    u = nodes.view(np.uint32)
    rec = np.zeros((I, 32), np.float32)
    ru = rec.view(np.uint32)

    def entry(c):
        row = nodes[c]
        if c >= I:
            return row[0:3], row[4:7], 0x80000000 | int(vals[c - I]), c - I
        return row[0:3], row[4:7], c, int(u[c, 3])

    for x in range(I):
        ents = []
        for c in ch[x]:
            ents += [entry(int(c))] if c >= I else [entry(int(g)) for g in ch[c]]
        for k, (mn, mx, code, last) in enumerate(ents):
            rec[x, 8 * k:8 * k + 3] = mn
            ru[x, 8 * k + 3] = code
            rec[x, 8 * k + 4:8 * k + 7] = mx
            ru[x, 8 * k + 7] = last
    return rec


@pytest.mark.parametrize("scene_fn", [lambda: scenes.falling_cubes(20, seed=3),
                                      lambda: scenes.falling_cubes(40, seed=3),
                                      lambda: scenes.stack_grid(14, 9, 14, seed=11)],
                         ids=["20-colliders", "40-colliders", "stack-grid"])
def test_traversal_records_match_tree(cuda_lib, scene_fn):
    """Each internal node's 4-wide traversal record holds exactly its grandchildren in leaf
    order with their node or leaf boxes, codes and last leaves: records of nodes inside one
    32-leaf chunk come from the leaf refit's warp lanes, the others from the cross-chunk list."""
    scene = scene_fn()
    gpu = GpuPhysics(scene, GpuPhysicsConfig(), capacities={"pair_capacity": 1 << 22})
    for tick in range(1, 4):
        gpu.dispatch_tick(tick)
        gpu.wait()
        ch = gpu.node_children().astype(np.int64)
        nodes = gpu.node_aabbs()
        _, vals = gpu.sorted_entries()
        want = _expected_records(ch, nodes, vals)
        got = gpu.node_records()
        assert got.shape == want.shape
        bad = np.nonzero((got.view(np.uint32) != want.view(np.uint32)).any(axis=1))[0]
        assert len(bad) == 0, f"tick {tick}: {len(bad)} records differ, first nodes {bad[:5]}"


def test_snapshot_reads_overlap_later_ticks(cuda_lib):
    """A snapshot read waits for the tick that last wrote its slot, not for ticks dispatched
    after it, and a tick that rewrites a slot waits for a read of it: reading tick k's slot
    after dispatching tick k + 1 gives the rows a fully synchronised read gives."""
    scene = scenes.stack_grid(10, 6, 10, seed=17)
    ref = GpuPhysics(scene, GpuPhysicsConfig())
    want = []
    for tick in range(1, 8):
        sub = ref.dispatch_tick(tick)
        ref.wait()
        want.append(ref.read_snapshot_transforms(sub.snapshot_slot).copy())
    gpu = GpuPhysics(scene, GpuPhysicsConfig())
    got, prev = [], None
    for tick in range(1, 8):
        sub = gpu.dispatch_tick(tick)
        if prev is not None:
            got.append(gpu.read_snapshot_transforms(prev.snapshot_slot).copy())
        prev = sub
    got.append(gpu.read_snapshot_transforms(prev.snapshot_slot).copy())
    for k, (a, b) in enumerate(zip(got, want)):
        assert_bitwise(a, b, f"snapshot of tick {k + 1}")
    # a slot read after later ticks rewrote it holds the newest writer's rows
    for tick in range(8, 11):
        gpu.dispatch_tick(tick)
        ref.dispatch_tick(tick)
    ref.wait()
    assert_bitwise(gpu.read_snapshot_transforms(10 % 3), ref.read_snapshot_transforms(10 % 3), "slot of tick 10")


def test_graph_and_direct_launch_agree(cuda_lib):
    scene = scenes.stack_grid(8, 6, 8, seed=1)
    a = GpuPhysics(scene, GpuPhysicsConfig(use_graph=True))
    b = GpuPhysics(scene, GpuPhysicsConfig(use_graph=False))
    for tick in range(1, 8):
        a.dispatch_tick(tick)
        b.dispatch_tick(tick)
    sa, sb = a.save_state(), b.save_state()
    assert_bitwise(sa["transforms"], sb["transforms"], "graph vs direct transforms")
    assert_bitwise(sa["velocities"], sb["velocities"], "graph vs direct velocities")


def test_one_step_from_identical_state(cuda_lib):
    """Load the oracle's state (pose, velocity, manifold) into the GPU and step once."""
    scene = scenes.stack_grid(10, 6, 10, seed=7)
    orc = oracle.OracleWorld(scene, GpuPhysicsConfig().to_c(), pair_capacity=1 << 22)
    for tick in range(1, 5):
        orc.step(tick)
    tr, vel = orc.state()
    man = orc.manifold()
    gpu = GpuPhysics(scene, GpuPhysicsConfig(), capacities={"pair_capacity": 1 << 22})
    gpu.load_state(tr, vel, manifold=man, manifold_tick=4)
    compare_tick(gpu, orc, 5)
    saved = gpu.save_state()
    assert saved["manifold_tick"] == 5
    assert np.array_equal(saved["manifold"]["metadata"][:, 2:], orc.manifold()["metadata"][:, 2:])
    assert_bitwise(saved["manifold"]["normal_penetration"], orc.manifold()["normal_penetration"], "manifold")
    assert_bitwise(saved["manifold"]["arm_a_impulse"], orc.manifold()["arm_a_impulse"], "manifold impulses")


def test_error_variants(cuda_lib):
    scene = scenes.falling_cubes(16, seed=2)
    gpu = GpuPhysics(scene)
    with pytest.raises(InvalidSnapshotSlot):
        gpu.read_snapshot_transforms(3)
    with pytest.raises(BodyIndexOutOfRange) as e:
        gpu.apply_impulse(16, (0, 0, 0), (1, 0, 0))
    assert e.value.body_index == 16 and e.value.body_count == 16
    with pytest.raises(NonFinite):
        gpu.apply_impulse(0, (np.nan, 0, 0), (1, 0, 0))
    assert gpu.snapshot(3) is None and gpu.snapshot(0) is not None


def test_apply_impulse_matches_formula(cuda_lib):
    """physics.wgsl:73-90 on a resting cube: dv = J/m, dw = I^-1 (r x J)."""
    scene = scenes.falling_cubes(1, seed=4)
    scene.velocities[:] = 0
    gpu = GpuPhysics(scene, GpuPhysicsConfig(collisions_enabled=False))
    pos = scene.transforms["position"][0, :3].astype(np.float64)
    gpu.apply_impulse(0, pos + np.array([0.0, 0.125, 0.0]), (1.0, 0.0, 0.0))
    st = gpu.save_state()
    inv_m = float(scene.masses["inverse_mass"][0, 0])
    assert st["velocities"]["linear"][0, 0] == pytest.approx(inv_m, rel=1e-6)
    inv_i = float(scene.masses["inverse_inertia_z"][0, 2])
    assert st["velocities"]["angular"][0, 2] == pytest.approx(-0.125 * inv_i, rel=1e-5)


def test_pair_overflow_sets_flag_without_overrun(cuda_lib):
    scene = scenes.stack_grid(10, 6, 10, seed=9)
    gpu = GpuPhysics(scene, GpuPhysicsConfig(), capacities={"pair_capacity": 64})
    gpu.dispatch_tick(1)
    rb = gpu.read_last_tick()
    assert rb.error_flags & abi.PAIR_OVERFLOW_FLAG
    assert rb.pair_count > 64
    pairs = gpu.pairs()
    assert len(pairs) == 64
    # which pairs survive an overflow depends on arrival order (as in the
    # reference, lbvh.wgsl:353-358); they are still real pairs, in canonical order
    orc = oracle.OracleWorld(scene, GpuPhysicsConfig().to_c(), pair_capacity=1 << 22)
    orc.step(1)
    assert rb.pair_count == orc.pair_count
    ref = {(int(a), int(b)) for a, b in orc.pairs()[["collider_a", "collider_b"]].tolist()}
    got = [(int(a), int(b)) for a, b in pairs[["collider_a", "collider_b"]].tolist()]
    assert got == sorted(got) and set(got) <= ref


def test_nan_input_sets_invalid_numeric(cuda_lib):
    scene = scenes.falling_cubes(32, seed=6)
    scene.velocities["linear"][5, 1] = np.nan
    gpu = GpuPhysics(scene)
    gpu.dispatch_tick(1)
    assert gpu.read_last_tick().error_flags & abi.INVALID_NUMERIC_FLAG


def test_capacity_errors(cuda_lib):
    from mechanic_b200.physics import BodyCapacity, ColliderCapacity
    scene = scenes.falling_cubes(64, seed=1)
    with pytest.raises(BodyCapacity) as e:
        GpuPhysics(scene, capacities={"max_bodies": 32})
    assert e.value.required == 64 and e.value.capacity == 32
    with pytest.raises(ColliderCapacity):
        GpuPhysics(scene, capacities={"max_colliders": 10})


def test_timings_and_determinism(cuda_lib):
    scene = scenes.stack_grid(16, 8, 16, seed=11)
    runs = []
    for _ in range(2):
        gpu = GpuPhysics(scene)
        for tick in range(1, 4):
            gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        assert rb.gpu_tick_ms is not None and rb.gpu_tick_ms > 0
        runs.append(gpu.save_state())
    assert_bitwise(runs[0]["transforms"], runs[1]["transforms"], "run-to-run transforms")
    assert_bitwise(runs[0]["velocities"], runs[1]["velocities"], "run-to-run velocities")


def test_standalone_sort_matches_stable_sort(cuda_lib):
    import torch
    from mechanic_b200 import ops
    rng = np.random.default_rng(0)
    for n in (1, 1000, 2048, 2049, 4096, 4097, 20_000, 300_001):   # one-CTA sort up to 4096 keys
        keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
        keys[: n // 3] = keys[0]                       # many ties
        vals = np.arange(n, dtype=np.uint32)
        k_out, v_out = ops.sort_keys(torch.from_numpy(keys.view(np.int64)).cuda(),
                                     torch.from_numpy(vals.view(np.int32)).cuda())
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k_out.cpu().numpy().view(np.uint64), keys[order])
        assert np.array_equal(v_out.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("items", [2, 4, 6, 8, 11, 16, 32])
def test_standalone_sort_every_tile_shape(cuda_lib, items):
    """Each onesweep tile shape (keys per thread) gives the stable order."""
    import torch
    from mechanic_b200 import ops, physics
    rng = np.random.default_rng(items)
    n = 123_457
    keys = rng.integers(0, 1 << 48, n, dtype=np.uint64)
    keys[::7] = keys[3]                                  # ties across tiles
    vals = np.arange(n, dtype=np.uint32)
    prev = physics.set_tuning(physics.TUNE_SORT_ITEMS, items)
    try:
        k_out, v_out = ops.sort_keys(torch.from_numpy(keys.view(np.int64)).cuda(),
                                     torch.from_numpy(vals.view(np.int32)).cuda(), key_bits=48)
        torch.cuda.synchronize()
    finally:
        physics.set_tuning(physics.TUNE_SORT_ITEMS, max(prev, 0))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k_out.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(v_out.cpu().numpy().view(np.uint32), vals[order])


def test_standalone_sort_above_2m_keys_default_tile(cuda_lib):
    """Above 2M keys the default tile is the 8,192-key one: still the stable order."""
    import torch
    from mechanic_b200 import ops
    rng = np.random.default_rng(17)
    n = 3_000_001
    keys = rng.integers(0, 1 << 40, n, dtype=np.uint64)
    keys[::11] = keys[5]                                 # ties across tiles
    vals = np.arange(n, dtype=np.uint32)
    k_out, v_out = ops.sort_keys(torch.from_numpy(keys.view(np.int64)).cuda(),
                                 torch.from_numpy(vals.view(np.int32)).cuda(), key_bits=40)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k_out.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(v_out.cpu().numpy().view(np.uint32), vals[order])


def test_grid_above_one_sort_tile_bitexact(cuda_lib):
    """16,000 colliders: the collider sort takes the onesweep passes, not the one-CTA sort."""
    scene = scenes.stack_grid(20, 10, 20, seed=13)
    assert scene.collider_count > 4096
    gpu, orc = make_pair(scene)
    for tick in range(1, 4):
        compare_tick(gpu, orc, tick)


@pytest.mark.parametrize("items", [8, 16, 32])
def test_pair_sort_tiles_bitexact(cuda_lib, items):
    """The pair-key sort's tile shapes (2,048, 4,096 and 8,192 keys) give the canonical pair list."""
    from mechanic_b200 import physics
    prev = physics.set_tuning(physics.TUNE_PAIR_SORT_ITEMS, items)
    try:
        scene = scenes.stack_grid(12, 8, 12, seed=3)
        gpu, orc = make_pair(scene)
        compare_tick(gpu, orc, 1)
        assert gpu.read_last_tick().pair_count > 4 * 8192
        compare_tick(gpu, orc, 2)
        gpu.close()
    finally:
        physics.set_tuning(physics.TUNE_PAIR_SORT_ITEMS, max(prev, 0))


@pytest.mark.parametrize("form", [1, 2, 3])
def test_heavy_tick_solve_forms_bitexact(cuda_lib, form):
    """The three forms of the heavy-tick solve (more active contacts than twice the bodies):
    per-contact atomics (1); per-contact slots summed per body through an incidence list (2);
    body a by run sums and atomics, body b by per-contact slots summed per body (3, the default)."""
    from mechanic_b200 import physics
    prev = physics.set_tuning(physics.TUNE_HEAVY_SOLVE, form)
    try:
        scene = scenes.stack_grid(12, 8, 12, seed=3)
        gpu, orc = make_pair(scene)
        compare_tick(gpu, orc, 1)
        assert gpu.read_last_tick().active_contact_count > 2 * scene.body_count
        compare_tick(gpu, orc, 2)
        gpu.close()
    finally:
        physics.set_tuning(physics.TUNE_HEAVY_SOLVE, max(prev, 0))


def test_standalone_sat_matches_oracle(cuda_lib):
    import torch
    from mechanic_b200 import ops
    rng = np.random.default_rng(1)
    n = 4096
    def boxes(seed_shift):
        q = scenes.Rng(seed_shift).unit_quaternions("q", n)
        axes = scenes.quat_matrix(q).astype(np.float32)
        b = np.zeros((n, 4, 4), np.float32)
        b[:, 0, :3] = rng.uniform(-0.4, 0.4, (n, 3))
        half = rng.uniform(0.05, 0.3, (n, 3)).astype(np.float32)
        b[:, 0, 3], b[:, 1, 3], b[:, 2, 3] = half[:, 0], half[:, 1], half[:, 2]
        b[:, 1, :3], b[:, 2, :3], b[:, 3, :3] = axes[:, :, 0], axes[:, :, 1], axes[:, :, 2]
        return b
    a, b = boxes(1), boxes(2)
    np_out, feat = ops.obb_sat(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    np_out, feat = np_out.cpu().numpy(), feat.cpu().numpy().view(np.uint32)
    for i in range(n):
        ref, f = oracle.obb_sat(a[i].reshape(-1), b[i].reshape(-1))
        assert f == feat[i]
        assert np.array_equal(ref.view(np.uint32), np_out[i].view(np.uint32)), i
