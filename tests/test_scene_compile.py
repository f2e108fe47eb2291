"""The mechanism compiler (compile.rs:394-609 restated in scenes.compile_mechanism)
against hand-built rows, and the loops_100k lattice (mechanic-bench main.rs:456-524)."""
import numpy as np

from mechanic_b200 import abi, scenes


def test_compiler_reproduces_four_bar_rows():
    ref = scenes.four_bar()
    got = scenes.compile_mechanism(scenes.four_bar(), [0, 1, 2, 3], [1, 2, 3, 0],
                                   [(0.5, 0, 0), (1, 0.5, 0), (0.5, 1, 0), (0, 0.5, 0)],
                                   [(1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0)])
    for k in ("mechanism_bodies", "bearings", "preorder", "root_flags", "body_components", "suppressed_pairs"):
        assert getattr(ref, k).tobytes() == getattr(got, k).tobytes(), k
    assert (got.coordinate_count, got.closure_count, got.max_depth) == (3, 1, 3)


def test_compiler_chain_topology_matches_generator():
    """Chains with closures, half the tree bearings driven: same tree, coordinates,
    parents, depths and preorder as the generator builds directly."""
    ref = scenes.bearing_chains(chains=30, links=5, seed=2, closure_fraction=0.3)
    m = ref.bearings["metadata"]
    pos = ref.transforms["position"][:, :3].astype(np.float64)
    anchor = pos[m[:, 0]] + ref.bearings["local_anchor_a"][:, :3]
    driven = np.zeros(len(m), bool)
    tree_rows = m[:, 2] != abi.INVALID_INDEX
    driven[tree_rows] = ref.drives["mode"][m[tree_rows, 2]] == abi.DRIVE_MODE_SPEED
    got = scenes.compile_mechanism(scenes.bearing_chains(chains=30, links=5, seed=2, closure_fraction=0.3),
                                   m[:, 0], m[:, 1], anchor, ref.bearings["local_axis_a"][:, :3], driven,
                                   drives=ref.drives)
    assert np.array_equal(got.bearings["metadata"], m)
    for f in ("metadata",):
        assert np.array_equal(got.mechanism_bodies[f], ref.mechanism_bodies[f])
    assert np.array_equal(got.mechanism_bodies["traversal"][:, :3], ref.mechanism_bodies["traversal"][:, :3])
    assert np.array_equal(got.preorder, ref.preorder)
    np.testing.assert_allclose(got.bearings["local_anchor_b"], ref.bearings["local_anchor_b"], atol=1e-6)
    assert (got.coordinate_count, got.closure_count, got.max_depth) == (
        ref.coordinate_count, ref.closure_count, ref.max_depth)


def test_loops_lattice_counts_and_tree():
    s = scenes.loops_grid(20, 10, 3)
    n = 20 * 10 * 3
    assert s.body_count == n
    assert s.bearing_count == 3 * (19 * 10 + 20 * 9) + 2
    assert s.coordinate_count == n - 1              # one component: a spanning tree
    assert s.closure_count == s.bearing_count - (n - 1)
    mb = s.mechanism_bodies
    root = s.root_flags.astype(bool)
    assert root.sum() == 1 and root[0]
    parent = mb["metadata"][:, 0].astype(np.int64)
    depth = mb["traversal"][:, 1].astype(np.int64)
    assert np.all(depth[~root] == depth[parent[~root]] + 1)
    # preorder is a BFS order: depths never decrease along it
    assert np.all(np.diff(depth[s.preorder]) >= 0)
    # each tree bearing joins the body to its parent; direction says which end the parent is
    j = mb["metadata"][~root, 1].astype(np.int64)
    ends = s.bearings["metadata"][j, :2].astype(np.int64)
    d = mb["metadata"][~root, 2]
    child = np.nonzero(~root)[0]
    assert np.all(np.where(d == 0, ends[:, 0], ends[:, 1]) == parent[child])
    assert np.all(np.where(d == 0, ends[:, 1], ends[:, 0]) == child)
    # 1 m cubes of density 500
    np.testing.assert_allclose(s.spatial_inertias["mass"][:, 0], 500.0)
