"""Articulated scenes on the CPU oracle, pinned to the reference's bench gates.

crates/mechanic-bench/src/main.rs:113-132, 211-216: four_bar (a 0.001 rad
perturbation of the first coordinate, collisions off) must run with
error_flags == 0, and invalid_loop (closure anchor moved by (0.2, 0.13, 0.07))
must raise CONSTRAINT_NON_CONVERGENCE_FLAG.  main.rs:570-580: the four-bar
scenes have 4 bodies, 3 tree bearings and 1 closure.
"""
import numpy as np

import oracle
from mechanic_b200 import abi, scenes


def _config(collisions: bool) -> abi.MkConfig:
    c = abi.MkConfig()
    c.collisions_enabled = int(collisions)
    c.mechanism_self_collisions = 1
    c.solver_iterations = 8
    return c


def _run_four_bar(invalid: bool, ticks: int = 60):
    scene = scenes.four_bar(invalid)
    w = oracle.OracleWorld(scene, _config(False))
    coords = np.zeros(3, abi.MECHANISM_COORDINATE)
    coords["angle"][0] = 0.001           # main.rs:114-131
    w.set_coordinates(coords)
    flags = 0
    for tick in range(1, ticks + 1):
        w.step(tick)
        flags |= int(w.diagnostics()["error_flags"])
    return w, flags


def test_four_bar_rows_match_bench_counts():
    for invalid in (False, True):
        s = scenes.four_bar(invalid)
        assert s.body_count == 4
        assert s.coordinate_count == 3
        assert int((s.bearings["metadata"][:, 3] != 0).sum()) == 1


def test_four_bar_converges_without_flags():
    w, flags = _run_four_bar(False)
    assert flags == 0
    d = w.diagnostics()
    assert int(d["max_anchor_micrometers"]) <= 10        # reference milestone: 9 um
    assert int(d["max_axis_microdegrees"]) <= 1000


def test_invalid_loop_raises_non_convergence():
    _, flags = _run_four_bar(True)
    assert flags & abi.CONSTRAINT_NON_CONVERGENCE_FLAG


def test_chain_forward_kinematics_keeps_tree_bearings_exact():
    """Tree bearings are satisfied by construction (coordinate-space FK): their anchor
    residual stays at the FP32 level while the chains swing under gravity and drives."""
    scene = scenes.bearing_chains(chains=24, links=5, seed=2, closure_fraction=0.0)
    w = oracle.OracleWorld(scene, _config(True))
    for tick in range(1, 31):
        w.step(tick)
        d = w.diagnostics()
        assert int(d["error_flags"]) & abi.INVALID_NUMERIC_FLAG == 0
        assert int(d["max_anchor_micrometers"]) <= 2
    tr, _ = w.state()
    assert np.isfinite(tr["position"]).all()


def test_reconstructed_velocities_follow_the_tree():
    """articulated.wgsl:431-456: a child's angular velocity is its parent's plus axis * speed."""
    scene = scenes.bearing_chains(chains=8, links=5, seed=4, closure_fraction=0.0)
    cfg = _config(False)
    w = oracle.OracleWorld(scene, cfg)
    w.step(1)
    _, vel = w.state()
    coords = w.coordinates()
    mb = scene.mechanism_bodies
    tr, _ = w.state()
    for body in range(scene.body_count):
        if mb["metadata"][body, 3]:
            continue
        parent = int(mb["metadata"][body, 0])
        br = scene.bearings[int(mb["metadata"][body, 1])]
        q = tr["rotation"][parent].astype(np.float64)
        axis = scenes.quat_rotate(q, br["local_axis_a"][:3].astype(np.float64))
        axis /= np.linalg.norm(axis)
        expect = vel["angular"][parent, :3] + axis * coords["angular_velocity"][int(br["metadata"][2])]
        assert np.allclose(vel["angular"][body, :3], expect, atol=1e-5)
