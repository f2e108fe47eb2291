"""Solver modes without a reference counterpart, against the CPU oracle.

Contact solve to a residual: the reference's relaxed-Jacobi passes repeated
until ||r|| <= tol * ||r_cold||.  The norms are FP64 sums in one fixed order
on both sides, so the stopping pass, the impulses and the body state must
agree bit for bit (0 ULP) with the oracle, like the fixed-pass form.
"""
import numpy as np
import pytest

from mechanic_b200 import scenes
from mechanic_b200.physics import GpuPhysicsConfig

from test_gpu_parity import assert_bitwise, compare_tick, make_pair

pytestmark = pytest.mark.gpu


def _residual_config(**kw):
    return GpuPhysicsConfig(contact_tolerance=1e-5, contact_max_iterations=512, **kw)


def test_residual_solve_bitexact_60_ticks(cuda_lib):
    scene = scenes.falling_cubes(1000, seed=0)
    gpu, orc = make_pair(scene, _residual_config())
    for tick in range(1, 61):
        compare_tick(gpu, orc, tick, check_tree=(tick % 20 == 1))
        rb = gpu.read_last_tick()
        st = orc.solve_stats()
        assert rb.contact_iterations == st["iterations"], f"tick {tick} passes"
        assert rb.contact_relative_residual == pytest.approx(st["relative_residual"], rel=0, abs=0)
        if rb.active_contact_count:
            assert st["converged"] == 1
            assert rb.contact_relative_residual <= 1e-5


def test_residual_cap_stops_at_max_iterations(cuda_lib):
    scene = scenes.falling_cubes(1000, seed=3)
    gpu, orc = make_pair(scene, GpuPhysicsConfig(contact_tolerance=1e-12, contact_max_iterations=9))
    for tick in range(1, 31):
        compare_tick(gpu, orc, tick, check_tree=False)
        rb = gpu.read_last_tick()
        if rb.active_contact_count:
            assert rb.contact_iterations == 9
            assert orc.solve_stats()["converged"] == 0


def test_residual_solve_on_cube_cylinder_grid(cuda_lib):
    scene = scenes.stack_grid(8, 6, 8, seed=5)
    gpu, orc = make_pair(scene, _residual_config())
    for tick in range(1, 6):
        compare_tick(gpu, orc, tick, check_tree=False)
        assert gpu.read_last_tick().contact_iterations == orc.solve_stats()["iterations"]
    assert_bitwise(gpu.contacts(), orc.contacts(), "contact rows")


def test_clipped_manifold_bitexact(cuda_lib):
    """MK_MANIFOLD_CLIPPED: up to four points per pair (collision.rs:68-103 rule), warm
    started point by point from the pair's previous rows."""
    from mechanic_b200 import abi
    scene = scenes.falling_cubes(1000, seed=0)
    gpu, orc = make_pair(scene, GpuPhysicsConfig(contact_manifold=abi.MANIFOLD_CLIPPED))
    multi = 0
    for tick in range(1, 61):
        compare_tick(gpu, orc, tick, check_tree=False)
        feats = gpu.features()
        if len(feats):
            multi = max(multi, int(((feats >> 25) & 3).max()) + 1)   # point index within its pair
    assert 2 <= multi <= 4
