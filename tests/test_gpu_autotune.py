"""The launch-shape autotuner (mk_autotune) through the C ABI.

Every launch shape it tries computes the same results (the sort, the ordered
appends and the solve are deterministic whatever their grid), so a handle
that was autotuned mid-run must stay bit-identical to one that was not, and
the handle's state must be restored after the search.
"""
import pytest

from mechanic_b200 import abi, scenes
from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_and_state(cuda_lib):
    scene = scenes.stack_grid(20, 10, 20, seed=4)
    caps = {"pair_capacity": 1 << 22}
    a = GpuPhysics(scene, GpuPhysicsConfig(), capacities=caps)
    b = GpuPhysics(scene, GpuPhysicsConfig(), capacities=caps)
    for tick in range(1, 6):
        a.dispatch_tick(tick)
        b.dispatch_tick(tick)
    before = a.save_state()
    tuning, ms = a.autotune(ticks=2)
    assert ms > 0 and tuning["sort_items"] in (2, 4, 6, 8, 11, 16)
    assert tuning["morton_mode"] in (abi.MORTON_39, abi.MORTON_30_ADAPTIVE)   # either key width: same pairs
    after = a.save_state()
    assert_bitwise(after["transforms"], before["transforms"], "restored transforms")
    assert_bitwise(after["velocities"], before["velocities"], "restored velocities")
    for tick in range(6, 16):
        a.dispatch_tick(tick)
        b.dispatch_tick(tick)
    sa, sb = a.save_state(manifold_capacity=0), b.save_state(manifold_capacity=0)
    assert_bitwise(sa["transforms"], sb["transforms"], "tuned vs default transforms")
    assert_bitwise(sa["velocities"], sb["velocities"], "tuned vs default velocities")


def test_explicit_tuning_is_applied(cuda_lib):
    scene = scenes.falling_cubes(500, seed=1)
    g = GpuPhysics(scene)
    g.set_tuning(sort_items=4, sort_ctas_per_sm=6, append_ctas_per_sm=16, solve_items=2)
    t = g.tuning()
    assert (t["sort_items"], t["sort_ctas_per_sm"], t["append_ctas_per_sm"], t["solve_items"]) == (4, 6, 16, 2)
    for tick in range(1, 4):
        g.dispatch_tick(tick)
    assert g.read_last_tick().error_flags == 0
