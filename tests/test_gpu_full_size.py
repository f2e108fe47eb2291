"""Parity at the benchmark configurations' own sizes, and the error of each
GPU result against the FP64 oracle.

Bit-exact (0 ULP) against the FP32 oracle, through the C ABI:
  * the 100,000-body stack (50 x 40 x 50 grid, 400,855 colliders), ticks 1-3:
    tick 1 is the overlapping start with about 14.0M candidate pairs and 9.5M
    contacts, the heaviest pass through the broadphase (lbvh.wgsl:84-398),
    the narrowphase (collision.wgsl:540-664) and the solve (:752-1069);
  * the 256-scene batch (body counts log-uniform in [64, 8192], 2% bearings),
    ticks 1-2;
  * 4,000 five-body bearing chains with 10% loop closures, in the reference's
    closure loop and in PCG to a 1e-5 relative residual.

FP64 error: for configs 1-3 the GPU state is loaded into the FP64 oracle,
which steps once; the GPU's FP32 poses, velocities and contact rows after the
same step are compared with it (oracle/errors.py).  The tables are printed in
the run's summary.  On the 100,000-body start the relaxed Jacobi solve
amplifies rounding differences (omega * lambda_max(D^-1 A) > 2 on its dense
contact graph), so there the velocities' FP64 error is reported, and bounded
only where the algorithm is stable.
"""
import numpy as np
import pytest

import oracle
from conftest import report
from mechanic_b200 import abi, learned, scenes
from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig
from oracle import errors

from test_gpu_parity import assert_bitwise, compare_tick

pytestmark = pytest.mark.gpu

def _need_host_memory(gb: float) -> None:
    """The oracle holds a heavy tick's pairs, contacts and manifold in host memory (about 15 GB
    for the 256-scene batch's 44M candidate pairs): skip rather than exhaust a small host."""
    import psutil
    avail = psutil.virtual_memory().available / 1e9
    if avail < gb:
        pytest.skip(f"needs {gb:.0f} GB of free host memory for the oracle, {avail:.0f} GB available")


# FP64 error bounds where the step is well conditioned (normwise relative,
# max |fp32 - fp64| / max |fp64|): a few hundred FP32 roundings deep.
REL_BOUND = 1e-4


def _start(gpu):
    st = gpu.save_state(manifold_capacity=1 << 24)
    return {"transforms": st["transforms"], "velocities": st["velocities"], "coordinates": st["coordinates"],
            "manifold": st["manifold"], "manifold_tick": st["manifold_tick"]}


def _fp64_table(name, scene, cfg, gpu, tick, pair_capacity):
    """Steps the GPU at `tick` and the FP64 oracle from the same state; returns the error table."""
    start = _start(gpu)
    gpu.dispatch_tick(tick)
    gpu.wait()
    st = gpu.save_state(manifold_capacity=0)
    res = {"transforms": st["transforms"], "velocities": st["velocities"], "contacts": gpu.contacts(),
           "contact_keys": gpu.contact_keys()}
    tab = errors.one_step_errors(scene, cfg.to_c(), start, tick, res, pair_capacity=pair_capacity)
    report(f"{name}: " + errors.summary_line(tab))
    return tab


def _assert_well_conditioned(tab):
    c = tab["counts"]
    assert c["fp32"] == c["fp64"] == c["matched"], c
    for key in ("position_m", "rotation", "linear_velocity_mps", "angular_velocity_rps", "point_arm_a_m",
                "point_arm_b_m", "depth_m", "normal", "impulse"):
        assert tab[key]["rel_inf"] <= REL_BOUND, (key, tab[key])


def test_plain_scale_full_size_ticks_1_to_3_bitexact(cuda_lib):
    _need_host_memory(16)
    scene = scenes.stack_grid(50, 40, 50, seed=0)
    cap = 1 << 24
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": cap})
    orc = oracle.OracleWorld(scene, cfg.to_c(), precision=32, pair_capacity=cap)
    compare_tick(gpu, orc, 1)
    rb = gpu.read_last_tick()
    assert (rb.pair_count, rb.contact_count) == (13_956_589, 9_469_469)
    for tick in (2, 3):
        compare_tick(gpu, orc, tick)
    gpu.close()


def test_plain_scale_fp64_error(cuda_lib):
    """One step from the generated state (tick 1, 9.5M contacts) and one from the state after
    tick 4 (a light tick), each against the FP64 oracle."""
    _need_host_memory(16)
    scene = scenes.stack_grid(50, 40, 50, seed=0)
    cap = 1 << 24
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": cap})
    heavy = _fp64_table("100k bodies, tick 1", scene, cfg, gpu, 1, cap)
    # the contact rows are written before the solve: only SAT decisions within rounding of a
    # threshold can differ between the precisions
    c = heavy["counts"]
    assert c["matched"] >= 0.999 * max(c["fp32"], c["fp64"]), c
    assert heavy["position_m"]["rel_inf"] <= 1e-6   # positions integrate the start velocities
    for tick in (2, 3, 4):
        gpu.dispatch_tick(tick)
    light = _fp64_table("100k bodies, tick 5", scene, cfg, gpu, 5, cap)
    c = light["counts"]
    assert c["matched"] >= 0.999 * max(c["fp32"], c["fp64"]), c
    assert light["position_m"]["rel_inf"] <= 1e-6
    gpu.close()


def test_plain_small_fp64_error(cuda_lib):
    scene = scenes.falling_cubes(1000, seed=0)
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics(scene, cfg)
    _assert_well_conditioned(_fp64_table("1,000 cubes, tick 1", scene, cfg, gpu, 1, 0))
    for tick in range(2, 31):
        gpu.dispatch_tick(tick)
    _assert_well_conditioned(_fp64_table("1,000 cubes, tick 31", scene, cfg, gpu, 31, 0))
    gpu.close()


def test_batched_256_scenes_full_size_bitexact(cuda_lib):
    _need_host_memory(48)
    lst = scenes.batched_uneven(256, seed=0)
    nb = sum(s.body_count for s in lst)
    nc = sum(s.collider_count for s in lst)
    cap = 1 << 26
    cfg = GpuPhysicsConfig()
    gpu = GpuPhysics.batch(lst, cfg, capacities={"max_bodies": nb, "max_colliders": nc, "max_bearings": 1 << 20,
                                                 "pair_capacity": cap})
    orc = oracle.OracleWorld.batch(lst, cfg.to_c(), pair_capacity=cap)
    for tick in (1, 2):
        compare_tick(gpu, orc, tick)
    gpu.close()


@pytest.mark.parametrize("mode", ["reference", "pcg"])
def test_chains_4000_full_size_bitexact(cuda_lib, mode):
    """The articulated config: 20,000 bodies in 4,000 five-body chains, 10% loop-closed."""
    scene = scenes.bearing_chains(4000)
    cfg = GpuPhysicsConfig() if mode == "reference" else learned.closure_config()
    cap = 1 << 22
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": cap})
    orc = oracle.OracleWorld(scene, cfg.to_c(), precision=32, pair_capacity=cap)
    for tick in (1, 2, 3):
        gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        orc.step(tick)
        d = orc.diagnostics()
        assert rb.error_flags == int(d["error_flags"]), tick
        assert (rb.pair_count, rb.contact_count) == (int(d["pair_count"]), int(d["contact_count"])), tick
        if mode == "pcg":
            assert rb.closure_iterations == orc.closure_stats()["pcg_iterations"], tick
        assert np.array_equal(gpu.pairs(), orc.pairs()), tick
        assert_bitwise(gpu.contacts(), orc.contacts(), f"tick {tick} contacts")
        st = gpu.save_state(manifold_capacity=0)
        tr, vel = orc.state()
        assert_bitwise(st["transforms"], tr, f"tick {tick} transforms")
        assert_bitwise(st["velocities"], vel, f"tick {tick} velocities")
        assert_bitwise(st["coordinates"], orc.coordinates(), f"tick {tick} coordinates")
    gpu.close()


@pytest.mark.parametrize("mode", ["reference", "pcg"])
def test_chains_4000_fp64_error(cuda_lib, mode):
    """One step of the articulated config against the FP64 oracle, with the reference's closure
    loop and with block-Jacobi PCG to a 1e-5 residual (the three-way comparison's GPU legs)."""
    scene = scenes.bearing_chains(4000)
    cfg = GpuPhysicsConfig() if mode == "reference" else learned.closure_config()
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": 1 << 22})
    for tick in (1, 2, 3):
        gpu.dispatch_tick(tick)
    tab = _fp64_table(f"4,000 chains ({mode} closures), tick 4", scene, cfg, gpu, 4, 1 << 22)
    c = tab["counts"]
    assert c["matched"] >= 0.999 * max(c["fp32"], c["fp64"], 1), c
    assert tab["position_m"]["rel_inf"] <= REL_BOUND
    gpu.close()
