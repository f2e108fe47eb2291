"""GPU parity of the articulated passes against the CPU oracle (through the C ABI).

Forward kinematics, bearing projection, coordinate advance and capture,
level-synchronous velocity reconstruction, validation and the loop-closure
Newton/PCG steps follow the oracle's arithmetic order; closure systems with
at most 512 coordinates also keep its summation order, so every case here is
compared bit for bit (0 ULP).
"""
import numpy as np
import pytest

import oracle
from mechanic_b200 import abi, scenes
from mechanic_b200.physics import CoordinateStateCount, DriveStateCount, GpuPhysics, GpuPhysicsConfig

pytestmark = pytest.mark.gpu


def _same(a, b, what):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    if a.tobytes() != b.tobytes():
        fa, fb = a.view(np.float32).reshape(len(a), -1), b.view(np.float32).reshape(len(b), -1)
        bad = np.nonzero((fa.view(np.uint32) != fb.view(np.uint32)).any(axis=1))[0]
        raise AssertionError(f"{what}: {len(bad)} rows differ, first {bad[:4]}: {fa[bad[:2]]} vs {fb[bad[:2]]}")


def _pair(scene, cfg):
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": 1 << 20})
    orc = oracle.OracleWorld(scene, cfg.to_c(), precision=32, pair_capacity=1 << 20)
    return gpu, orc


def _compare(gpu, orc, tick, what):
    gpu.dispatch_tick(tick)
    rb = gpu.read_last_tick()
    orc.step(tick)
    d = orc.diagnostics()
    assert rb.error_flags == int(d["error_flags"]), f"{what} tick {tick} flags"
    assert round(rb.anchor_residual_meters * 1e6) == int(d["max_anchor_micrometers"])
    assert round(rb.axis_residual_degrees * 1e6) == int(d["max_axis_microdegrees"])
    st = gpu.save_state(manifold_capacity=0)
    tr, vel = orc.state()
    _same(st["transforms"], tr, f"{what} tick {tick} transforms")
    _same(st["velocities"], vel, f"{what} tick {tick} velocities")
    _same(st["coordinates"], orc.coordinates(), f"{what} tick {tick} coordinates")
    return rb


@pytest.mark.parametrize("invalid", [False, True])
def test_four_bar_bitexact_and_gate(cuda_lib, invalid):
    scene = scenes.four_bar(invalid)
    cfg = GpuPhysicsConfig(collisions_enabled=False)
    gpu, orc = _pair(scene, cfg)
    coords = np.zeros(3, abi.MECHANISM_COORDINATE)
    coords["angle"][0] = 0.001
    gpu.initialize_mechanism_coordinates(coords)
    orc.set_coordinates(coords)
    flags = 0
    for tick in range(1, 61):
        flags |= _compare(gpu, orc, tick, "four_bar").error_flags
    _same(gpu.links(), orc.links(), "final links")
    if invalid:
        assert flags & abi.CONSTRAINT_NON_CONVERGENCE_FLAG
    else:
        assert flags == 0


def test_chains_with_closures_and_contacts_bitexact(cuda_lib):
    scene = scenes.bearing_chains(chains=40, links=5, seed=1, closure_fraction=0.3, height=0.5)
    gpu, orc = _pair(scene, GpuPhysicsConfig())
    for tick in range(1, 31):
        _compare(gpu, orc, tick, "chains")
    assert np.array_equal(gpu.pairs(), orc.pairs())


def _with_closure_grid(mode, make):
    from mechanic_b200 import physics
    prev = physics.set_tuning(physics.TUNE_CLOSURE_GRID, mode)
    try:
        return make()
    finally:
        physics.set_tuning(physics.TUNE_CLOSURE_GRID, max(prev, 0))


def test_grid_closure_loop_bitexact(cuda_lib):
    """The closure loop spread over the whole cooperative grid (grid barriers between its
    phases) gives the oracle's values bit for bit on a system small enough for the serial
    dot order."""
    scene = scenes.bearing_chains(chains=40, links=5, seed=1, closure_fraction=0.3, height=0.5)
    gpu, orc = _with_closure_grid(2, lambda: _pair(scene, GpuPhysicsConfig()))
    for tick in range(1, 16):
        _compare(gpu, orc, tick, "grid closure loop")


def test_grid_and_block_closure_loops_agree(cuda_lib):
    """Above 1,024 closure coordinates the dot products sum per 1,024-coordinate chunk in
    chunk order, so one block and the whole grid compute the same values."""
    scene = scenes.bearing_chains(chains=3000, links=5, seed=4, closure_fraction=0.1, height=0.5)
    runs = []
    for mode in (1, 2):
        gpu = _with_closure_grid(mode, lambda: GpuPhysics(scene, GpuPhysicsConfig(), capacities={"pair_capacity": 1 << 21}))
        for tick in range(1, 9):
            gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        runs.append((gpu.save_state(manifold_capacity=0), rb))
        gpu.close()
    (a, ra), (b, rb) = runs
    assert ra.closure_iterations == rb.closure_iterations
    _same(a["transforms"], b["transforms"], "grid vs block transforms")
    _same(a["velocities"], b["velocities"], "grid vs block velocities")
    _same(a["coordinates"], b["coordinates"], "grid vs block coordinates")


def test_chains_without_self_collisions_bitexact(cuda_lib):
    scene = scenes.bearing_chains(chains=16, links=5, seed=3, closure_fraction=0.0, height=0.3)
    gpu, orc = _pair(scene, GpuPhysicsConfig(mechanism_self_collisions=False))
    for tick in range(1, 21):
        _compare(gpu, orc, tick, "chains no self collision")


def test_drive_and_coordinate_counts_are_checked(cuda_lib):
    scene = scenes.bearing_chains(chains=4, links=5, seed=0)
    gpu = GpuPhysics(scene)
    with pytest.raises(DriveStateCount) as e:
        gpu.write_mechanism_drives(abi.passive_drive_rows(3))
    assert (e.value.provided, e.value.required) == (3, 16)
    with pytest.raises(CoordinateStateCount):
        gpu.initialize_mechanism_coordinates(np.zeros(15, abi.MECHANISM_COORDINATE))
    gpu.write_mechanism_drives(abi.passive_drive_rows(16))
    gpu.dispatch_tick(1)
    assert gpu.read_last_tick().error_flags & abi.INVALID_NUMERIC_FLAG == 0


@pytest.mark.parametrize("scenario", ["four_bar", "invalid_loop"])
def test_bench_runner_linkage_gates(cuda_lib, scenario):
    """The mechanic-bench gates (main.rs:113-132, 211-216) through the runner."""
    from mechanic_b200 import bench_cli
    out = bench_cli.run(scenario, None, None, 120, 0, 1 << 16)
    assert out["correctness_passed"], out["error_flags"]
    if scenario == "four_bar":
        assert out["anchor_residual_m"] <= 1e-5


@pytest.mark.parametrize("mode", ["reference", "pcg"])
def test_loop_lattice_long_slot_runs_bitexact(cuda_lib, mode):
    """mechanic-bench's loop lattice (main.rs:456-524) at 20 x 20 x 3: 1,083 closures on one
    spanning tree, so the coordinates near its root lie on hundreds of closure branches (38 of
    them on more than 256, up to 1,444).  Those runs are summed by a warp in the same serial
    order as the one-thread runs: coordinates, state and contacts equal the oracle's bit for bit."""
    from mechanic_b200 import learned
    scene = scenes.loops_grid(20, 20, 3)
    cfg = GpuPhysicsConfig() if mode == "reference" else learned.closure_config(
        preconditioner=abi.PRECOND_DIAGONAL, max_iterations=16)
    gpu, orc = _pair(scene, cfg)
    # disturb the lattice so the closures are not converged from the start
    coords = np.zeros(scene.coordinate_count, abi.MECHANISM_COORDINATE)
    coords["angle"][::7] = 0.01
    gpu.initialize_mechanism_coordinates(coords)
    orc.set_coordinates(coords)
    for tick in range(1, 4):
        _compare(gpu, orc, tick, f"loop lattice {mode}")
    _same(gpu.contacts(), orc.contacts(), "loop lattice contacts")
