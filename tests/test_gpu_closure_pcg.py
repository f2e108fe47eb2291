"""Closure solve to a residual (MK_CLOSURE_PCG_RESIDUAL) against the CPU oracle.

PCG per Newton step with FP64 dot products summed in one fixed order, 2 x 2
block-Jacobi preconditioner: GPU and oracle agree bit for bit (0 ULP) on the
coordinates and the body state, and on the iteration counts.  With the
learned preconditioner the network outputs (tensor-core arithmetic) are read
back from the GPU and given to the oracle, and the rest must again agree bit
for bit.
"""
import numpy as np
import pytest

import oracle
from mechanic_b200 import abi, learned, scenes
from mechanic_b200.net_init import init_params
from mechanic_b200.physics import GpuPhysics

from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def _run(scene, cfg, ticks, coords=None, params=None):
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": 1 << 20})
    orc = oracle.OracleWorld(scene, cfg.to_c(), pair_capacity=1 << 20)
    if coords is not None:
        gpu.initialize_mechanism_coordinates(coords)
        orc.set_coordinates(coords)
    if params is not None:
        gpu.set_preconditioner_network(params)
    for tick in range(1, ticks + 1):
        gpu.dispatch_tick(tick)
        rb = gpu.read_last_tick()
        if params is not None:
            orc.set_precond_outputs(gpu.closure_block_outputs())
        orc.step(tick)
        cs = orc.closure_stats()
        assert rb.closure_iterations == cs["pcg_iterations"], f"tick {tick}"
        assert rb.closure_relative_residual == cs["max_relative_residual"], f"tick {tick}"
        assert rb.error_flags == int(orc.diagnostics()["error_flags"])
        st = gpu.save_state(manifold_capacity=0)
        tr, vel = orc.state()
        assert_bitwise(st["transforms"], tr, f"tick {tick} transforms")
        assert_bitwise(st["velocities"], vel, f"tick {tick} velocities")
        assert_bitwise(st["coordinates"], orc.coordinates(), f"tick {tick} coordinates")
    gb, ob = gpu.closure_blocks(), orc.closure_blocks()
    cols = [c for c in range(16) if c != 6]   # column 6 is log(a / d): CUDA logf against a rounded double log
    np.testing.assert_array_equal(gb[:, cols], ob[:, cols])
    np.testing.assert_allclose(gb[:, 6], ob[:, 6], rtol=1e-6, atol=1e-7)
    return gpu, orc


def test_four_bar_pcg_bitexact(cuda_lib):
    cfg = learned.closure_config(collisions_enabled=False)
    coords = np.zeros(3, abi.MECHANISM_COORDINATE)
    coords["angle"][0] = 0.001
    gpu, orc = _run(scenes.four_bar(False), cfg, 60, coords)
    assert gpu.read_last_tick().error_flags == 0


def test_chains_pcg_loop_blocks_bitexact(cuda_lib):
    cfg = learned.closure_config()
    gpu, orc = _run(scenes.bearing_chains(chains=40, links=5, seed=1, closure_fraction=0.5, height=0.5), cfg, 10)
    # per-loop blocks are exact up to the ridge: one or two iterations per Newton step
    cs = orc.closure_stats()
    assert cs["pcg_iterations"] <= 2 * cs["newton_steps"]
    assert cs["max_relative_residual"] <= 1e-5


@pytest.mark.parametrize("mode", [1, 2], ids=["block", "grid"])
def test_long_loops_pcg_pieces_bitexact(cuda_lib, mode):
    """Sixteen-body loops (15 closure coordinates each, more than one block holds): the
    per-loop blocks are pieces of 5 coordinates, the rank of a closure's constraint rows, so
    every piece is positive definite; one block and the whole grid match the oracle."""
    cfg = learned.closure_config(max_iterations=64)
    prev = _closure_grid(mode)
    try:
        gpu, orc = _run(scenes.bearing_chains(chains=24, links=16, seed=3, closure_fraction=1.0, height=0.5),
                        cfg, 4)
    finally:
        _closure_grid(max(prev, 0))
    assert orc.closure_stats()["max_relative_residual"] < 1.0   # the iteration does not blow up


def test_chains_pcg_pair_blocks_bitexact(cuda_lib):
    cfg = learned.closure_config(max_iterations=64)
    cfg.preconditioner = abi.PRECOND_PAIR_BLOCKS
    _run(scenes.bearing_chains(chains=40, links=5, seed=1, closure_fraction=0.5, height=0.5), cfg, 8)


def test_learned_preconditioner_bitexact_given_outputs(cuda_lib):
    cfg = learned.closure_config(learned=True, max_iterations=64)
    gpu, orc = _run(scenes.bearing_chains(chains=40, links=5, seed=2, closure_fraction=0.5, height=0.5), cfg, 6,
                    params=init_params(9, out_scale=1.0))
    cs = orc.closure_stats()
    assert cs["learned_blocks"] + cs["rejected_blocks"] > 0


def _closure_grid(mode):
    from mechanic_b200 import physics
    return physics.set_tuning(physics.TUNE_CLOSURE_GRID, mode)


@pytest.mark.parametrize("precond", [abi.PRECOND_BLOCK_JACOBI, abi.PRECOND_PAIR_BLOCKS])
def test_grid_closure_pcg_bitexact(cuda_lib, precond):
    """The evaluate and PCG kernels spread over the whole cooperative grid (grid barriers
    between phases) agree with the oracle bit for bit."""
    cfg = learned.closure_config(max_iterations=64)
    cfg.preconditioner = precond
    prev = _closure_grid(2)
    try:
        _run(scenes.bearing_chains(chains=40, links=5, seed=1, closure_fraction=0.5, height=0.5), cfg, 6)
    finally:
        _closure_grid(max(prev, 0))


def test_grid_and_block_closure_pcg_agree_and_match_oracle(cuda_lib):
    """Above 1,024 closure coordinates the FP64 dot products sum per 1,024-coordinate
    chunk in chunk order: one block and the whole grid give the oracle's values."""
    scene = scenes.bearing_chains(chains=1500, links=5, seed=6, closure_fraction=0.2, height=0.5)
    cfg = learned.closure_config()
    for mode in (1, 2):
        prev = _closure_grid(mode)
        try:
            _run(scene, cfg, 3)
        finally:
            _closure_grid(max(prev, 0))
