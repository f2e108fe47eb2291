"""mechanic-bench compatible headless runner over the C ABI.

Mirrors crates/mechanic-bench/src/main.rs: scenario builders, a warm-up, a
measured tick loop (dispatch, wait, read_last_tick) and one JSON line with
the reference's field names and gate logic (main.rs:155-272).  Scenarios:

  smoke        1,024 touching 1 m cubes (main.rs:366, build_dense)
  dense_100k   100,000 touching 1 m cubes (main.rs:369, build_dense)
  plain_small  1,000 falling 0.25 m cubes with random pose and velocity
  plain_scale  100,000-body grid at 0.26 m with 20% hollow cylinders
  plain_medium the same mix on a 30 x 30 x 30 grid (27,000 bodies; profiling size)
  four_bar     four-bar linkage, first coordinate perturbed by 0.001 rad, collisions off
               (main.rs:113-132); passes with error_flags == 0
  invalid_loop the four-bar with its closure anchor moved (main.rs:211-216); passes when
               CONSTRAINT_NON_CONVERGENCE_FLAG is raised
  chains_20k   4,000 five-link bearing chains, 10% loop-closed (the articulated config)
  loops_100k   100 x 100 x 10 lattice of 1 m cubes joined by 198,009 bearings, 98,010 of them
               loop closures (main.rs:370, build_loops_100k)

    python -m mechanic_b200.bench_cli --scenario dense_100k [--seconds N] [--warmup N]
                                      [--ticks N] [--warmup-ticks N]
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import abi, scenes
from .physics import GpuPhysics, GpuPhysicsConfig

SCENARIOS = {
    "smoke": lambda: scenes.dense_grid(1024),
    "dense_100k": lambda: scenes.dense_grid(100_000),
    "plain_small": lambda: scenes.falling_cubes(1000, seed=0),
    "plain_scale": lambda: scenes.stack_grid(50, 40, 50, seed=0),
    "plain_medium": lambda: scenes.stack_grid(30, 30, 30, seed=0),
    "four_bar": lambda: scenes.four_bar(False),
    "invalid_loop": lambda: scenes.four_bar(True),
    "chains_20k": lambda: scenes.bearing_chains(),
    "loops_100k": lambda: scenes.loops_grid(100, 100, 10),
}
SHORT = {"smoke", "plain_small", "four_bar", "invalid_loop"}
LINKAGES = {"four_bar", "invalid_loop"}


def percentile_95(sorted_values):
    """main.rs:546-549: rank = ceil(len * 95 / 100)."""
    rank = math.ceil(len(sorted_values) * 95 / 100)
    return sorted_values[max(rank, 1) - 1]


def run(scenario: str, seconds: int | None, warmup: int | None, ticks: int | None,
        warmup_ticks: int | None, pair_capacity: int) -> dict:
    start = time.perf_counter()
    scene = SCENARIOS[scenario]()
    construction_ms = (time.perf_counter() - start) * 1e3
    seconds = seconds if seconds is not None else (1 if scenario in SHORT else 30)
    warmup = warmup if warmup is not None else (0 if scenario in SHORT else 5)
    warm = warmup_ticks if warmup_ticks is not None else warmup * 60
    measured = ticks if ticks is not None else seconds * 60
    cfg = GpuPhysicsConfig(solver_iterations=8, collisions_enabled=scenario not in LINKAGES)
    gpu = GpuPhysics(scene, cfg, capacities={"pair_capacity": pair_capacity})
    if scenario in LINKAGES:   # main.rs:114-131: perturb the first coordinate by 0.001 rad
        coords = np.zeros(scene.coordinate_count, abi.MECHANISM_COORDINATE)
        coords["angle"][0] = 0.001
        gpu.initialize_mechanism_coordinates(coords)
    for tick in range(1, warm + 1):
        gpu.dispatch_tick(tick)
    gpu.wait()
    engine, gpu_ms = [], []
    stages = [[] for _ in range(7)]
    flags = pairs = contacts = active = 0
    anchor = axis = 0.0
    for tick in range(1, measured + 1):
        t0 = time.perf_counter()
        sub = gpu.dispatch_tick(warm + tick)
        gpu.wait(sub.submission_index)
        rb = gpu.read_last_tick()
        flags |= rb.error_flags
        pairs, contacts, active = max(pairs, rb.pair_count), max(contacts, rb.contact_count), \
            max(active, rb.active_contact_count)
        anchor, axis = max(anchor, rb.anchor_residual_meters), max(axis, rb.axis_residual_degrees)
        gpu_ms.append(rb.gpu_tick_ms)
        kt = rb.kernel_timings
        for s, v in zip(stages, (kt.integration_ms, kt.mechanism_ms, kt.broadphase_ms, kt.narrowphase_ms,
                                 kt.contact_solver_ms, kt.bearings_ms, kt.snapshot_ms)):
            s.append(v)
        engine.append((time.perf_counter() - t0) * 1e3)
    engine.sort()
    gpu_ms.sort()
    for s in stages:
        s.sort()
    mean = sum(engine) / len(engine)
    tps = 1000.0 / mean
    gpu_p95 = percentile_95(gpu_ms)
    if scenario == "invalid_loop":   # main.rs:211-216: the bad loop must be reported
        correctness = bool(flags & abi.CONSTRAINT_NON_CONVERGENCE_FLAG)
    else:
        correctness = flags == 0
    budget = tps >= 60.0 and gpu_p95 <= 16.67
    out = {
        "type": "benchmark", "scenario": scenario, "adapter": "NVIDIA B200 (libmechanic_b200)",
        "backend": "CUDA", "bodies": scene.body_count, "colliders": scene.collider_count,
        "bearings": scene.bearing_count, "warmup_ticks": warm, "measured_ticks": measured,
        "construction_ms": round(construction_ms, 3), "mean_engine_tick_ms": round(mean, 3),
        "p95_engine_tick_ms": round(percentile_95(engine), 3), "p95_gpu_tick_ms": round(gpu_p95, 3),
        "kernel_pipeline_p95_ms": round(gpu_p95, 3), "physics_tps": round(tps, 2),
    }
    for name, s in zip(("integration", "mechanism", "broadphase", "narrowphase", "contact_solver", "bearings",
                        "snapshot"), stages):
        out[f"kernel_{name}_p95_ms"] = round(percentile_95(s), 3)
    out.update({"pairs": pairs, "contacts": contacts, "active_contacts": active,
                "anchor_residual_m": round(anchor, 8), "axis_residual_deg": round(axis, 8),
                "error_flags": flags, "timing_source": "cuda_events", "kernel_coverage_complete": True,
                "correctness_passed": correctness, "budget_passed": budget,
                "gate_passed": correctness and budget})
    gpu.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="mechanic_b200.bench_cli")
    ap.add_argument("--scenario", default="smoke", choices=sorted(SCENARIOS))
    ap.add_argument("--seconds", type=int)
    ap.add_argument("--warmup", type=int)
    ap.add_argument("--ticks", type=int, help="measured ticks (overrides --seconds)")
    ap.add_argument("--warmup-ticks", type=int, help="warm-up ticks (overrides --warmup)")
    ap.add_argument("--pair-capacity", type=int, default=1 << 24)
    ap.add_argument("--exit-zero", action="store_true",
                    help="exit 0 whatever the gate says (runs under a profiler, whose replays break the budget)")
    a = ap.parse_args(argv)
    out = run(a.scenario, a.seconds, a.warmup, a.ticks, a.warmup_ticks, a.pair_capacity)
    print(json.dumps(out), flush=True)
    return 0 if out["gate_passed"] or a.exit_zero else 1


if __name__ == "__main__":
    raise SystemExit(main())
