"""Benchmark: body-steps/s of the rigid-body step at 100,000 bodies.

Workload (N=1): the 100,000-body stack (50x40x50 grid at 0.26 m, 20% hollow
cylinders with 16 OBB segments each, 400,855 colliders, 8 PGS iterations),
stepped K ticks from its generated state; a step is one tick of the whole
scene.  Warm-up ticks run from the same state, which is then reloaded, so
the timed ticks are ticks 1..K of the configuration's trajectory whatever W
is.  With torchrun (N>1) every rank steps its own replica (a single scene
does not shard) and the slowest rank's device time sets the throughput.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  Device time comes from CUDA events around each tick's
graph launch on the handle's stream; between ticks L2 is not flushed because
the state a tick reads and writes (about 150 MB at this size, stated in the
JSON line) is larger than the 126 MB L2 (--flush-l2 zeroes a 256 MB buffer
between ticks instead); `e2e`
repeats the run through the C ABI with a per-tick host readback of the
snapshot ring (what a renderer consumes) and the diagnostics, wall-clocked.
The reference arm times the CPU restatement of the same tick on all host
cores (the reference's own wgpu pipeline needs a graphics stack, which this
machine does not have).

Two further measurements ride along in the same JSON line ("forms"):
  residual_1e-5  the contact solve iterated to a 1e-5 relative residual, the
                 cached (plain) start against the learned warm start, on the
                 1,000-cube config (60 ticks).  The 100,000-body config is not
                 used for it: its overlapping start has dozens of contacts per
                 body, where the reference's relaxed Jacobi (omega 0.125)
                 diverges when it is iterated beyond its fixed 8 passes.
  batched        the 256-scene batched config (body counts log-uniform in
                 [64, 8192], about 413,000 bodies, 2% bearings) in one handle,
                 K ticks; under torchrun the scenes are sharded across ranks
                 (contiguous ranges balanced by body count) and the slowest
                 rank's device time sets the throughput.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "body-steps/s at 100k bodies, plain vs learned+batched, at equal 1e-5 residual"
UNIT = "body-steps/s"
WORKLOAD = "plain step, 100,000 bodies (50x40x50 grid, 0.26 m, 20% hollow cylinders), 8 PGS iterations"
PAIR_CAPACITY = 1 << 24
# Algorithmic bytes (minimal compulsory traffic) per unit, FP32 rows as in the ABI.
BYTES_SOLVE_PER_CONTACT_ITER = 284     # contact 64 + idx 4 + 2 x (v 16 + w 16 + world mass 48) + lambda 4 + 2 x 24 deltas
BYTES_APPLY_PER_BODY_ITER = 112        # deltas 24 + velocities 32 read, velocities 32 + deltas 24 written
BYTES_PREPARE_PER_CONTACT = 340        # contact 64 + 2 x (v/w 32 + world mass 48) + manifold 96, 16 + 48 + 4 written
# broadphase per collider: AABB + Morton 140 (collider 64 + pose 32 read, AABB 32 + key/value 12 written),
# onesweep sort 2 x 12 per 8-bit digit pass over the key mode's bits + 12 histogram read, Karras 24,
# refit 96 + 32, traversal 32
KEY_BITS = {0: 63, 1: 30, 2: 48, 3: 39, 4: 30}   # MK_MORTON_63, _REFERENCE_30, _48, _39, _30_ADAPTIVE


def bytes_broadphase_per_collider(morton_mode: int) -> int:
    passes = (KEY_BITS[morton_mode] + 7) // 8
    return 140 + (2 * 12 * passes + 12) + 24 + 96 + 32 + 32
# per candidate pair: traversal output 8 + pair-key sort (5 digit passes x 16 + 8)
BYTES_BROADPHASE_PER_PAIR = 8 + 88


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the residual-form and batched measurements")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--flush-l2", action="store_true", help="zero a 256 MB buffer between timed ticks")
    ap.add_argument("--full-form", action="store_true",
                    help="measure the 1,250,000-body full form (reference passes, plain and learned to 1e-5) and exit")
    ap.add_argument("--long-loops", action="store_true",
                    help="the closure preconditioners on 400 sixteen-body loops (longer than one per-loop block) "
                         "and exit")
    ap.add_argument("--cpu-table", action="store_true",
                    help="time the CPU restatement on every configuration (all cores and one core) and exit")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        # nvidia-smi needs a moment to start: wait for its first row, then keep only
        # the rows that arrive from here on
        self.skip = 0
        deadline = time.time() + 5.0
        while self.proc is not None and time.time() < deadline and self._rows() == 0:
            time.sleep(0.02)
        self.skip = self._rows()
        return self

    def _rows(self):
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.endswith("\n"))
        except OSError:
            return 0

    def __exit__(self, *exc):
        if self.proc is not None:
            # a short timed region may end between two samples: wait (bounded) for the
            # sample that covers its end
            deadline = time.time() + 1.0
            while time.time() < deadline and self._rows() < self.skip + 2:
                time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        lines = open(self.path).readlines()
        for line in lines[max(self.skip - 1, 0):]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]), "power": float(parts[3]),
                             "hw": parts[5], "hw_thermal": parts[6], "sw_thermal": parts[7],
                             "power_cap": parts[8]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [r for r in rows if r["power"] > 200.0] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hw_thermal", "hw_thermal_slowdown"),
                          ("sw_thermal", "sw_thermal_slowdown"), ("power_cap", "sw_power_cap")):
            if any(r[key].lower() == "active" for r in rows):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded), "sm_max_mhz": max(r["max"] for r in rows),
                "samples": len(rows), "samples_under_load": len(loaded), "reasons": reasons}


# ------------------------------------------------------------- cpu legs
def bench_config(scene, args, world: int = 1) -> dict:
    """The workload description both arms print (the same keys and values)."""
    # HBM state every tick reads and writes: per body position, rotation, velocities,
    # inverse mass, mass row, world inverse inertia, root flag, deltas, snapshot (240 B);
    # per collider its row, world box, AABB, keys and values (ping-pong), LBVH node boxes,
    # records, children, parents and visit counters (316 B)
    working_set = 240 * scene.body_count + 316 * scene.collider_count
    return {"workload": WORKLOAD, "bodies": scene.body_count, "colliders": scene.collider_count,
            "ticks": f"1..{args.steps} from the generated state (warm-up state reloaded)",
            "seed": args.seed, "pair_capacity": PAIR_CAPACITY,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": ("flushed between ticks (256 MB written)" if args.flush_l2 else
                   f"not flushed: per-tick state {working_set / 1e6:.0f} MB > 126 MB L2")}


def cpu_trajectory(scene, ticks: int, budget_s: float, threads: int, keep_world: bool = False):
    """Steps the CPU oracle along ticks 1..ticks, stopping early once budget_s has passed.
    With keep_world the oracle world comes back as a fourth item (its state after the
    last tick stepped), so the same sample also serves as the checker of the GPU run."""
    import oracle
    from mechanic_b200.physics import GpuPhysicsConfig
    oracle.set_threads(threads)
    w = oracle.OracleWorld(scene, GpuPhysicsConfig().to_c(), pair_capacity=PAIR_CAPACITY)   # the GPU arm's config
    t0 = time.perf_counter()
    done = 0
    for tick in range(1, ticks + 1):
        w.step(tick)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    elapsed = time.perf_counter() - t0
    if keep_world:
        return done, elapsed, oracle.threads(), w
    return done, elapsed, oracle.threads()


def parity_against_oracle(gpu, scene, reset, done: int, world) -> dict:
    """Checks the GPU's trajectory with the CPU baseline's own sample: the GPU steps ticks
    1..done again from the generated state (outside every timed region) and its poses and
    velocities are compared bit for bit with the FP32 oracle's after the same ticks; then
    one more tick from that identical state is compared with the FP64 oracle (normwise
    relative error of each quantity)."""
    import numpy as np
    from oracle import errors
    from mechanic_b200.physics import GpuPhysicsConfig
    reset()
    for tick in range(1, done + 1):
        gpu.dispatch_tick(tick)
    gpu.wait()
    cap = 1 << 21   # the manifold of a light tick (tens of thousands of rows)
    st = gpu.save_state(manifold_capacity=cap)
    tr, vel = world.state()
    same_tr = bool(np.array_equal(np.ascontiguousarray(st["transforms"]).view(np.uint8),
                                  np.ascontiguousarray(tr).view(np.uint8)))
    same_vel = bool(np.array_equal(np.ascontiguousarray(st["velocities"]).view(np.uint8),
                                   np.ascontiguousarray(vel).view(np.uint8)))
    out = {"checker": f"FP32 oracle over ticks 1..{done} (the cpu_baseline sample)", "ticks_bitexact": done,
           "transforms_bitexact": same_tr, "velocities_bitexact": same_vel, "fp64_one_step": None}
    if len(st["manifold"]) >= cap:   # a heavy tick's manifold: too large for a one-step FP64 check here
        return out
    start = {"transforms": st["transforms"], "velocities": st["velocities"], "coordinates": st["coordinates"],
             "manifold": st["manifold"], "manifold_tick": st["manifold_tick"]}
    nxt = done + 1
    gpu.dispatch_tick(nxt)
    gpu.wait()
    after = gpu.save_state(manifold_capacity=0)
    res = {"transforms": after["transforms"], "velocities": after["velocities"], "contacts": gpu.contacts(),
           "contact_keys": gpu.contact_keys()}
    tab = errors.one_step_errors(scene, GpuPhysicsConfig().to_c(), start, nxt, res, pair_capacity=PAIR_CAPACITY)
    keys = ("position_m", "rotation", "linear_velocity_mps", "angular_velocity_rps", "point_arm_a_m", "depth_m",
            "normal", "impulse")
    out["checker"] += f", then the FP64 oracle for tick {nxt} from the identical state"
    out["fp64_one_step"] = {"tick": nxt, "contacts": tab["counts"],
                            "rel_inf": {k: tab[k]["rel_inf"] for k in keys},
                            "max_abs": {k: tab[k]["max_abs"] for k in keys}}
    return out


def cpu_table(budget_s: float = 20.0) -> dict:
    """The CPU restatement timed on the host's cores and on one core for every
    configuration (a bounded sample of each: the ticks that fit `budget_s`, at
    least one), for the CPU baseline table.  Prints nothing; returns the rows."""
    import oracle
    from mechanic_b200 import learned, scenes
    from mechanic_b200.physics import GpuPhysicsConfig
    oracle.build()
    cores = os.cpu_count() or 1
    # (name, scenes, config, ticks, thread counts).  The overlapping first tick of configs 2
    # and 4 (14M and 44M candidate pairs) takes minutes on one core, so those are timed on
    # all cores only; config 5's first tick (145M pairs) needs more host memory than a
    # sample is worth and is not timed.
    configs = [
        ("1: 1,000 cubes", lambda: [scenes.falling_cubes(1000, seed=0)], GpuPhysicsConfig(), 60, (cores, 1)),
        ("2: 100,000 mixed bodies", lambda: [scenes.stack_grid(50, 40, 50, seed=0)], GpuPhysicsConfig(), 120,
         (cores,)),
        ("3: 4,000 chains, closure PCG to 1e-5", lambda: [scenes.bearing_chains(4000)],
         learned.closure_config(), 60, (cores, 1)),
        ("4: 256 batched scenes", lambda: scenes.batched_uneven(256, seed=0), GpuPhysicsConfig(), 60, (cores,)),
    ]
    rows = []
    for name, make, cfg, ticks, thread_counts in configs:
        lst = make()
        for threads in thread_counts:
            oracle.set_threads(threads)
            w = (oracle.OracleWorld.batch(lst, cfg.to_c(), pair_capacity=1 << 28) if len(lst) > 1 else
                 oracle.OracleWorld(lst[0], cfg.to_c(), pair_capacity=1 << 28))
            bodies = sum(x.body_count for x in lst)
            t0 = time.perf_counter()
            done = 0
            for tick in range(1, ticks + 1):
                w.step(tick)
                done += 1
                if time.perf_counter() - t0 > budget_s:
                    break
            el = time.perf_counter() - t0
            rows.append({"config": name, "threads": oracle.threads(), "ticks": f"1..{done} of {ticks}",
                         "seconds": round(el, 2), "body_steps_per_s": bodies * done / el})
            del w
    return {"cpu_table": rows, "host_cores": cores}


def run_reference(args, scene):
    """The CPU restatement on all host cores (reference arm)."""
    threads = os.cpu_count() or 1
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    from mechanic_b200.physics import GpuPhysicsConfig
    warm = oracle.OracleWorld(scene, GpuPhysicsConfig().to_c(), pair_capacity=PAIR_CAPACITY)
    for tick in range(1, args.warmup + 1):
        warm.step(tick)
    del warm
    done, elapsed, used = cpu_trajectory(scene, args.steps, 150.0, threads)
    value = scene.body_count * done / elapsed
    sample = (f"ticks 1..{done} of the {args.steps}-tick trajectory of the same scene, CPU restatement "
              f"(oracle, FP32) on {used} threads")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 0,
        "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": bench_config(scene, args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's wgpu pipeline needs a graphics stack that is unavailable on this box; "
                "this arm times the CPU restatement of the same tick",
    }


# ------------------------------------------------------------ extra forms
def measure_residual_forms(local: int, ticks: int = 60):
    """Config 1 iterated to a 1e-5 residual: cached start against the learned one."""
    import torch
    from mechanic_b200 import learned, scenes
    from mechanic_b200.physics import GpuPhysics
    weights = os.path.join(ROOT, "mechanic_b200", "data", "warm_start.npy")
    params = np.load(weights) if os.path.exists(weights) else None
    scene = scenes.falling_cubes(1000, seed=0)
    out = {"workload": "1,000 cubes, 60 ticks, contact passes until ||r|| <= 1e-5 ||r_cold|| (cap 512)"}
    forms = [("plain", learned.residual_config(device=local), None)]
    if params is not None:
        forms.append(("learned", learned.residual_config(learned=True, device=local), params))
    for name, cfg, prm in forms:
        with GpuPhysics(scene, cfg) as g:
            if prm is not None:
                g.set_warm_start_network(prm)
            passes, ms, used, conv = [], 0.0, {}, 0
            torch.cuda.synchronize()
            for t in range(1, ticks + 1):
                g.dispatch_tick(t)
                rb = g.read_last_tick()
                passes.append(rb.contact_iterations)
                ms += rb.gpu_tick_ms
                used[rb.warm_start_used] = used.get(rb.warm_start_used, 0) + 1
                conv += int(rb.contact_relative_residual <= 1e-5)
        out[name] = {"value": scene.body_count * ticks / (ms / 1e3), "unit": UNIT,
                     "passes_per_tick": float(np.mean(passes)), "ticks_converged": conv, "ticks": ticks,
                     "start_used": {("cached", "learned", "learned rejected")[k]: v for k, v in used.items()}}
    if "learned" in out:
        out["pass_ratio_plain_over_learned"] = out["plain"]["passes_per_tick"] / max(out["learned"]["passes_per_tick"], 1e-9)
    return out


def measure_closure_forms(local: int, ticks: int = 20, chains: int = 4000, links: int = 5,
                          closure_fraction: float = 0.1):
    """The articulated config (4,000 five-body chains, 10% loop-closed; or other chains):
    closure PCG to a 1e-5 relative residual under each preconditioner -- the reference's
    diagonal (Jacobi) one, exact 2 x 2 blocks, the network-corrected 2 x 2 blocks (trained
    here on the GPU on the first ticks' systems) and per-loop block Jacobi (exact on loops of
    at most 8 coordinates; longer loops are cut into blocks of 8).  PCG iterations per tick
    (12 Newton steps, at most 256 iterations each), the largest relative residual reached, and
    the device time per tick."""
    from mechanic_b200 import abi, learned, scenes
    from mechanic_b200.physics import GpuPhysics
    scene = scenes.bearing_chains(chains, links=links, closure_fraction=closure_fraction)
    xs, ts, _ = learned.collect_closure_samples(scene, 8, learned.closure_config(
        preconditioner=abi.PRECOND_PAIR_BLOCKS, device=local))
    out = {"workload": f"{chains} chains of {links} bodies, {closure_fraction:.0%} loop-closed, closure PCG until "
                       f"||r|| <= 1e-5 ||r0|| (cap 256 per Newton step), ticks 1..{ticks}"}
    forms = [("diagonal (reference Jacobi)", abi.PRECOND_DIAGONAL), ("pair blocks", abi.PRECOND_PAIR_BLOCKS)]
    if len(xs):
        params, _ = learned.train_preconditioner(xs, ts, steps=2000)
        out["training"] = f"network trained on {len(xs)} 2 x 2 blocks of ticks 1-8 (pair-block runs)"
        forms.append(("learned pair blocks", abi.PRECOND_LEARNED))
    else:   # a loop of more than five coordinates has a singular J^T J: its blocks have no inverse to learn
        params = None
        out["training"] = ("no training targets: every loop's J^T J is singular (more coordinates than the rank "
                           "5 of its closure's rows)")
    forms.append(("block Jacobi (per loop)", abi.PRECOND_BLOCK_JACOBI))
    for name, pc in forms:
        with GpuPhysics(scene, learned.closure_config(preconditioner=pc, device=local)) as g:
            if pc == abi.PRECOND_LEARNED:
                g.set_preconditioner_network(params)
            its, res, ms = [], [], 0.0
            for t in range(1, ticks + 1):
                g.dispatch_tick(t)
                rb = g.read_last_tick()
                its.append(rb.closure_iterations)
                res.append(rb.closure_relative_residual)
                ms += rb.gpu_tick_ms
        out[name] = {"pcg_iterations_per_tick": float(np.mean(its)), "max_relative_residual": float(np.max(res)),
                     "ticks_at_tolerance": int(sum(r <= 1e-5 for r in res)), "ms_per_tick": ms / ticks}
    d, b = out["diagonal (reference Jacobi)"], out["block Jacobi (per loop)"]
    out["iteration_ratio_diagonal_over_block"] = d["pcg_iterations_per_tick"] / max(b["pcg_iterations_per_tick"], 1e-9)
    if "learned pair blocks" in out:
        out["iteration_ratio_pair_over_learned"] = (out["pair blocks"]["pcg_iterations_per_tick"] /
                                                    max(out["learned pair blocks"]["pcg_iterations_per_tick"], 1e-9))
    return out


def measure_full_forms(local: int, ticks: int = 6) -> dict:
    """The full form at scale, ticks 1..`ticks` from the generated state.

    Closures: the 1,250,000-body scene (the 100,000-body mix on a 100^3 lattice and 50,000
    five-body chains, 10% loop-closed) with the reference's 12 x 8 closure rounds, and with
    closure PCG to 1e-5 under per-loop block Jacobi and under the network-corrected blocks.  Its
    chains have dynamic roots, so its contact solve keeps the reference's interleaved fixed
    passes (device.rs:1108-1155), which the residual mode does not iterate.
    Contacts: the 1,000,000-body lattice alone, 8 fixed passes against passes until 1e-5 with the
    cached and with the learned warm start (cap 512)."""
    import torch
    from mechanic_b200 import abi, learned, scenes
    from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig
    warm = np.load(os.path.join(ROOT, "mechanic_b200", "data", "warm_start.npy"))
    xs, ts, _ = learned.collect_closure_samples(scenes.bearing_chains(4000), 8, learned.closure_config(
        preconditioner=abi.PRECOND_PAIR_BLOCKS, device=local))
    precond, _ = learned.train_preconditioner(xs, ts, steps=2000)
    caps = {"pair_capacity": 1 << 28}
    full = scenes.config_full()
    lattice = scenes.stack_grid(100, 100, 100, seed=0)
    forms = [
        ("full: reference passes", full, GpuPhysicsConfig(device=local)),
        ("full: closure PCG to 1e-5, block Jacobi", full,
         GpuPhysicsConfig(device=local, closure_mode=abi.CLOSURE_PCG_RESIDUAL, closure_tolerance=1e-5)),
        ("full: closure PCG to 1e-5, learned blocks", full,
         GpuPhysicsConfig(device=local, closure_mode=abi.CLOSURE_PCG_RESIDUAL, closure_tolerance=1e-5,
                          preconditioner=abi.PRECOND_LEARNED)),
        ("lattice: 8 contact passes", lattice, GpuPhysicsConfig(device=local)),
        ("lattice: contacts to 1e-5, cached start", lattice,
         GpuPhysicsConfig(device=local, contact_tolerance=1e-5, contact_max_iterations=512)),
        ("lattice: contacts to 1e-5, learned start", lattice,
         GpuPhysicsConfig(device=local, contact_tolerance=1e-5, contact_max_iterations=512,
                          warm_start=abi.WARM_LEARNED)),
    ]
    out = {"workload": f"full: 1,250,000 bodies ({full.collider_count} colliders); lattice: 1,000,000 bodies "
                       f"({lattice.collider_count} colliders); ticks 1..{ticks} from the generated state"}
    for name, scene, cfg in forms:
        with GpuPhysics(scene, cfg, capacities=caps) as g:
            if cfg.warm_start == abi.WARM_LEARNED:
                g.set_warm_start_network(warm)
            if cfg.preconditioner == abi.PRECOND_LEARNED:
                g.set_preconditioner_network(precond)
            rows = []
            for t in range(1, ticks + 1):
                g.dispatch_tick(t)
                rb = g.read_last_tick()
                rows.append({"tick": t, "ms": round(rb.gpu_tick_ms, 3), "contacts": rb.contact_count,
                             "active": rb.active_contact_count, "contact_passes": rb.contact_iterations,
                             "contact_rel_residual": rb.contact_relative_residual,
                             "closure_pcg_iterations": rb.closure_iterations,
                             "closure_rel_residual": rb.closure_relative_residual, "flags": rb.error_flags,
                             "warm_start_used": rb.warm_start_used})
            ms = sum(r["ms"] for r in rows)
            out[name] = {"ticks": rows, "ms_per_tick": ms / ticks,
                         "body_steps_per_s": scene.body_count * ticks / (ms / 1e3)}
        torch.cuda.synchronize()
    return out


def measure_batched(args, rank: int, world: int, local: int):
    """The 256-scene batched config (sharded by scene across ranks)."""
    import torch
    from mechanic_b200 import abi, scenes, sharding
    from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig
    lst = scenes.batched_uneven(256, seed=args.seed)
    counts = [s.body_count for s in lst]
    mine = [lst[i] for i in sharding.partition(counts, world)[rank]]
    nb = sum(s.body_count for s in mine)
    nc = sum(s.collider_count for s in mine)
    cfg = GpuPhysicsConfig(device=local, closure_mode=abi.CLOSURE_PCG_RESIDUAL)
    g = GpuPhysics.batch(mine, cfg, capacities={"max_bodies": nb, "max_colliders": nc, "max_bearings": 1 << 20,
                                                 "pair_capacity": 1 << 26})
    st = g.state_buffers()
    stream = torch.cuda.ExternalStream(st.stream, device=torch.device("cuda", local))
    for t in range(1, args.warmup + 1):
        g.dispatch_tick(t)
    g.wait()
    tuning = g.autotune(ticks=2)[0] if not args.no_autotune else g.tuning()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    flags = 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            starts[k].record(stream)
            g.dispatch_tick(args.warmup + k + 1)
            ends[k].record(stream)
            flags |= g.read_last_tick().error_flags
    torch.cuda.synchronize()
    ms = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    ms = sharding.max_over_ranks(ms, device=torch.device("cuda", local)) if world > 1 else ms
    launches = g.tick_kernel_count() * args.steps
    g.close()
    return {"workload": "256 scenes, body counts log-uniform in [64, 8192], 2% bearings, one handle per rank, "
                        f"ticks {args.warmup + 1}..{args.warmup + args.steps}, closure PCG per-loop blocks",
            "bodies": int(sum(counts)), "scenes": 256, "value": sum(counts) * args.steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / args.steps, "scaling": "strong (scenes sharded)" if world > 1 else "single",
            "gpu_launches": launches, "error_flags_seen": flags, "launch_shapes": tuning}


# ------------------------------------------------------------------ ours
def main():
    args = parse()
    rank, world, local = dist_env()
    from mechanic_b200 import scenes
    if args.cpu_table:
        if rank == 0:
            print(json.dumps(cpu_table()), flush=True)
        return
    if args.full_form:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(measure_full_forms(local)), flush=True)
        return
    if args.long_loops:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(measure_closure_forms(local, chains=400, links=16, closure_fraction=1.0)), flush=True)
        return
    scene = scenes.stack_grid(50, 40, 50, seed=args.seed)

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, scene)), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    from mechanic_b200 import abi
    from mechanic_b200.physics import GpuPhysics, GpuPhysicsConfig

    gpu = GpuPhysics(scene, GpuPhysicsConfig(device=local), capacities={"pair_capacity": PAIR_CAPACITY})
    initial = {"transforms": scene.transforms.copy(), "velocities": scene.velocities.copy()}
    st = gpu.state_buffers()
    stream = torch.cuda.ExternalStream(st.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}") if args.flush_l2 else None

    def reset():
        gpu.load_state(initial["transforms"], initial["velocities"], manifold=np.zeros(0, abi.CONTACT),
                       manifold_tick=0)

    # warm-up from the initial state; from the state it leaves, the autotuner times
    # the next 8 ticks per candidate launch shape (restoring the state before each;
    # light ticks are most of the timed trajectory) and keeps the fastest; then the
    # initial state is reloaded
    for tick in range(1, args.warmup + 1):
        gpu.dispatch_tick(tick)
    gpu.wait()
    tuning, tuned_ms = gpu.autotune(ticks=8) if not args.no_autotune else (gpu.tuning(), None)
    reset()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stage_ms = {"broadphase": 0.0, "narrowphase": 0.0, "contact_solver": 0.0, "integration": 0.0}
    solve_bytes = 0.0
    broad_bytes = 0.0
    counts = []
    flags = 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                if flush is not None:
                    flush.zero_()
                starts[k].record(stream)
                gpu.dispatch_tick(k + 1)
                ends[k].record(stream)
                rb = gpu.read_last_tick()   # stage events of this tick (synchronizes)
                flags |= rb.error_flags
                kt = rb.kernel_timings
                stage_ms["integration"] += kt.integration_ms
                stage_ms["broadphase"] += kt.broadphase_ms
                stage_ms["narrowphase"] += kt.narrowphase_ms
                stage_ms["contact_solver"] += kt.contact_solver_ms
                counts.append((rb.pair_count, rb.contact_count, rb.active_contact_count))
                broad_bytes += (bytes_broadphase_per_collider(tuning["morton_mode"]) * scene.collider_count
                                + BYTES_BROADPHASE_PER_PAIR * rb.pair_count)
                # the apply touches at most the active contacts' bodies (2 per contact): light
                # ticks apply only those, so counting every body would overstate the traffic
                applied = min(scene.body_count, 2 * rb.active_contact_count)
                solve_bytes += (8 * (BYTES_SOLVE_PER_CONTACT_ITER * rb.active_contact_count
                                     + BYTES_APPLY_PER_BODY_ITER * applied)
                                + BYTES_PREPARE_PER_CONTACT * rb.contact_count)
        torch.cuda.synchronize()
    per_tick = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(per_tick))
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * scene.body_count * args.steps / (total_ms / 1e3)

    # ---- end to end through the C ABI with host buffers
    reset()
    pinned = torch.empty(scene.body_count * abi.TRANSFORM.itemsize, dtype=torch.uint8, pin_memory=True)
    rows = np.frombuffer(pinned.numpy().data, dtype=abi.TRANSFORM, count=scene.body_count)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # the snapshot ring's use: tick k's slot is copied to the host while tick k + 1
    # runs (the read waits for tick k and its copy only); every tick's slot is read
    prev = None
    for k in range(args.steps):
        sub = gpu.dispatch_tick(k + 1)             # H2D: the 64-byte tick row
        if prev is not None:
            gpu.read_snapshot_transforms(prev.snapshot_slot, rows)   # D2H: tick k's snapshot slot
        prev = sub
    gpu.read_snapshot_transforms(prev.snapshot_slot, rows)
    e2e_flags = gpu.read_last_tick().error_flags   # D2H: 32-byte diagnostics of the last tick
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * scene.body_count * args.steps / e2e_s

    kernels_per_tick = gpu.tick_kernel_count()
    gpu_launches = kernels_per_tick * args.steps
    forms = None
    if not args.no_forms:
        forms = {"batched": measure_batched(args, rank, world, local)}
        if rank == 0 and world == 1:
            forms["residual_1e-5"] = measure_residual_forms(local)
            forms["closure_1e-5"] = measure_closure_forms(local)
    solve_ms = stage_ms["contact_solver"]
    broad_ms = stage_ms["broadphase"]
    peaks = {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
    peak = peaks.get("hbm_gbs")
    peak_note = "measured" if peak else "fallback"
    peak = peak or 6650.0
    solve_gbs = solve_bytes / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    broad_gbs = broad_bytes / (broad_ms / 1e3) / 1e9 if broad_ms > 0 else 0.0
    stages = {
        "broadphase": {"kernel": "broadphase stage (bounds + Morton, onesweep sort, Karras, refit, traversal, "
                                 "pair-key sort)", "achieved": broad_gbs, "ms": broad_ms,
                       "bytes_per_step": broad_bytes / args.steps},
        "contact_solve": {"kernel": "contact solve stage (k_prepare + k_solve_all: 8 x (solve + apply))",
                          "achieved": solve_gbs, "ms": solve_ms, "bytes_per_step": solve_bytes / args.steps},
    }
    dominant = max(stages, key=lambda k: stages[k]["ms"])
    other = "contact_solve" if dominant == "broadphase" else "broadphase"

    if rank == 0:
        cpu = None
        parity = None
        if not args.no_cpu_baseline and world == 1:
            done, elapsed, used, oworld = cpu_trajectory(scene, args.steps, 30.0, os.cpu_count() or 1,
                                                         keep_world=True)
            cpu = {"value": scene.body_count * done / elapsed, "unit": UNIT, "cores": used, "kind": "port",
                   "sample": f"ticks 1..{done} of the same trajectory on the CPU restatement (FP32), {used} threads, "
                             f"{elapsed:.1f} s"}
            parity = parity_against_oracle(gpu, scene, reset, done, oworld)
            del oworld
        tick1 = counts[0] if counts else (0, 0, 0)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": bench_config(scene, args, world),
            "run": {"tick1_pairs_contacts_active": list(tick1), "launch_shapes": tuning,
                    "autotune": "mk_autotune over the 8 ticks after the warm-up, state restored" if tuned_ms else "off"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 64,
                    "d2h_bytes_per_step": scene.body_count * abi.TRANSFORM.itemsize + 32 / args.steps,
                    "pipelining": "tick k's snapshot slot is read while tick k + 1 runs; diagnostics read after "
                                  "the last tick", "error_flags": e2e_flags},
            "roofline": {"bound": "hbm", "kernel": stages[dominant]["kernel"],
                         "achieved": stages[dominant]["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": stages[dominant]["achieved"] / peak, "peak_source": peak_note, "traffic": None,
                         "traffic_note": "the line is a stage of several kernels; per-kernel ncu DRAM bytes are in "
                                         "profiles/ (k_solve_all heavy tick: 142 B per contact and pass, against "
                                         f"{BYTES_SOLVE_PER_CONTACT_ITER} algorithmic: the body rows hit L2)",
                         "algorithmic_bytes_per_step": stages[dominant]["bytes_per_step"],
                         "secondary": {"kernel": stages[other]["kernel"], "achieved": stages[other]["achieved"],
                                       "frac": stages[other]["achieved"] / peak,
                                       "algorithmic_bytes_per_step": stages[other]["bytes_per_step"]},
                         "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()}},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks.summary(),
            "gpu_launches": gpu_launches,
            "error_flags": flags,
            "forms": forms,
        }
        print(json.dumps(out), flush=True)
    gpu.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
