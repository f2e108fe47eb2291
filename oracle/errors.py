"""Error of FP32 results against the FP64 restatement (TEST INFRASTRUCTURE ONLY).

The FP64 oracle (``OracleWorld(precision=64)``) runs the same algorithm as
the FP32 one -- the reference's kernels in their operation order, including
the i32 fixed-point velocity deltas of collision.wgsl:752-906 -- with every
float in double.  Stepping it once from the state an FP32 result started
from and comparing the two says how far the FP32 arithmetic of one tick
lands from the exact-arithmetic answer of the same algorithm.

Contacts are matched by (collider a, collider b, row within the pair) -- the
contact rows themselves carry bodies and a manifold slot, so the collider
keys come beside them; a
contact that exists in one result only (an SAT or activity decision that
flips between the precisions) is counted, not compared.  For every compared
quantity the table gives the largest absolute difference, its 99th
percentile, and the normwise relative error max|d| / max|x64|.
"""
from __future__ import annotations

import numpy as np

INVALID = 0xFFFFFFFF


def _stats(f32: np.ndarray, f64: np.ndarray) -> dict:
    d = np.abs(np.asarray(f32, np.float64) - np.asarray(f64, np.float64))
    if d.size == 0:
        return {"max_abs": 0.0, "p99_abs": 0.0, "rel_inf": 0.0, "n": 0}
    scale = float(np.max(np.abs(f64)))
    return {"max_abs": float(d.max()), "p99_abs": float(np.percentile(d, 99)),
            "rel_inf": float(d.max() / scale) if scale > 0 else float(d.max()), "n": int(d.size)}


def _ranked(pair: np.ndarray) -> np.ndarray:
    """(collider pair key, row rank inside its pair) as one structured key, so a clipped
    manifold's several rows per pair match one to one."""
    order = np.argsort(pair, kind="stable")
    rank = np.zeros(len(pair), np.uint64)
    if len(pair):
        sp = pair[order]
        start = np.r_[True, sp[1:] != sp[:-1]]
        run_start = np.maximum.accumulate(np.where(start, np.arange(len(sp)), 0))
        rank[order] = (np.arange(len(sp)) - run_start).astype(np.uint64)
    out = np.zeros(len(pair), np.dtype([("p", np.uint64), ("r", np.uint64)]))
    out["p"], out["r"] = pair, rank
    return out


def contact_errors(rows32: np.ndarray, keys32: np.ndarray, rows64: np.ndarray, keys64: np.ndarray) -> dict:
    """rows32: GpuContact rows (abi.CONTACT) with their collider-pair keys; rows64: (K, 16)
    doubles from contacts_f64() with the FP64 world's contact_keys()."""
    a = _ranked(np.asarray(keys32, np.uint64))
    b = _ranked(np.asarray(keys64, np.uint64))
    common, ia, ib = np.intersect1d(a, b, assume_unique=True, return_indices=True)
    x = rows32[ia]
    y = rows64[ib]
    np32, aa32, ab32 = x["normal_penetration"], x["arm_a_impulse"], x["arm_b"]
    np64, aa64, ab64 = y[:, 4:8], y[:, 8:12], y[:, 12:16]
    return {
        "counts": {"fp32": int(len(rows32)), "fp64": int(len(rows64)), "matched": int(len(common))},
        "point_arm_a_m": _stats(aa32[:, :3], aa64[:, :3]),
        "point_arm_b_m": _stats(ab32[:, :3], ab64[:, :3]),
        "normal": _stats(np32[:, :3], np64[:, :3]),
        "depth_m": _stats(np32[:, 3], np64[:, 3]),
        "impulse": _stats(aa32[:, 3], aa64[:, 3]),
    }


def state_errors(transforms32: np.ndarray, velocities32: np.ndarray, state64) -> dict:
    """FP32 body state (abi.TRANSFORM / abi.VELOCITY rows) against state_f64() arrays."""
    p64, r64, l64, a64 = state64
    return {
        "position_m": _stats(transforms32["position"][:, :3], p64[:, :3]),
        "rotation": _stats(transforms32["rotation"], r64),
        "linear_velocity_mps": _stats(velocities32["linear"][:, :3], l64[:, :3]),
        "angular_velocity_rps": _stats(velocities32["angular"][:, :3], a64[:, :3]),
    }


def one_step_errors(scene, config, start: dict, tick: int, fp32_result: dict, pair_capacity: int = 0) -> dict:
    """Steps the FP64 oracle once from `start` (transforms, velocities, manifold rows,
    manifold tick, coordinates) at `tick`, and compares `fp32_result` (transforms,
    velocities, contacts and contact_keys after the same step) with it."""
    import oracle
    w = oracle.OracleWorld(scene, config, precision=64, pair_capacity=pair_capacity)
    w.set_state(np.ascontiguousarray(start["transforms"]), np.ascontiguousarray(start["velocities"]))
    if start.get("coordinates") is not None and len(start["coordinates"]):
        w.set_coordinates(start["coordinates"])
    if start.get("manifold") is not None and len(start["manifold"]):
        w.set_manifold(start["manifold"], start["manifold_tick"])
    w.step(tick)
    out = {"tick": tick, "bodies": scene.body_count}
    out.update(state_errors(fp32_result["transforms"], fp32_result["velocities"], w.state_f64()))
    out.update(contact_errors(fp32_result["contacts"], fp32_result["contact_keys"], w.contacts_f64(),
                              w.contact_keys()))
    return out


def summary_line(table: dict) -> str:
    keys = ("position_m", "rotation", "linear_velocity_mps", "angular_velocity_rps", "point_arm_a_m",
            "depth_m", "normal", "impulse")
    parts = [f"{k}: max {table[k]['max_abs']:.3g} (rel {table[k]['rel_inf']:.3g})" for k in keys if k in table]
    c = table.get("counts", {})
    return f"tick {table.get('tick')}: contacts fp32 {c.get('fp32')} fp64 {c.get('fp64')} matched " \
           f"{c.get('matched')}; " + "; ".join(parts)
