"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the CPU legs of bench.py may
import this package.  It is the checker of the CUDA library, never a
fallback for it.  See oracle.h for what it restates and how it is pinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mechanic_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
SOURCES = [os.path.join(HERE, "oracle.cpp"), os.path.join(HERE, "oracle.h")]


def build(force: bool = False) -> str:
    """Compile the restatement: FP32 parity needs -ffp-contract=off (one IEEE
    operation per source operation, like the CUDA build's --fmad=false)."""
    newest = max(os.path.getmtime(s) for s in SOURCES)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-fPIC", "-shared", "-Wall", "-Wno-unused-function", SOURCES[0], "-o", LIB_PATH + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build()
        L = C.CDLL(path)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.or_create.restype = vp
        L.or_create.argtypes = [vp, vp, C.c_int, u32]
        L.or_destroy.argtypes = [vp]
        L.or_step.argtypes = [vp, u64]
        L.or_count.restype = u64
        L.or_count.argtypes = [vp, C.c_int]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        for name in ("or_get_state", "or_set_state"):
            getattr(L, name).argtypes = [vp, vp, vp]
        L.or_get_state_f64.argtypes = [vp, vp, vp, vp, vp]
        for name in ("or_get_diagnostics", "or_get_pairs", "or_get_contacts", "or_get_contacts_f64",
                     "or_get_contact_keys", "or_get_features", "or_get_active",
                     "or_get_collider_keys", "or_get_aabbs", "or_get_world_masses",
                     "or_get_coordinates", "or_set_coordinates", "or_get_links", "or_get_karras"):
            getattr(L, name).argtypes = [vp, vp]
        L.or_get_sorted.argtypes = [vp, vp, vp]
        L.or_get_solve_stats.argtypes = [vp, vp, vp]
        L.or_set_batch.argtypes = [vp, vp, u32]
        L.or_get_closure_stats.argtypes = [vp, vp, vp]
        L.or_set_precond_outputs.argtypes = [vp, vp, u32]
        L.or_get_closure_blocks.restype = u32
        L.or_get_closure_blocks.argtypes = [vp, vp]
        L.or_set_warm_predictions.argtypes = [vp, vp, u32]
        L.or_get_snapshot.argtypes = [vp, u32, vp]
        L.or_get_manifold.restype = u32
        L.or_get_manifold.argtypes = [vp, vp, u32]
        L.or_set_manifold.argtypes = [vp, vp, u32, u64]
        L.or_obb_sat_f32.restype = u32
        L.or_obb_sat_f32.argtypes = [vp, vp, vp]
        L.or_contact_point_f32.argtypes = [vp, vp, vp, vp]
        L.or_cpu_obb_sat.restype = C.c_int
        L.or_cpu_obb_sat.argtypes = [vp] * 7
        L.or_cpu_contact_manifold.restype = C.c_int
        L.or_cpu_contact_manifold.argtypes = [vp] * 8
        L.or_morton30.restype = u32
        L.or_morton30.argtypes = [C.c_float] * 3
        L.or_morton63.restype = u64
        L.or_morton63.argtypes = [C.c_float] * 7
        L.or_morton48.restype = u64
        L.or_morton48.argtypes = [C.c_float] * 7
        L.or_morton39.restype = u64
        L.or_morton39.argtypes = [C.c_float] * 7
        L.or_morton30a.restype = u64
        L.or_morton30a.argtypes = [C.c_float] * 7
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def threads() -> int:
    return int(lib().or_get_threads())


def _p(a):
    return None if a is None else a.ctypes.data


class OracleWorld:
    """One scene stepped by the CPU restatement (precision 32 or 64)."""

    def __init__(self, scene, config: abi.MkConfig | None = None, precision: int = 32,
                 pair_capacity: int = 0):
        self.scene = scene
        self._creation = scene.creation()
        self._config = config
        self.precision = precision
        self.B, self.C = scene.body_count, scene.collider_count
        self.h = lib().or_create(C.byref(self._creation),
                                 C.byref(config) if config is not None else None,
                                 precision, pair_capacity)
        if not self.h:
            raise RuntimeError("oracle creation failed")

    @classmethod
    def batch(cls, scene_list, config: abi.MkConfig | None = None, precision: int = 32, pair_capacity: int = 0):
        """Several independent scenes as one world (the concatenation mk_create_batch makes)."""
        from mechanic_b200 import scenes as _scenes
        combined, collider_scene = _scenes.concatenate(scene_list)
        w = cls(combined, config, precision, pair_capacity)
        w._collider_scene = np.ascontiguousarray(collider_scene, np.uint32)
        if len(scene_list) > 1:
            lib().or_set_batch(w.h, _p(w._collider_scene), len(scene_list))
        return w

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().or_destroy(h)
            self.h = None

    def step(self, tick: int) -> None:
        lib().or_step(self.h, tick)

    def count(self, what: int) -> int:
        return int(lib().or_count(self.h, what))

    @property
    def pair_count(self):
        return self.count(0)

    @property
    def contact_count(self):
        return self.count(1)

    @property
    def active_count(self):
        return self.count(2)

    def state(self):
        tr = np.zeros(self.B, abi.TRANSFORM)
        vel = np.zeros(self.B, abi.VELOCITY)
        lib().or_get_state(self.h, _p(tr), _p(vel))
        return tr, vel

    def state_f64(self):
        arrs = [np.zeros((self.B, 4)) for _ in range(4)]
        lib().or_get_state_f64(self.h, *[_p(a) for a in arrs])
        return arrs

    def set_state(self, transforms, velocities):
        lib().or_set_state(self.h, _p(transforms), _p(velocities))

    def diagnostics(self):
        d = np.zeros(1, abi.DIAGNOSTICS)
        lib().or_get_diagnostics(self.h, _p(d))
        return d[0]

    def solve_stats(self) -> dict:
        """Outcome of the last residual-mode contact solve."""
        u = np.zeros(3, np.uint32)
        d = np.zeros(2, np.float64)
        lib().or_get_solve_stats(self.h, _p(u), _p(d))
        return {"iterations": int(u[0]), "chosen": int(u[1]), "converged": int(u[2]),
                "s0": float(d[0]), "sk": float(d[1]),
                "relative_residual": float(np.sqrt(d[1] / d[0])) if d[0] > 0 else 0.0}

    def closure_stats(self) -> dict:
        """Closure solve outcome of the last step (MK_CLOSURE_PCG_RESIDUAL)."""
        u = np.zeros(4, np.uint32)
        d = np.zeros(1, np.float64)
        lib().or_get_closure_stats(self.h, _p(u), _p(d))
        return {"newton_steps": int(u[0]), "pcg_iterations": int(u[1]), "learned_blocks": int(u[2]),
                "rejected_blocks": int(u[3]), "max_relative_residual": float(d[0])}

    def set_precond_outputs(self, out) -> None:
        """Preconditioner network outputs (12 x blocks x 3) for the next step."""
        out = np.ascontiguousarray(out, np.float32).ravel()
        lib().or_set_precond_outputs(self.h, _p(out), len(out))

    def closure_blocks(self):
        n = int(lib().or_get_closure_blocks(self.h, None))
        out = np.zeros((n, 16), np.float32)
        if n:
            lib().or_get_closure_blocks(self.h, _p(out))
        return out

    def set_warm_predictions(self, pred) -> None:
        """Learned warm-start impulses, by active position, for the next step's solve."""
        pred = np.ascontiguousarray(pred, np.float32)
        lib().or_set_warm_predictions(self.h, _p(pred), len(pred))

    def pairs(self):
        out = np.zeros(self.pair_count, abi.PAIR)
        lib().or_get_pairs(self.h, _p(out))
        return out

    def contacts(self):
        out = np.zeros(self.contact_count, abi.CONTACT)
        lib().or_get_contacts(self.h, _p(out))
        return out

    def contacts_f64(self):
        out = np.zeros((self.contact_count, 16))
        lib().or_get_contacts_f64(self.h, _p(out))
        return out

    def contact_keys(self):
        out = np.zeros(self.contact_count, np.uint64)
        lib().or_get_contact_keys(self.h, _p(out))
        return out

    def features(self):
        out = np.zeros(self.contact_count, np.uint32)
        lib().or_get_features(self.h, _p(out))
        return out

    def active(self):
        out = np.zeros(self.active_count, np.uint32)
        lib().or_get_active(self.h, _p(out))
        return out

    def collider_keys(self):
        out = np.zeros(self.C, np.uint64)
        lib().or_get_collider_keys(self.h, _p(out))
        return out

    def sorted_entries(self):
        k = np.zeros(self.C, np.uint64)
        v = np.zeros(self.C, np.uint32)
        lib().or_get_sorted(self.h, _p(k), _p(v))
        return k, v

    def aabbs(self):
        out = np.zeros((self.C, 8), np.float32)
        lib().or_get_aabbs(self.h, _p(out))
        return out

    def world_masses(self):
        out = np.zeros((self.B, 12), np.float32)
        lib().or_get_world_masses(self.h, _p(out))
        return out

    def karras(self):
        out = np.zeros((max(self.C - 1, 0), 2), np.uint32)
        if self.C > 1:
            lib().or_get_karras(self.h, _p(out))
        return out

    def snapshot(self, slot: int):
        out = np.zeros(self.B, abi.TRANSFORM)
        lib().or_get_snapshot(self.h, slot, _p(out))
        return out

    def coordinates(self):
        out = np.zeros(self.count(6), abi.MECHANISM_COORDINATE)
        lib().or_get_coordinates(self.h, _p(out))
        return out

    def set_coordinates(self, coords):
        lib().or_set_coordinates(self.h, _p(np.ascontiguousarray(coords)))

    def links(self):
        out = np.zeros(self.B, abi.LINK_STATE)
        lib().or_get_links(self.h, _p(out))
        return out

    def manifold(self):
        n = self.count(5)
        out = np.zeros(n, abi.CONTACT)
        got = lib().or_get_manifold(self.h, _p(out), n)
        return out[:got]

    def set_manifold(self, rows, last_tick: int):
        rows = np.ascontiguousarray(rows)
        lib().or_set_manifold(self.h, _p(rows), len(rows), last_tick)


def obb_sat(box_a: np.ndarray, box_b: np.ndarray):
    np_out = np.zeros(4, np.float32)
    a = np.ascontiguousarray(box_a, np.float32)
    b = np.ascontiguousarray(box_b, np.float32)
    feat = lib().or_obb_sat_f32(_p(a), _p(b), _p(np_out))
    return np_out, int(feat)


def cpu_obb_sat(ca, qa, ha, cb, qb, hb):
    arrs = [np.ascontiguousarray(x, np.float32) for x in (ca, qa, ha, cb, qb, hb)]
    out = np.zeros(4, np.float32)
    ok = lib().or_cpu_obb_sat(*[_p(a) for a in arrs], _p(out))
    return (out[:3], float(out[3])) if ok else None


def cpu_contact_manifold(ca, qa, ha, cb, qb, hb):
    arrs = [np.ascontiguousarray(x, np.float32) for x in (ca, qa, ha, cb, qb, hb)]
    out = np.zeros(4, np.float32)
    pts = np.zeros((4, 3), np.float32)
    n = lib().or_cpu_contact_manifold(*[_p(a) for a in arrs], _p(out), _p(pts))
    if n == 0:
        return None
    return out[:3], float(out[3]), pts[:n]


def morton30(x, y, z) -> int:
    return int(lib().or_morton30(x, y, z))


def morton63(x, y, z, lo=(0.0, 0.0, 0.0), scale=1.0) -> int:
    """63-bit key of a centre in the frame (lo, scale) of the tick's centre bounds."""
    return int(lib().or_morton63(x, y, z, lo[0], lo[1], lo[2], scale))


def morton30a(x, y, z, lo=(0.0, 0.0, 0.0), scale=1.0) -> int:
    """10 bits per axis over the tick's centre bounds (lo, scale = 1023 / largest extent)."""
    return int(lib().or_morton30a(x, y, z, lo[0], lo[1], lo[2], scale))


def morton39(x, y, z, lo=(0.0, 0.0, 0.0), scale=1.0) -> int:
    """13 bits per axis over the tick's centre bounds (lo, scale = 8191 / largest extent)."""
    return int(lib().or_morton39(x, y, z, lo[0], lo[1], lo[2], scale))


def morton48(x, y, z, lo=(0.0, 0.0, 0.0), scale=1.0) -> int:
    """48-bit key (16 bits per axis) of a centre in the frame (lo, scale)."""
    return int(lib().or_morton48(x, y, z, lo[0], lo[1], lo[2], scale))
