"""Host mirror of mechanic-gpu's ``GpuPhysics`` over the C ABI.

Method names, argument meaning and error behaviour follow
crates/mechanic-gpu/src/device.rs:369-1663; the wgpu ``device``/``queue``
parameters disappear because the handle owns its CUDA stream.  Every call
goes through libmechanic_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmechanic_b200.so")

EXPORTS = [
    "mk_config_default", "mk_create", "mk_destroy", "mk_dispatch_tick", "mk_wait",
    "mk_read_last_tick", "mk_read_snapshot", "mk_snapshot_buffers", "mk_apply_impulse",
    "mk_write_drives", "mk_init_coordinates", "mk_body_count", "mk_has_gpu_timestamps",
    "mk_state_buffers", "mk_save_state", "mk_load_state", "mk_read_buffer", "mk_version",
    "mk_last_error", "mk_op_sort_scratch_bytes", "mk_op_sort_keys", "mk_op_obb_sat",
    "mk_tick_kernel_count", "mk_set_tuning", "mk_op_sort_keys_static",
    "mk_mlp_param_count", "mk_op_mlp_scratch_bytes", "mk_op_mlp_forward", "mk_op_mlp_gradient",
    "mk_op_mlp_train", "mk_set_warm_start_network", "mk_read_warm_start_samples",
    "mk_set_preconditioner_network", "mk_create_batch", "mk_scene_offsets", "mk_get_handle_tuning",
    "mk_set_handle_tuning", "mk_autotune", "mk_selftest_bounded_wait", "mk_published_state",
    "mk_interpolate_snapshot",
]

_lib = None


def library(path: str | None = None):
    """Loads libmechanic_b200.so.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; build it with `python -m mechanic_b200.build`")
    L = C.CDLL(path)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    sig = {
        "mk_config_default": (None, [vp]),
        "mk_create": (i32, [vp, vp, vp, vp, vp]),
        "mk_destroy": (None, [vp]),
        "mk_dispatch_tick": (i32, [vp, u64, vp]),
        "mk_wait": (i32, [vp, u64]),
        "mk_read_last_tick": (i32, [vp, vp]),
        "mk_read_snapshot": (i32, [vp, C.c_uint8, vp, u32, vp]),
        "mk_snapshot_buffers": (i32, [vp, C.c_uint8, vp, vp, vp]),
        "mk_apply_impulse": (i32, [vp, u32, vp, vp, vp]),
        "mk_write_drives": (i32, [vp, vp, u32, vp]),
        "mk_init_coordinates": (i32, [vp, vp, u32, vp]),
        "mk_body_count": (u32, [vp]),
        "mk_has_gpu_timestamps": (i32, [vp]),
        "mk_state_buffers": (i32, [vp, vp]),
        "mk_save_state": (i32, [vp, vp, vp]),
        "mk_load_state": (i32, [vp, vp, vp]),
        "mk_read_buffer": (i32, [vp, u32, vp, u64, vp, vp]),
        "mk_version": (C.c_char_p, []),
        "mk_last_error": (C.c_char_p, []),
        "mk_op_sort_scratch_bytes": (u64, [u32]),
        "mk_op_sort_keys": (i32, [vp, vp, vp, vp, u32, u32, vp, u64, vp]),
        "mk_op_obb_sat": (i32, [vp, vp, u32, vp, vp, vp]),
        "mk_tick_kernel_count": (u32, [vp]),
        "mk_set_tuning": (i32, [u32, u32]),
        "mk_op_sort_keys_static": (i32, [vp, vp, vp, vp, u32, u32, vp]),
        "mk_mlp_param_count": (u32, []),
        "mk_op_mlp_scratch_bytes": (u64, [u32]),
        "mk_op_mlp_forward": (i32, [vp, vp, u32, vp, u32, vp, u64, vp, vp]),
        "mk_op_mlp_gradient": (i32, [vp, vp, vp, vp, u32, vp, vp, u64, vp, vp]),
        "mk_op_mlp_train": (i32, [vp, vp, vp, vp, vp, vp, u32, u32, u32, C.c_float, u32, vp, vp, u64, vp, vp]),
        "mk_set_warm_start_network": (i32, [vp, vp, u32, vp]),
        "mk_read_warm_start_samples": (i32, [vp, vp, vp, u32, vp, vp]),
        "mk_set_preconditioner_network": (i32, [vp, vp, u32, vp]),
        "mk_create_batch": (i32, [vp, u32, vp, vp, vp, vp]),
        "mk_scene_offsets": (i32, [vp, vp, vp, u32]),
        "mk_get_handle_tuning": (i32, [vp, vp]),
        "mk_set_handle_tuning": (i32, [vp, vp, vp]),
        "mk_autotune": (i32, [vp, u32, vp, vp, vp]),
        "mk_selftest_bounded_wait": (i32, [u32, u32, vp, vp]),
        "mk_published_state": (i32, [vp, vp]),
        "mk_interpolate_snapshot": (i32, [vp, C.c_float, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


# ------------------------------------------------------------------ errors
class GpuPhysicsError(Exception):
    """GpuPhysicsError (device.rs:131-174) and the other ABI error variants."""

    def __init__(self, err: abi.MkError):
        self.code = int(err.code)
        self.required = int(err.required)
        self.capacity = int(err.capacity)
        self.provided = int(err.provided)
        self.body_index = int(err.body_index)
        self.body_count = int(err.body_count)
        self.slot = int(err.slot)
        super().__init__(err.message.decode(errors="replace"))


class BodyCapacity(GpuPhysicsError): pass          # noqa: E701
class BearingCapacity(GpuPhysicsError): pass       # noqa: E701
class ColliderCapacity(GpuPhysicsError): pass      # noqa: E701
class DriveStateCount(GpuPhysicsError): pass       # noqa: E701
class CoordinateStateCount(GpuPhysicsError): pass  # noqa: E701
class BodyIndexOutOfRange(GpuPhysicsError): pass   # noqa: E701  GpuImpulseError
class NonFinite(GpuPhysicsError): pass             # noqa: E701  GpuImpulseError
class InvalidSnapshotSlot(GpuPhysicsError): pass   # noqa: E701  GpuReadbackError
class DeviceFailure(GpuPhysicsError): pass         # noqa: E701  FailureStatus::DeviceFailure
class InvalidArgument(GpuPhysicsError): pass       # noqa: E701
class PairCapacity(GpuPhysicsError): pass          # noqa: E701

_ERRORS = {
    abi.MK_ERR_BODY_CAPACITY: BodyCapacity, abi.MK_ERR_BEARING_CAPACITY: BearingCapacity,
    abi.MK_ERR_COLLIDER_CAPACITY: ColliderCapacity, abi.MK_ERR_DRIVE_STATE_COUNT: DriveStateCount,
    abi.MK_ERR_COORDINATE_STATE_COUNT: CoordinateStateCount,
    abi.MK_ERR_BODY_INDEX_OUT_OF_RANGE: BodyIndexOutOfRange, abi.MK_ERR_NON_FINITE: NonFinite,
    abi.MK_ERR_INVALID_SNAPSHOT_SLOT: InvalidSnapshotSlot, abi.MK_ERR_DEVICE_FAILURE: DeviceFailure,
    abi.MK_ERR_INVALID_ARGUMENT: InvalidArgument, abi.MK_ERR_PAIR_CAPACITY: PairCapacity,
}


def _raise(rc: int, err: abi.MkError | None = None):
    if rc == abi.MK_OK:
        return
    if err is None or err.code == 0:
        err = abi.MkError()
        err.code = rc
        err.message = (library().mk_last_error() or b"")[:255]
    raise _ERRORS.get(rc, GpuPhysicsError)(err)


# ----------------------------------------------------------------- config
@dataclasses.dataclass
class GpuPhysicsConfig:
    """GpuPhysicsConfig (device.rs:22-41) plus the B200 build's switches."""

    collisions_enabled: bool = True
    mechanism_self_collisions: bool = True
    solver_iterations: int = 8
    morton_mode: int = abi.MORTON_39
    closure_mode: int = abi.CLOSURE_REFERENCE
    use_graph: bool = True
    device: int = 0
    warm_start: int = abi.WARM_CACHED
    contact_tolerance: float = 0.0          # > 0: contact passes until ||r|| <= tol * ||r_cold||
    contact_max_iterations: int = 0         # 0 => 512
    closure_tolerance: float = 0.0          # 0 => 1e-5 (CLOSURE_PCG_RESIDUAL)
    closure_max_iterations: int = 0         # 0 => 256
    preconditioner: int = abi.PRECOND_BLOCK_JACOBI
    contact_manifold: int = abi.MANIFOLD_POINT

    def to_c(self) -> abi.MkConfig:
        c = abi.config_default()   # equals mk_config_default's row (checked by a CPU test)
        c.collisions_enabled = int(self.collisions_enabled)
        c.mechanism_self_collisions = int(self.mechanism_self_collisions)
        c.solver_iterations = int(self.solver_iterations)
        c.morton_mode = int(self.morton_mode)
        c.closure_mode = int(self.closure_mode)
        c.use_graph = int(self.use_graph)
        c.device = int(self.device)
        c.warm_start = int(self.warm_start)
        c.contact_tolerance = float(self.contact_tolerance)
        c.contact_max_iterations = int(self.contact_max_iterations)
        c.closure_tolerance = float(self.closure_tolerance)
        c.closure_max_iterations = int(self.closure_max_iterations)
        c.preconditioner = int(self.preconditioner)
        c.contact_manifold = int(self.contact_manifold)
        return c


@dataclasses.dataclass
class GpuTickSubmission:
    tick_index: int
    snapshot_slot: int
    submission_index: int


@dataclasses.dataclass
class GpuKernelTimings:
    integration_ms: float
    mechanism_ms: float
    broadphase_ms: float
    narrowphase_ms: float
    contact_solver_ms: float
    bearings_ms: float
    snapshot_ms: float


@dataclasses.dataclass
class GpuTickReadback:
    gpu_tick_ms: float | None
    kernel_timings: GpuKernelTimings | None
    error_flags: int
    pair_count: int
    contact_count: int
    active_contact_count: int
    anchor_residual_meters: float
    axis_residual_degrees: float
    closure_iterations: int = 0
    closure_relative_residual: float = 0.0
    contact_iterations: int = 0
    warm_start_used: int = 0
    contact_relative_residual: float = 0.0


class GpuPhysics:
    """One scene on one GPU (device.rs:199-234)."""

    def __init__(self, scene, config: GpuPhysicsConfig | None = None, capacities=None):
        L = library()
        self.scene = scene
        self._creation = scene.creation()
        self._config = (config or GpuPhysicsConfig()).to_c()
        caps = None
        if capacities is not None:
            caps = abi.MkCapacities()
            for k, v in dict(capacities).items():
                setattr(caps, k, int(v))
        self._caps = caps
        h = C.c_void_p()
        err = abi.MkError()
        rc = L.mk_create(C.byref(self._creation), C.byref(self._config),
                         C.byref(caps) if caps is not None else None, C.byref(h), C.byref(err))
        _raise(rc, err)
        self._h = h
        self._body_count = scene.body_count

    @classmethod
    def batch(cls, scene_list, config: GpuPhysicsConfig | None = None, capacities=None) -> "GpuPhysics":
        """Independent scenes stepped together by one handle (mk_create_batch)."""
        from . import scenes as _scenes
        self = cls.__new__(cls)
        L = library()
        self.scene = _scenes.concatenate(scene_list)[0]   # host-side view of the concatenated rows
        self._scene_list = list(scene_list)
        arr = (abi.MkCreation * len(scene_list))(*[s.creation() for s in scene_list])
        self._creation = arr
        self._config = (config or GpuPhysicsConfig()).to_c()
        caps = None
        if capacities is not None:
            caps = abi.MkCapacities()
            for k, v in dict(capacities).items():
                setattr(caps, k, int(v))
        self._caps = caps
        h = C.c_void_p()
        err = abi.MkError()
        rc = L.mk_create_batch(arr, len(scene_list), C.byref(self._config),
                               C.byref(caps) if caps is not None else None, C.byref(h), C.byref(err))
        _raise(rc, err)
        self._h = h
        self._body_count = self.scene.body_count
        return self

    def tuning(self) -> dict:
        t = abi.MkTuning()
        _raise(library().mk_get_handle_tuning(self._h, C.byref(t)))
        return {f: int(getattr(t, f)) for f, _ in abi.MkTuning._fields_}

    def set_tuning(self, **fields) -> None:
        t = abi.MkTuning(**self.tuning())
        for k, v in fields.items():
            setattr(t, k, int(v))
        err = abi.MkError()
        _raise(library().mk_set_handle_tuning(self._h, C.byref(t), C.byref(err)), err)

    def autotune(self, ticks: int = 5):
        """Times candidate launch shapes from the current state and applies the fastest;
        returns (tuning dict, ms per tick)."""
        t = abi.MkTuning()
        ms = C.c_double()
        err = abi.MkError()
        _raise(library().mk_autotune(self._h, int(ticks), C.byref(t), C.byref(ms), C.byref(err)), err)
        return {f: int(getattr(t, f)) for f, _ in abi.MkTuning._fields_}, float(ms.value)

    def scene_offsets(self):
        """(body offsets, collider offsets) per scene, each with the total appended."""
        n = int(library().mk_scene_offsets(self._h, None, None, 0))
        bo = np.zeros(n + 1, np.uint32)
        co = np.zeros(n + 1, np.uint32)
        library().mk_scene_offsets(self._h, bo.ctypes.data, co.ctypes.data, n + 1)
        return bo, co

    @classmethod
    def new_with_config(cls, scene, config: GpuPhysicsConfig, capacities=None) -> "GpuPhysics":
        return cls(scene, config, capacities)

    def close(self):
        if getattr(self, "_h", None):
            library().mk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- GpuPhysics methods ------------------------------------------------
    def dispatch_tick(self, tick_index: int) -> GpuTickSubmission:
        out = abi.MkSubmission()
        _raise(library().mk_dispatch_tick(self._h, int(tick_index), C.byref(out)))
        return GpuTickSubmission(int(out.tick_index), int(out.snapshot_slot), int(out.submission_index))

    def wait(self, submission_index: int = 0) -> None:
        _raise(library().mk_wait(self._h, int(submission_index)))

    def read_last_tick(self) -> GpuTickReadback:
        out = abi.MkTickReadback()
        _raise(library().mk_read_last_tick(self._h, C.byref(out)))
        t = out.kernel_timings
        timings = GpuKernelTimings(t.integration_ms, t.mechanism_ms, t.broadphase_ms, t.narrowphase_ms,
                                   t.contact_solver_ms, t.bearings_ms, t.snapshot_ms)
        return GpuTickReadback(out.gpu_tick_ms, timings, out.error_flags, out.pair_count, out.contact_count,
                               out.active_contact_count, out.anchor_residual_meters,
                               out.axis_residual_degrees, out.closure_iterations,
                               out.closure_relative_residual, out.contact_iterations,
                               out.warm_start_used, out.contact_relative_residual)

    def read_snapshot_transforms(self, slot: int, out: np.ndarray | None = None) -> np.ndarray:
        rows = out if out is not None else np.zeros(self._body_count, abi.TRANSFORM)
        err = abi.MkError()
        _raise(library().mk_read_snapshot(self._h, int(slot) & 0xFF, rows.ctypes.data, len(rows),
                                          C.byref(err)), err)
        return rows

    def snapshot(self, slot: int):
        """Device pointers (positions, rotations) of a snapshot slot, or None."""
        if not 0 <= slot < abi.SNAPSHOT_RING_SIZE:
            return None
        p, r = C.c_void_p(), C.c_void_p()
        err = abi.MkError()
        _raise(library().mk_snapshot_buffers(self._h, slot, C.byref(p), C.byref(r), C.byref(err)), err)
        return int(p.value), int(r.value)

    def published_state(self) -> abi.MkPublishedState:
        """PublishedGpuState (runtime.rs:60-75): the newest complete pair of snapshot slots."""
        out = abi.MkPublishedState()
        _raise(library().mk_published_state(self._h, C.byref(out)))
        return out

    def interpolate_snapshot(self, alpha: float, positions_out: int, rotations_out: int, stream: int = 0) -> None:
        """Render hand-off: positions and rotations a fraction `alpha` of the way from the
        published previous slot to the current one, into device buffers (float4 per body)."""
        err = abi.MkError()
        _raise(library().mk_interpolate_snapshot(self._h, float(alpha), positions_out, rotations_out,
                                                  stream or None, C.byref(err)), err)

    def apply_impulse(self, body_index: int, world_point, impulse) -> None:
        p = (C.c_float * 3)(*[float(x) for x in world_point])
        j = (C.c_float * 3)(*[float(x) for x in impulse])
        err = abi.MkError()
        _raise(library().mk_apply_impulse(self._h, int(body_index), p, j, C.byref(err)), err)

    def write_mechanism_drives(self, drives: np.ndarray) -> None:
        drives = np.ascontiguousarray(drives, abi.MECHANISM_DRIVE)
        err = abi.MkError()
        _raise(library().mk_write_drives(self._h, drives.ctypes.data if len(drives) else None, len(drives),
                                         C.byref(err)), err)

    def initialize_mechanism_coordinates(self, coordinates: np.ndarray) -> None:
        coordinates = np.ascontiguousarray(coordinates, abi.MECHANISM_COORDINATE)
        err = abi.MkError()
        _raise(library().mk_init_coordinates(self._h, coordinates.ctypes.data if len(coordinates) else None,
                                             len(coordinates), C.byref(err)), err)

    def body_count(self) -> int:
        return int(library().mk_body_count(self._h))

    def tick_kernel_count(self) -> int:
        return int(library().mk_tick_kernel_count(self._h))

    def has_gpu_timestamps(self) -> bool:
        return bool(library().mk_has_gpu_timestamps(self._h))

    # -- B200 additions --------------------------------------------------------
    def state_buffers(self) -> abi.MkDeviceState:
        out = abi.MkDeviceState()
        _raise(library().mk_state_buffers(self._h, C.byref(out)))
        return out

    def save_state(self, manifold_capacity: int | None = None):
        tr = np.zeros(self._body_count, abi.TRANSFORM)
        vel = np.zeros(self._body_count, abi.VELOCITY)
        q = int(self.scene.coordinate_count)
        coords = np.zeros(max(q, 1), abi.MECHANISM_COORDINATE)
        cap = int(manifold_capacity if manifold_capacity is not None else 1 << 22)
        man = np.zeros(cap, abi.CONTACT)
        st = abi.MkHostState(tr.ctypes.data, vel.ctypes.data, coords.ctypes.data, man.ctypes.data, cap, 0, 0)
        err = abi.MkError()
        _raise(library().mk_save_state(self._h, C.byref(st), C.byref(err)), err)
        n = min(int(st.manifold_count), cap)
        return {"transforms": tr, "velocities": vel, "coordinates": coords[:q],
                "manifold": man[:n].copy(), "manifold_tick": int(st.manifold_tick)}

    def load_state(self, transforms=None, velocities=None, coordinates=None, manifold=None,
                   manifold_tick: int = 0) -> None:
        keep = []

        def p(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data
        man = None if manifold is None else np.ascontiguousarray(manifold, abi.CONTACT)
        st = abi.MkHostState(p(transforms, abi.TRANSFORM), p(velocities, abi.VELOCITY),
                             p(coordinates, abi.MECHANISM_COORDINATE),
                             None if man is None else (man.ctypes.data if len(man) else
                                                       np.zeros(1, abi.CONTACT).ctypes.data),
                             0 if man is None else len(man), 0 if man is None else len(man),
                             int(manifold_tick))
        keep.append(man)
        err = abi.MkError()
        _raise(library().mk_load_state(self._h, C.byref(st), C.byref(err)), err)

    def read_buffer(self, buffer_id: int, dtype, row_bytes: int) -> np.ndarray:
        count = C.c_uint64()
        err = abi.MkError()
        _raise(library().mk_read_buffer(self._h, buffer_id, None, 0, C.byref(count), C.byref(err)), err)
        n = int(count.value)
        raw = np.zeros(max(n * row_bytes, 1), np.uint8)
        _raise(library().mk_read_buffer(self._h, buffer_id, raw.ctypes.data, raw.nbytes, C.byref(count),
                                        C.byref(err)), err)
        return raw[: n * row_bytes].view(dtype)

    def set_warm_start_network(self, params: np.ndarray) -> None:
        """Loads the warm-start network (MK_WARM_LEARNED uses it from the next tick on)."""
        p = np.ascontiguousarray(params, np.float32)
        err = abi.MkError()
        _raise(library().mk_set_warm_start_network(self._h, p.ctypes.data, len(p), C.byref(err)), err)

    def set_preconditioner_network(self, params: np.ndarray) -> None:
        """Loads the closure preconditioner network (MK_PRECOND_LEARNED)."""
        p = np.ascontiguousarray(params, np.float32)
        err = abi.MkError()
        _raise(library().mk_set_preconditioner_network(self._h, p.ctypes.data, len(p), C.byref(err)), err)

    def closure_slots(self):
        """Jacobian columns of the last evaluated Newton step: (pd (n, 3), ad (n, 3), coord, closure)."""
        raw = self.read_buffer(abi.BUF_CLOSURE_SLOTS, np.float32, 32).reshape(-1, 8)
        return raw[:, 0:3], raw[:, 4:7], raw[:, 3].view(np.uint32), raw[:, 7].view(np.uint32)

    def closure_blocks(self):
        return self.read_buffer(abi.BUF_CLOSURE_BLOCKS, np.float32, 64).reshape(-1, 16)

    def closure_block_outputs(self):
        return self.read_buffer(abi.BUF_CLOSURE_BLOCK_OUTPUTS, np.float32, 12).reshape(12, -1, 3)

    def warm_start_samples(self):
        """(inputs (n, 16), targets (n,)) of the last tick's active contacts."""
        count = C.c_uint32()
        err = abi.MkError()
        _raise(library().mk_read_warm_start_samples(self._h, None, None, 0, C.byref(count), C.byref(err)), err)
        n = int(count.value)
        feats = np.zeros((max(n, 1), 16), np.float32)
        targ = np.zeros(max(n, 1), np.float32)
        _raise(library().mk_read_warm_start_samples(self._h, feats.ctypes.data, targ.ctypes.data, n, C.byref(count),
                                                     C.byref(err)), err)
        return feats[:n], targ[:n]

    # convenience views of internal buffers (last completed tick)
    def pairs(self):
        return self.read_buffer(abi.BUF_PAIRS, abi.PAIR, 8)

    def contacts(self):
        return self.read_buffer(abi.BUF_CONTACTS, abi.CONTACT, 64)

    def contact_keys(self):
        """collider a << 32 | collider b of each contact row (0xffffffff: the ground)."""
        return self.read_buffer(abi.BUF_CONTACT_KEYS, np.uint64, 8)

    def features(self):
        return self.read_buffer(abi.BUF_CONTACT_FEATURES, np.uint32, 4)

    def active(self):
        return self.read_buffer(abi.BUF_ACTIVE, np.uint32, 4)

    def sorted_entries(self):
        return (self.read_buffer(abi.BUF_SORTED_KEYS, np.uint64, 8),
                self.read_buffer(abi.BUF_SORTED_VALUES, np.uint32, 4))

    def collider_keys(self):
        return self.read_buffer(abi.BUF_COLLIDER_KEYS, np.uint64, 8)

    def aabbs(self):
        return self.read_buffer(abi.BUF_COLLIDER_AABBS, np.float32, 32).reshape(-1, 8)

    def node_children(self):
        return self.read_buffer(abi.BUF_NODE_CHILDREN, np.uint32, 8).reshape(-1, 2)

    def node_aabbs(self):
        """(2C - 1, 8) float32: min.xyz, w, max.xyz, 0 per node (internal nodes first, then sorted leaves)."""
        return self.read_buffer(abi.BUF_NODE_AABBS, np.float32, 32).reshape(-1, 8)

    def node_records(self):
        """(C - 1, 32) float32: the 4-wide traversal record of each internal node, entries
        {min.xyz, code bits} {max.xyz, last-leaf bits} of its grandchildren in leaf order."""
        return self.read_buffer(abi.BUF_NODE_RECORDS, np.float32, 128).reshape(-1, 32)

    def world_masses(self):
        return self.read_buffer(abi.BUF_WORLD_MASSES, np.float32, 48).reshape(-1, 12)

    def links(self):
        return self.read_buffer(abi.BUF_LINKS, abi.LINK_STATE, 48)

    def warm_predictions(self):
        return self.read_buffer(abi.BUF_WARM_PREDICTIONS, np.float32, 4)


TUNE_SORT_ITEMS = 1
TUNE_CLOSURE_GRID = 2   # reference-mode closure loop: 0 by size, 1 one block, 2 the whole grid
TUNE_HEAVY_SOLVE = 3    # heavy-tick contact solve: 0 default, 1 scatter (atomics), 2 gather (slots), 3 split
TUNE_PAIR_SORT_ITEMS = 4   # pair-key sort tile (keys per thread as TUNE_SORT_ITEMS; 32 = 512 x 16); 0 default


def set_tuning(key: int, value: int) -> int:
    """Process-wide tuning knob (mk_set_tuning); applies to handles created afterwards."""
    return int(library().mk_set_tuning(int(key), int(value)))


def selftest_bounded_wait(which: int, spin_limit: int = 1000) -> abi.MkWaitProbe:
    """Runs one bounded-wait probe (abi.WAIT_PROBE_*) on the current device."""
    out = abi.MkWaitProbe()
    err = abi.MkError()
    _raise(library().mk_selftest_bounded_wait(int(which), int(spin_limit), C.byref(out), C.byref(err)), err)
    return out


def version() -> str:
    return library().mk_version().decode()
