"""ABI rows of mechanic-gpu as numpy dtypes and ctypes structures.

Every row keeps the byte layout of its ``#[repr(C)]`` twin in
crates/mechanic-gpu/src/abi.rs (sizes asserted at abi.rs:298-315); the
ctypes structures mirror include/mechanic_b200.h one to one.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

PAIR_OVERFLOW_FLAG = 1 << 0                 # abi.rs:4
INVALID_NUMERIC_FLAG = 1 << 1               # abi.rs:7
CONSTRAINT_NON_CONVERGENCE_FLAG = 1 << 2    # abi.rs:10
MANIFOLD_OVERFLOW_FLAG = 1 << 3             # abi.rs:13
DEVICE_WAIT_TIMEOUT_FLAG = 1 << 4           # no reference counterpart (bounded device waits)

DRIVE_MODE_PASSIVE = 0                      # abi.rs:256
DRIVE_MODE_SPEED = 1                        # abi.rs:259
DRIVE_MODE_ANGLE = 2                        # abi.rs:262

INVALID_INDEX = 0xFFFFFFFF
SNAPSHOT_RING_SIZE = 3                      # lib.rs:51
FIXED_DT_SECONDS = np.float32(1.0 / 60.0)   # lib.rs:31
MAX_BODIES = 131_072                        # lib.rs:36
MAX_BEARINGS = 262_144                      # lib.rs:39
MAX_COLLIDERS = 131_072                     # lib.rs:42
MAX_CONTACT_PAIRS = 2_097_152               # lib.rs:45

MORTON_63 = 0
MORTON_REFERENCE_30 = 1
MORTON_48 = 2
MORTON_39 = 3
MORTON_30_ADAPTIVE = 4
CLOSURE_REFERENCE = 0
CLOSURE_PCG_RESIDUAL = 1
WARM_CACHED = 0
WARM_LEARNED = 1
WARM_LEARNED_REJECTED = 2
PRECOND_BLOCK_JACOBI = 0
PRECOND_LEARNED = 1
PRECOND_PAIR_BLOCKS = 2
PRECOND_DIAGONAL = 3       # the reference's Jacobi preconditioner, iterated to the residual
MANIFOLD_POINT = 0
MANIFOLD_CLIPPED = 1

# ---------------------------------------------------------------- numpy rows
f4 = (np.float32, 4)
u4 = (np.uint32, 4)
TRANSFORM = np.dtype([("position", f4), ("rotation", f4)])                       # 32 B
VELOCITY = np.dtype([("linear", f4), ("angular", f4)])                           # 32 B
MASS = np.dtype([("inverse_mass", f4), ("inverse_inertia_x", f4),
                 ("inverse_inertia_y", f4), ("inverse_inertia_z", f4)])          # 64 B
SPATIAL_INERTIA = np.dtype([("mass", f4), ("inertia_x", f4), ("inertia_y", f4),
                            ("inertia_z", f4)])                                  # 64 B
COLLIDER = np.dtype([("local_center", f4), ("local_rotation", f4),
                     ("half_extents", f4), ("metadata", u4)])                    # 64 B
BEARING = np.dtype([("local_anchor_a", f4), ("local_anchor_b", f4),
                    ("local_axis_a", f4), ("local_axis_b", f4), ("metadata", u4)])  # 80 B
PAIR = np.dtype([("collider_a", np.uint32), ("collider_b", np.uint32)])         # 8 B
CONTACT = np.dtype([("metadata", u4), ("normal_penetration", f4),
                    ("arm_a_impulse", f4), ("arm_b", f4)])                       # 64 B
PERSISTENT_MANIFOLD = np.dtype([("pair_tick", u4), ("normal_penetration", f4),
                                ("point_impulse", f4)])                          # 48 B
MECHANISM_BODY = np.dtype([("metadata", u4), ("traversal", u4),
                           ("bind_relative_position", f4),
                           ("bind_relative_rotation", f4)])                      # 64 B
MECHANISM_COORDINATE = np.dtype([("angle", np.float32),
                                 ("angular_velocity", np.float32)])              # 8 B
MECHANISM_DRIVE = np.dtype([("mode", np.uint32), ("max_acceleration", np.float32),
                            ("max_speed", np.float32), ("target_speed", np.float32),
                            ("target_angle", np.float32), ("min_angle", np.float32),
                            ("max_angle", np.float32), ("padding", np.float32)])  # 32 B
LINK_STATE = np.dtype([("position", f4), ("rotation", f4), ("metadata", u4)])   # 48 B
CONTRACTION_NODE = np.dtype([("metadata", u4)])                                  # 16 B
TICK_CONFIG = np.dtype([(n, np.uint32) for n in ("body_count", "tick_index", "snapshot_slot",
                                                  "collider_count")]
                       + [(n, np.float32) for n in ("delta_seconds", "gravity_y",
                                                    "linear_damping", "angular_damping")]
                       + [(n, np.uint32) for n in ("bearing_count", "suppression_count",
                                                    "pair_capacity", "flags", "hash_capacity",
                                                    "solver_iterations", "reserved_a",
                                                    "reserved_b")])              # 64 B
DIAGNOSTICS = np.dtype([(n, np.uint32) for n in (
    "error_flags", "pair_count", "contact_count", "max_anchor_micrometers",
    "max_axis_microdegrees", "active_contact_count", "reserved_b", "reserved_c")])  # 32 B

ROW_SIZES = {
    "GpuTickConfig": (TICK_CONFIG, 64), "GpuDiagnostics": (DIAGNOSTICS, 32),
    "GpuTransform": (TRANSFORM, 32), "GpuVelocity": (VELOCITY, 32),
    "GpuMass": (MASS, 64), "GpuSpatialInertia": (SPATIAL_INERTIA, 64),
    "GpuCollider": (COLLIDER, 64), "GpuBearing": (BEARING, 80), "GpuPair": (PAIR, 8),
    "GpuContact": (CONTACT, 64), "GpuPersistentManifold": (PERSISTENT_MANIFOLD, 48),
    "GpuMechanismBody": (MECHANISM_BODY, 64),
    "GpuMechanismCoordinate": (MECHANISM_COORDINATE, 8),
    "GpuMechanismDrive": (MECHANISM_DRIVE, 32), "GpuLinkState": (LINK_STATE, 48),
    "GpuContractionNode": (CONTRACTION_NODE, 16),
}


def passive_drive_rows(count: int) -> np.ndarray:
    """``GpuMechanismDrive::PASSIVE`` rows (abi.rs:266-275): never clamp an angle."""
    rows = np.zeros(count, MECHANISM_DRIVE)
    rows["mode"] = DRIVE_MODE_PASSIVE
    rows["min_angle"] = -np.inf
    rows["max_angle"] = np.inf
    return rows


# ------------------------------------------------------------ ctypes mirror
_vp = C.c_void_p


class MkCreation(C.Structure):
    _fields_ = [
        ("body_count", C.c_uint32), ("collider_count", C.c_uint32),
        ("bearing_count", C.c_uint32), ("suppression_count", C.c_uint32),
        ("coordinate_count", C.c_uint32), ("max_depth", C.c_uint32),
        ("transforms", _vp), ("velocities", _vp), ("masses", _vp),
        ("spatial_inertias", _vp), ("colliders", _vp), ("bearings", _vp),
        ("suppressed_pairs", _vp), ("mechanism_bodies", _vp), ("root_flags", _vp),
        ("preorder", _vp), ("body_components", _vp), ("drives", _vp),
        ("closure_count", C.c_uint32), ("has_dynamic_root", C.c_uint32),
    ]


class MkConfig(C.Structure):
    _fields_ = [
        ("collisions_enabled", C.c_uint32), ("mechanism_self_collisions", C.c_uint32),
        ("solver_iterations", C.c_uint32), ("morton_mode", C.c_uint32),
        ("closure_mode", C.c_uint32), ("use_graph", C.c_uint32),
        ("delta_seconds", C.c_float), ("gravity_y", C.c_float),
        ("linear_damping", C.c_float), ("angular_damping", C.c_float),
        ("device", C.c_int32), ("warm_start", C.c_uint32),
        ("contact_tolerance", C.c_float), ("contact_max_iterations", C.c_uint32),
        ("closure_tolerance", C.c_float), ("closure_max_iterations", C.c_uint32),
        ("preconditioner", C.c_uint32), ("contact_manifold", C.c_uint32),
    ]


class MkPublishedState(C.Structure):
    _fields_ = [("generation", C.c_uint64), ("previous_slot", C.c_uint8), ("current_slot", C.c_uint8),
                ("pad", C.c_uint8 * 6), ("previous_tick", C.c_uint64), ("current_tick", C.c_uint64),
                ("body_count", C.c_uint32), ("ticks_published", C.c_uint32)]


class MkWaitProbe(C.Structure):
    _fields_ = [("error_flags", C.c_uint32), ("blocks_launched", C.c_uint32), ("blocks_finished", C.c_uint32),
                ("pad", C.c_uint32), ("lookback_prefix", C.c_uint64), ("elapsed_ms", C.c_double)]


WAIT_PROBE_GRID_BARRIER = 0
WAIT_PROBE_LOOKBACK = 1
WAIT_PROBE_MBARRIER = 2


def config_default() -> MkConfig:
    """The values mk_config_default writes (GpuPhysicsConfig::default,
    device.rs:33-41, plus this build's key width), filled without loading the
    CUDA library so that CPU-only code can build a configuration row."""
    c = MkConfig()
    c.collisions_enabled = 1
    c.mechanism_self_collisions = 1
    c.solver_iterations = 8
    c.morton_mode = MORTON_39
    c.closure_mode = CLOSURE_REFERENCE
    c.use_graph = 1
    return c


class MkCapacities(C.Structure):
    _fields_ = [("max_bodies", C.c_uint32), ("max_colliders", C.c_uint32),
                ("max_bearings", C.c_uint32), ("pair_capacity", C.c_uint32)]


class MkError(C.Structure):
    _fields_ = [("code", C.c_int32), ("body_index", C.c_uint32), ("body_count", C.c_uint32),
                ("slot", C.c_uint32), ("required", C.c_uint64), ("capacity", C.c_uint64),
                ("provided", C.c_uint64), ("message", C.c_char * 256)]


class MkSubmission(C.Structure):
    _fields_ = [("tick_index", C.c_uint64), ("snapshot_slot", C.c_uint8),
                ("pad", C.c_uint8 * 7), ("submission_index", C.c_uint64)]


class MkKernelTimings(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "integration_ms", "mechanism_ms", "broadphase_ms", "narrowphase_ms",
        "contact_solver_ms", "bearings_ms", "snapshot_ms")]


class MkTickReadback(C.Structure):
    _fields_ = [("has_timestamps", C.c_uint32), ("error_flags", C.c_uint32),
                ("gpu_tick_ms", C.c_double), ("kernel_timings", MkKernelTimings),
                ("pair_count", C.c_uint32), ("contact_count", C.c_uint32),
                ("active_contact_count", C.c_uint32), ("anchor_residual_meters", C.c_float),
                ("axis_residual_degrees", C.c_float), ("closure_iterations", C.c_uint32),
                ("closure_relative_residual", C.c_double), ("contact_iterations", C.c_uint32),
                ("warm_start_used", C.c_uint32), ("contact_relative_residual", C.c_double)]


class MkTuning(C.Structure):
    _fields_ = [("sort_items", C.c_uint32), ("sort_ctas_per_sm", C.c_uint32),
                ("append_ctas_per_sm", C.c_uint32), ("solve_items", C.c_uint32), ("morton_mode", C.c_uint32)]


class MkDeviceState(C.Structure):
    _fields_ = [(n, _vp) for n in (
        "positions", "rotations", "linear_velocities", "angular_velocities",
        "inverse_masses", "coordinates", "diagnostics", "stream")]


class MkHostState(C.Structure):
    _fields_ = [("transforms", _vp), ("velocities", _vp), ("coordinates", _vp),
                ("manifold_contacts", _vp), ("manifold_capacity", C.c_uint32),
                ("manifold_count", C.c_uint32), ("manifold_tick", C.c_uint64)]


# MkError codes (include/mechanic_b200.h)
MK_OK = 0
MK_ERR_BODY_CAPACITY = 1
MK_ERR_BEARING_CAPACITY = 2
MK_ERR_COLLIDER_CAPACITY = 3
MK_ERR_DRIVE_STATE_COUNT = 4
MK_ERR_COORDINATE_STATE_COUNT = 5
MK_ERR_BODY_INDEX_OUT_OF_RANGE = 6
MK_ERR_NON_FINITE = 7
MK_ERR_INVALID_SNAPSHOT_SLOT = 8
MK_ERR_DEVICE_FAILURE = 9
MK_ERR_INVALID_ARGUMENT = 10
MK_ERR_PAIR_CAPACITY = 11

# internal buffer ids (mk_read_buffer)
BUF_SORTED_KEYS = 0
BUF_SORTED_VALUES = 1
BUF_COLLIDER_AABBS = 2
BUF_NODE_CHILDREN = 3
BUF_NODE_AABBS = 4
BUF_PAIRS = 5
BUF_CONTACTS = 6
BUF_ACTIVE = 7
BUF_COLLIDER_KEYS = 8
BUF_CONTACT_FEATURES = 9
BUF_WORLD_MASSES = 10
BUF_LINKS = 11
BUF_WARM_PREDICTIONS = 12
BUF_WARM_FEATURES = 13
BUF_CLOSURE_SLOTS = 14
BUF_CLOSURE_BLOCKS = 15
BUF_CLOSURE_BLOCK_OUTPUTS = 16
BUF_NODE_RECORDS = 17
BUF_CONTACT_KEYS = 18


def ptr(a: np.ndarray | None) -> int | None:
    """Host address of a C-contiguous array (None stays None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "ABI arrays must be C-contiguous"
    return a.ctypes.data
