/*
 * mechanic_b200.h — C ABI of the B200-native Mechanic rigid-body step.
 *
 * The library replaces the wgpu compute path of mechanic-gpu (Rust + WGSL)
 * with hand-written sm_100a CUDA behind plain `extern "C"` entry points:
 * plain pointers and sizes, no C++ or torch types.  Every row type below keeps
 * the byte layout of the matching `#[repr(C)]` row in
 * crates/mechanic-gpu/src/abi.rs, so a caller that already flattens a
 * `CompiledCreation` into GPU rows (device.rs:429-523, :1699-1808) hands the
 * same bytes to `mk_create`.
 *
 * Conventions (mirroring GpuPhysics, crates/mechanic-gpu/src/device.rs:369-1663):
 *   - every fallible call returns an `int` status (MK_OK == 0) and fills an
 *     optional `MkError` with the fields of the Rust error variant it mirrors;
 *   - nothing aborts or throws across the ABI; CUDA failures map to
 *     MK_ERR_DEVICE_FAILURE (runtime.rs:43 `DeviceFailure(String)`);
 *   - a handle owns all of its device memory, one CUDA stream and one CUDA
 *     graph per tick shape; host arrays passed in are copied and stay owned by
 *     the caller;
 *   - a handle is not reentrant (one thread at a time, like `&self` on one
 *     wgpu queue); distinct handles may be used concurrently.
 */
#ifndef MECHANIC_B200_H
#define MECHANIC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MK_API __attribute__((visibility("default")))
#else
#define MK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Failure flags OR-ed into GpuDiagnostics.error_flags (abi.rs:3-13).
 * ------------------------------------------------------------------------- */
#define MK_PAIR_OVERFLOW_FLAG               (1u << 0) /* abi.rs:4  */
#define MK_INVALID_NUMERIC_FLAG             (1u << 1) /* abi.rs:7  */
#define MK_CONSTRAINT_NON_CONVERGENCE_FLAG  (1u << 2) /* abi.rs:10 */
#define MK_MANIFOLD_OVERFLOW_FLAG           (1u << 3) /* abi.rs:13 */
/* No counterpart in the reference: a bounded device-side spin-wait (ordered
 * compaction, radix look-back) gave up instead of hanging the GPU. */
#define MK_DEVICE_WAIT_TIMEOUT_FLAG         (1u << 4)

/* Drive modes (abi.rs:255-262). */
#define MK_DRIVE_MODE_PASSIVE 0u
#define MK_DRIVE_MODE_SPEED   1u
#define MK_DRIVE_MODE_ANGLE   2u

#define MK_INVALID_INDEX 0xffffffffu
#define MK_SNAPSHOT_RING_SIZE 3u /* lib.rs:51 */

/* Reference fixed capacities (lib.rs:36-48).  Here they are only defaults:
 * MkCapacities makes every one a creation-time parameter. */
#define MK_DEFAULT_MAX_BODIES        131072u
#define MK_DEFAULT_MAX_BEARINGS      262144u
#define MK_DEFAULT_MAX_COLLIDERS     131072u
#define MK_DEFAULT_MAX_CONTACT_PAIRS 2097152u

/* ---------------------------------------------------------------------------
 * ABI rows (abi.rs:15-296).  Sizes are asserted in mk_abi.cu and in tests.
 * ------------------------------------------------------------------------- */
typedef struct GpuTickConfig {          /* abi.rs:18-51, 64 bytes */
    uint32_t body_count;
    uint32_t tick_index;
    uint32_t snapshot_slot;
    uint32_t collider_count;
    float delta_seconds;
    float gravity_y;
    float linear_damping;
    float angular_damping;
    uint32_t bearing_count;
    uint32_t suppression_count;
    uint32_t pair_capacity;
    uint32_t flags;
    uint32_t hash_capacity;
    uint32_t solver_iterations;
    uint32_t reserved_a;               /* sort_count in the reference (device.rs:881) */
    uint32_t reserved_b;               /* coordinate count (device.rs:882) */
} GpuTickConfig;

typedef struct GpuDiagnostics {         /* abi.rs:56-73, 32 bytes */
    uint32_t error_flags;
    uint32_t pair_count;
    uint32_t contact_count;
    uint32_t max_anchor_micrometers;
    uint32_t max_axis_microdegrees;
    uint32_t active_contact_count;
    uint32_t reserved_b;
    uint32_t reserved_c;
} GpuDiagnostics;

typedef struct GpuTransform { float position[4]; float rotation[4]; } GpuTransform;   /* abi.rs:78 */
typedef struct GpuVelocity { float linear[4]; float angular[4]; } GpuVelocity;        /* abi.rs:88 */

typedef struct GpuMass {                /* abi.rs:98-107, 64 bytes */
    float inverse_mass[4];
    float inverse_inertia_x[4];
    float inverse_inertia_y[4];
    float inverse_inertia_z[4];
} GpuMass;

typedef struct GpuSpatialInertia {      /* abi.rs:112-121, 64 bytes */
    float mass[4];
    float inertia_x[4];
    float inertia_y[4];
    float inertia_z[4];
} GpuSpatialInertia;

typedef struct GpuCollider {            /* abi.rs:126-135, 64 bytes */
    float local_center[4];              /* w: segment-centre radius (full cylinder) */
    float local_rotation[4];
    float half_extents[4];              /* w: outer radius (full cylinder) */
    uint32_t metadata[4];               /* body, part slot, generation, ground role 0..16 */
} GpuCollider;

typedef struct GpuBearing {             /* abi.rs:140-151, 80 bytes */
    float local_anchor_a[4];
    float local_anchor_b[4];
    float local_axis_a[4];
    float local_axis_b[4];
    uint32_t metadata[4];               /* body a, body b, coordinate or MK_INVALID_INDEX, closure flag */
} GpuBearing;

typedef struct GpuPair { uint32_t collider_a; uint32_t collider_b; } GpuPair;          /* abi.rs:156 */

typedef struct GpuContact {             /* abi.rs:166-175, 64 bytes */
    uint32_t metadata[4];               /* body a, body b, manifold slot, point count */
    float normal_penetration[4];
    float arm_a_impulse[4];
    float arm_b[4];                     /* w: near-face axes (pairs) or -1 (analytic cylinder ground) */
} GpuContact;

typedef struct GpuPersistentManifold {  /* abi.rs:180-187, 48 bytes */
    uint32_t pair_tick[4];
    float normal_penetration[4];
    float point_impulse[4];
} GpuPersistentManifold;

typedef struct GpuMechanismBody {       /* abi.rs:192-201, 64 bytes */
    uint32_t metadata[4];               /* parent, tree bearing row, direction, root flag */
    uint32_t traversal[4];              /* component, depth, preorder, postorder */
    float bind_relative_position[4];
    float bind_relative_rotation[4];
} GpuMechanismBody;

typedef struct GpuMechanismCoordinate { float angle; float angular_velocity; } GpuMechanismCoordinate; /* abi.rs:206 */

typedef struct GpuMechanismDrive {      /* abi.rs:220-238, 32 bytes */
    uint32_t mode;
    float max_acceleration;
    float max_speed;
    float target_speed;
    float target_angle;
    float min_angle;
    float max_angle;
    float padding;
} GpuMechanismDrive;

typedef struct GpuLinkState {           /* abi.rs:281-288, 48 bytes */
    float position[4];
    float rotation[4];
    uint32_t metadata[4];
} GpuLinkState;

typedef struct GpuContractionNode { uint32_t metadata[4]; } GpuContractionNode;      /* abi.rs:293 */

/* ---------------------------------------------------------------------------
 * Status codes and error record.
 * Each MK_ERR_* mirrors one Rust error variant; the fields of MkError that the
 * variant carries are filled, the rest are zero.
 * ------------------------------------------------------------------------- */
enum {
    MK_OK = 0,
    MK_ERR_BODY_CAPACITY = 1,            /* GpuPhysicsError::BodyCapacity{required,capacity} device.rs:136 */
    MK_ERR_BEARING_CAPACITY = 2,         /* GpuPhysicsError::BearingCapacity device.rs:144 */
    MK_ERR_COLLIDER_CAPACITY = 3,        /* GpuPhysicsError::ColliderCapacity device.rs:152 */
    MK_ERR_DRIVE_STATE_COUNT = 4,        /* GpuPhysicsError::DriveStateCount{provided,required} device.rs:160 */
    MK_ERR_COORDINATE_STATE_COUNT = 5,   /* GpuPhysicsError::CoordinateStateCount device.rs:168 */
    MK_ERR_BODY_INDEX_OUT_OF_RANGE = 6,  /* GpuImpulseError::BodyIndexOutOfRange{body_index,body_count} device.rs:180 */
    MK_ERR_NON_FINITE = 7,               /* GpuImpulseError::NonFinite device.rs:188 */
    MK_ERR_INVALID_SNAPSHOT_SLOT = 8,    /* GpuReadbackError::InvalidSnapshotSlot(u8) device.rs:117 */
    MK_ERR_DEVICE_FAILURE = 9,           /* FailureStatus::DeviceFailure(String) runtime.rs:43 */
    MK_ERR_INVALID_ARGUMENT = 10,        /* no reference counterpart: null pointer / inconsistent sizes */
    MK_ERR_PAIR_CAPACITY = 11,           /* CapacityKind::ContactPairs runtime.rs:13 (creation-time check) */
};

typedef struct MkError {
    int32_t code;
    uint32_t body_index;
    uint32_t body_count;
    uint32_t slot;
    uint64_t required;
    uint64_t capacity;
    uint64_t provided;
    char message[256];
} MkError;

/* Lifecycle state and terminal failure of a loaded scene (runtime.rs:7-56). */
enum { MK_CAPACITY_BODIES = 0, MK_CAPACITY_BEARINGS = 1, MK_CAPACITY_CONTACT_PAIRS = 2 };
enum {
    MK_FAILURE_NONE = 0,
    MK_FAILURE_INVALID_TOPOLOGY = 1,
    MK_FAILURE_CONSTRAINT_NON_CONVERGENCE = 2,
    MK_FAILURE_CAPACITY_OVERFLOW = 3,
    MK_FAILURE_INVALID_NUMERIC_STATE = 4,
    MK_FAILURE_DEVICE_FAILURE = 5,
};
enum { MK_STATUS_BUILDING = 0, MK_STATUS_PAUSED = 1, MK_STATUS_RUNNING = 2, MK_STATUS_FAILED = 3 };

/* ---------------------------------------------------------------------------
 * Creation, configuration and capacities.
 * ------------------------------------------------------------------------- */

/* Flattened CompiledCreation: exactly the rows device.rs uploads.
 * Arrays marked "optional" may be NULL. */
typedef struct MkCreation {
    uint32_t body_count;
    uint32_t collider_count;
    uint32_t bearing_count;
    uint32_t suppression_count;
    uint32_t coordinate_count;           /* tree bearings (loop_topology.tree_bearings.len()) */
    uint32_t max_depth;                  /* max GpuMechanismBody.traversal[1]; 0 => no mechanism */
    const GpuTransform* transforms;      /* body_count: root translation (w unused) + rotation */
    const GpuVelocity* velocities;       /* optional: body_count initial velocities; the reference uploads zeros (device.rs:442) */
    const GpuMass* masses;               /* body_count */
    const GpuSpatialInertia* spatial_inertias; /* optional: body_count */
    const GpuCollider* colliders;        /* collider_count, contiguous per body */
    const GpuBearing* bearings;          /* bearing_count */
    const GpuPair* suppressed_pairs;     /* suppression_count, body pairs sorted ascending (low, high) */
    const GpuMechanismBody* mechanism_bodies; /* optional when max_depth == 0: body_count */
    const uint32_t* root_flags;          /* optional: body_count; NULL => every body is a root */
    const uint32_t* preorder;            /* optional when max_depth == 0: body_count */
    const uint32_t* body_components;     /* optional: body_count mechanism component per body */
    const GpuMechanismDrive* drives;     /* optional: coordinate_count (NULL => passive rows) */
    uint32_t closure_count;              /* bearings with metadata[3] != 0 */
    uint32_t has_dynamic_root;           /* a root with inverse mass > 0 (device.rs:1687-1695) */
} MkCreation;

/* GpuPhysicsConfig (device.rs:22-41) plus B200-build switches. */
typedef struct MkConfig {
    uint32_t collisions_enabled;         /* default 1 */
    uint32_t mechanism_self_collisions;  /* default 1 */
    uint32_t solver_iterations;          /* default 8 */
    uint32_t morton_mode;                /* MK_MORTON_39 (default), MK_MORTON_30_ADAPTIVE, MK_MORTON_48, MK_MORTON_63 or
                                            MK_MORTON_REFERENCE_30 */
    uint32_t closure_mode;               /* MK_CLOSURE_* */
    uint32_t use_graph;                  /* 1: capture the tick into a CUDA graph (default) */
    float delta_seconds;                 /* 0 => 1/60 (lib.rs:31) */
    float gravity_y;                     /* 0 => -9.81 (device.rs:872) */
    float linear_damping;                /* 0 => 0.999 */
    float angular_damping;               /* 0 => 0.98 */
    int32_t device;                      /* CUDA device ordinal */
    uint32_t warm_start;                 /* MK_WARM_CACHED (default) or MK_WARM_LEARNED */
    float contact_tolerance;             /* 0 (default): solver_iterations fixed passes (device.rs:1343-1416);
                                            > 0: passes until ||r|| <= tolerance * ||r_cold|| (no reference
                                            counterpart) */
    uint32_t contact_max_iterations;     /* cap on passes when contact_tolerance > 0; 0 => 512 */
    float closure_tolerance;             /* MK_CLOSURE_PCG_RESIDUAL: relative PCG residual; 0 => 1e-5 */
    uint32_t closure_max_iterations;     /* MK_CLOSURE_PCG_RESIDUAL: PCG iterations per Newton step; 0 => 256 */
    uint32_t preconditioner;             /* MK_PRECOND_BLOCK_JACOBI (default), _LEARNED, _PAIR_BLOCKS, _DIAGONAL */
    uint32_t contact_manifold;           /* MK_MANIFOLD_POINT (default) or MK_MANIFOLD_CLIPPED */
} MkConfig;

#define MK_MANIFOLD_POINT       0u  /* collision.wgsl:540-620: one averaged point per colliding pair */
#define MK_MANIFOLD_CLIPPED     1u  /* collision.rs:68-103 rule: up to four contained vertices per pair */

#define MK_WARM_CACHED          0u  /* collision.wgsl:774-839: cached impulse x 0.5 (x 1 for cylinder-ground) */
#define MK_WARM_LEARNED         1u  /* warm-start network next to the cached start; the lower residual wins */

#define MK_PRECOND_BLOCK_JACOBI 0u  /* per-closure-loop blocks: Cholesky of J^T J on each loop's coordinates */
#define MK_PRECOND_LEARNED      1u  /* 2 x 2 blocks of consecutive closure coordinates, inverse from the network */
#define MK_PRECOND_PAIR_BLOCKS  2u  /* 2 x 2 blocks, exact 2 x 2 inverse (the learned form's own baseline) */
#define MK_PRECOND_DIAGONAL     3u  /* the reference's Jacobi preconditioner r / diag(J^T J) (closure.wgsl:343-400) */

#define MK_MORTON_63            0u  /* 21 bits/axis over the tick's bounds of the collider centres (cubic cells),
                                       index tie-break through a stable sort */
#define MK_MORTON_REFERENCE_30  1u  /* lbvh.wgsl:93-98: 10 bits/axis, 1 m cells */
#define MK_MORTON_48            2u  /* 16 bits/axis over the same bounds; two radix passes fewer than
                                       MK_MORTON_63 (cells of extent / 65535) */
#define MK_MORTON_39            3u  /* default: 13 bits/axis over the same bounds; one radix pass fewer than
                                       MK_MORTON_48 (cells of extent / 8191) */
#define MK_MORTON_30_ADAPTIVE   4u  /* 10 bits/axis over the same bounds; one radix pass fewer than MK_MORTON_39
                                       (cells of extent / 1023, coarse for large scenes with dense clusters):
                                       mk_autotune chooses between the two by timing */

#define MK_CLOSURE_REFERENCE    0u  /* closure.wgsl:333-427: 8 fixed diagonal-PCG rounds per Newton step */
#define MK_CLOSURE_PCG_RESIDUAL 1u  /* parallel block-Jacobi PCG to a relative residual, FP64 reductions */

typedef struct MkCapacities {
    uint32_t max_bodies;                 /* 0 => body_count */
    uint32_t max_colliders;              /* 0 => collider_count */
    uint32_t max_bearings;               /* 0 => bearing_count */
    uint32_t pair_capacity;              /* 0 => MK_DEFAULT_MAX_CONTACT_PAIRS; candidate pairs and contacts */
} MkCapacities;

typedef struct MkHandle MkHandle;

typedef struct MkSubmission {            /* GpuTickSubmission (device.rs:63-71) */
    uint64_t tick_index;
    uint8_t snapshot_slot;
    uint8_t pad[7];
    uint64_t submission_index;
} MkSubmission;

typedef struct MkKernelTimings {         /* GpuKernelTimings (device.rs:96-112) */
    double integration_ms;
    double mechanism_ms;
    double broadphase_ms;
    double narrowphase_ms;
    double contact_solver_ms;
    double bearings_ms;
    double snapshot_ms;
} MkKernelTimings;

typedef struct MkTickReadback {          /* GpuTickReadback (device.rs:73-92) */
    uint32_t has_timestamps;             /* always 1: CUDA events */
    uint32_t error_flags;
    double gpu_tick_ms;
    MkKernelTimings kernel_timings;
    uint32_t pair_count;
    uint32_t contact_count;
    uint32_t active_contact_count;
    float anchor_residual_meters;
    float axis_residual_degrees;
    uint32_t closure_iterations;         /* no reference counterpart: PCG iterations used by the closure solve */
    double closure_relative_residual;    /* no reference counterpart: final ||r||/||r0|| of the closure PCG */
    uint32_t contact_iterations;         /* no reference counterpart: contact passes run (warm pass included) */
    uint32_t warm_start_used;            /* MK_WARM_CACHED, MK_WARM_LEARNED, or 2: learned start rejected */
    double contact_relative_residual;    /* no reference counterpart: last ||r|| / ||r_cold|| (residual mode) */
} MkTickReadback;

/* Device pointers of the live state (all borrowed, valid until mk_destroy). */
typedef struct MkDeviceState {
    void* positions;            /* float4[body_count] */
    void* rotations;            /* float4[body_count] */
    void* linear_velocities;    /* float4[body_count] */
    void* angular_velocities;   /* float4[body_count] */
    void* inverse_masses;       /* float[body_count] */
    void* coordinates;          /* GpuMechanismCoordinate[coordinate_count] */
    void* diagnostics;          /* GpuDiagnostics */
    void* stream;               /* cudaStream_t the handle issues work on */
} MkDeviceState;

/* Host copy of everything a tick reads and writes besides the constant rows,
 * so that "one step from an identical state" can be replayed (no reference
 * counterpart: the reference checkpoints only the snapshot ring). */
typedef struct MkHostState {
    GpuTransform* transforms;            /* body_count */
    GpuVelocity* velocities;             /* body_count */
    GpuMechanismCoordinate* coordinates; /* coordinate_count (may be NULL when 0) */
    GpuContact* manifold_contacts;       /* optional: capacity rows of the previous tick's contacts */
    uint32_t manifold_capacity;          /* rows available in manifold_contacts */
    uint32_t manifold_count;             /* out (save) / in (load) */
    uint64_t manifold_tick;              /* tick that wrote the manifold rows (out / in) */
} MkHostState;

/* PublishedGpuState (runtime.rs:60-75): the newest complete pair of snapshot
 * slots.  Each mk_dispatch_tick publishes its tick (publish_tick,
 * runtime.rs:222-237): previous <- current, current <- (tick % 3, tick).
 * The slots' contents are complete once the submission has finished. */
typedef struct MkPublishedState {
    uint64_t generation;                 /* changes with every handle (scene) created in the process */
    uint8_t previous_slot;
    uint8_t current_slot;
    uint8_t pad[6];
    uint64_t previous_tick;
    uint64_t current_tick;
    uint32_t body_count;
    uint32_t ticks_published;            /* 0, 1 or 2: how many of the pair hold a tick */
} MkPublishedState;

/* Internal buffers readable for parity checks (mk_read_buffer). */
enum {
    MK_BUF_SORTED_KEYS = 0,        /* uint64[collider_count] Morton keys in sorted order */
    MK_BUF_SORTED_VALUES = 1,      /* uint32[collider_count] collider index in sorted order */
    MK_BUF_COLLIDER_AABBS = 2,     /* float4 min, float4 max per collider */
    MK_BUF_NODE_CHILDREN = 3,      /* uint2[collider_count-1] Karras children (leaves offset by C-1) */
    MK_BUF_NODE_AABBS = 4,         /* float4 min, float4 max per node (2C-1) */
    MK_BUF_PAIRS = 5,              /* GpuPair[pair_count], canonical (collider_a ascending, then collider_b) */
    MK_BUF_CONTACTS = 6,           /* GpuContact[contact_count] after the solve */
    MK_BUF_ACTIVE = 7,             /* uint32[active_count] contact indices */
    MK_BUF_COLLIDER_KEYS = 8,      /* uint64[collider_count] Morton key per collider (unsorted) */
    MK_BUF_CONTACT_FEATURES = 9,   /* uint32[contact_count]: SAT axis index 0..14 | near_face_axes << 8 */
    MK_BUF_WORLD_MASSES = 10,      /* float4 x 3 per body */
    MK_BUF_LINKS = 11,             /* GpuLinkState[body_count] final mechanism links */
    MK_BUF_WARM_PREDICTIONS = 12,  /* float[active_count] learned warm-start impulses (MK_WARM_LEARNED) */
    MK_BUF_WARM_FEATURES = 13,     /* float[active_count][16] warm-start network inputs (contact_tolerance > 0) */
    MK_BUF_CLOSURE_SLOTS = 14,     /* MK_CLOSURE_PCG_RESIDUAL, last evaluated Newton step, per closure-branch joint:
                                      {position column xyz, coordinate (u32 bits)}, {axis column xyz, closure (u32)} */
    MK_BUF_CLOSURE_BLOCKS = 15,    /* float[blocks][16] preconditioner network inputs of the same step */
    MK_BUF_CLOSURE_BLOCK_OUTPUTS = 16, /* float[12][blocks][3] (t11, t12, t22) the network gave at each Newton step */
    MK_BUF_NODE_RECORDS = 17,      /* float4[8] per internal node (collider_count-1): its traversal record, up to
                                      four grandchildren in leaf order as {min.xyz, code} {max.xyz, last leaf};
                                      code = node index or 0x80000000 | collider index; unused entries zero */
    MK_BUF_CONTACT_KEYS = 18,      /* uint64[contact_count]: collider a << 32 | collider b (0xffffffff for the
                                      ground) of each contact row */
};

/* ---------------------------------------------------------------------------
 * GpuPhysics replacement (device.rs:369-1663).
 * ------------------------------------------------------------------------- */

/* Defaults of MkConfig (GpuPhysicsConfig::default, device.rs:33-41). */
MK_API void mk_config_default(MkConfig* config);

/* GpuPhysics::new_with_config (device.rs:399).  Checks capacities first
 * (device.rs:405-422) and reports BodyCapacity / BearingCapacity /
 * ColliderCapacity with {required, capacity}.  `capacities == NULL` applies
 * the reference's fixed limits (lib.rs:36-45); otherwise each zero field is
 * sized to the creation (pair_capacity 0 => MK_DEFAULT_MAX_CONTACT_PAIRS). */
MK_API int mk_create(const MkCreation* creation, const MkConfig* config,
              const MkCapacities* capacities, MkHandle** out, MkError* err);

MK_API void mk_destroy(MkHandle* handle);

/* Batched independent scenes (no reference counterpart): `scene_count`
 * creations stepped together by every launch of one handle.  Rows are
 * concatenated scene by scene with their body, bearing, coordinate and
 * mechanism-component indices offset; colliders of different scenes never
 * pair (each collider's sorted key carries its scene index in the top bits
 * and the traversal stops at its scene's last leaf), while all other stages
 * run over the concatenated rows as one scene.  Snapshots, state buffers and
 * readbacks are the concatenated arrays; mk_scene_offsets gives the slices.
 * Error flags and counts are totals over the batch; a contact or closure
 * tolerance applies to the batch's joint residual.  Capacities apply to the
 * totals. */
MK_API int mk_create_batch(const MkCreation* scenes, uint32_t scene_count, const MkConfig* config,
                           const MkCapacities* capacities, MkHandle** out, MkError* err);
/* Body and collider offset of each scene plus the totals (scene_count + 1 entries each,
 * at most `capacity` written); returns the scene count (1 for mk_create handles). */
MK_API int mk_scene_offsets(const MkHandle* handle, uint32_t* body_offsets, uint32_t* collider_offsets,
                            uint32_t capacity);

/* GpuPhysics::dispatch_tick (device.rs:859-961): asynchronous on the
 * handle's stream; errors surface through GpuDiagnostics flags. */
MK_API int mk_dispatch_tick(MkHandle* handle, uint64_t tick_index, MkSubmission* out);

/* Replaces device.poll(wait_indefinitely) for one submission. */
MK_API int mk_wait(MkHandle* handle, uint64_t submission_index);

/* GpuPhysics::read_last_tick (device.rs:1439-1524). Blocks on the last tick. */
MK_API int mk_read_last_tick(MkHandle* handle, MkTickReadback* out);

/* GpuPhysics::read_snapshot_transforms (device.rs:1534-1570); `out` holds
 * `capacity` rows of caller-owned host memory (pinned memory copies fastest).
 * MK_ERR_INVALID_SNAPSHOT_SLOT for slot >= 3.  Reads the slot as the last
 * dispatched tick that wrote it left it, and waits for that tick and the copy
 * only: ticks dispatched after it keep running (the copy runs on the handle's
 * copy stream), so a caller that dispatches tick k + 1 before reading tick k's
 * slot overlaps the two. */
MK_API int mk_read_snapshot(MkHandle* handle, uint8_t slot, GpuTransform* out,
                     uint32_t capacity, MkError* err);

/* GpuPhysics::snapshot(slot).positions()/rotations() (device.rs:1578-1610):
 * borrowed device pointers (float4 rows). */
MK_API int mk_snapshot_buffers(MkHandle* handle, uint8_t slot, void** positions,
                        void** rotations, MkError* err);

/* Render hand-off between the published pair (scheduler.rs:69-73 gives the
 * fraction alpha of the way from the previous to the current tick): writes
 * body_count float4 positions lerp(p_prev, p_cur, alpha) and float4 unit
 * rotations slerp(q_prev, q_cur, alpha) along the shorter arc into caller
 * device memory (16-byte aligned), on `stream`, after the ticks that wrote
 * both slots; the next tick that rewrites either slot waits for it.  alpha
 * outside [0, 1] returns MK_ERR_INVALID_ARGUMENT.  No graphics interop: the
 * outputs are plain device buffers. */
MK_API int mk_published_state(MkHandle* handle, MkPublishedState* out);
MK_API int mk_interpolate_snapshot(MkHandle* handle, float alpha, void* positions_out, void* rotations_out,
                                   void* stream, MkError* err);

/* GpuPhysics::apply_impulse (device.rs:821-857 / physics.wgsl:73-90). */
MK_API int mk_apply_impulse(MkHandle* handle, uint32_t body_index,
                     const float world_point[3], const float impulse[3], MkError* err);

/* GpuPhysics::write_mechanism_drives (device.rs:1622-1640). */
MK_API int mk_write_drives(MkHandle* handle, const GpuMechanismDrive* drives,
                    uint32_t count, MkError* err);

/* GpuPhysics::initialize_mechanism_coordinates (device.rs:1646-1662). */
MK_API int mk_init_coordinates(MkHandle* handle, const GpuMechanismCoordinate* coordinates,
                        uint32_t count, MkError* err);

/* GpuPhysics::body_count / has_gpu_timestamps (device.rs:1573-1586). */
MK_API uint32_t mk_body_count(const MkHandle* handle);
MK_API int mk_has_gpu_timestamps(const MkHandle* handle);

/* Borrowed device pointers of the live state (positions()/rotations()/...,
 * device.rs:1588-1610). */
MK_API int mk_state_buffers(MkHandle* handle, MkDeviceState* out);

/* Checkpoint / restore of the mutable state (no reference counterpart). */
MK_API int mk_save_state(MkHandle* handle, MkHostState* out, MkError* err);
MK_API int mk_load_state(MkHandle* handle, const MkHostState* in, MkError* err);

/* Copies an internal buffer (MK_BUF_*) of the last completed tick to host
 * memory; `*count` receives the number of valid rows. */
MK_API int mk_read_buffer(MkHandle* handle, uint32_t buffer_id, void* host,
                   uint64_t capacity_bytes, uint64_t* count, MkError* err);

/* Number of this library's kernels one tick launches (kernel nodes of the
 * captured tick graph; 0 before the first capture or without a graph). */
MK_API uint32_t mk_tick_kernel_count(const MkHandle* handle);

/* Process-wide tuning knobs read when a tick is captured (mk_create) or an
 * operation is launched.  Keys: MK_TUNE_SORT_ITEMS (keys per thread of a
 * radix-sort tile: 2, 4, 6, 8, 11 or 16, or 32 for the 8,192-key tile of 512
 * threads x 16 keys; 0 = size-based default);
 * MK_TUNE_CLOSURE_GRID (the closure solves, the reference's loop and the PCG
 * to a residual: 0 = by size, one block below 512 closures and the whole grid
 * from there, 1 = always one block, 2 = always the grid; both give the same
 * results).  Returns the
 * previous value, or -1 for an unknown key. */
#define MK_TUNE_SORT_ITEMS 1u
#define MK_TUNE_CLOSURE_GRID 2u
/* Contact solve of heavy ticks (more active contacts than twice the bodies):
 * 0 = the default (the fastest measured form); 1 = scatter: per-contact
 * atomic adds into the bodies' delta rows; 2 = gather: each contact writes
 * its fixed-point deltas to its own slot and each body sums its contacts'
 * slots through an incidence list; 3 = split: body a (contacts arrive grouped
 * by it) by warp-summed atomics, body b through slots and incidence lists.
 * Same bits in every form. */
#define MK_TUNE_HEAVY_SOLVE 3u
/* Tile of the pair-key sort (keys per thread, as MK_TUNE_SORT_ITEMS; 0 = the
 * default), fixed when a tick is captured: the pair count is known on the
 * device only. */
#define MK_TUNE_PAIR_SORT_ITEMS 4u
MK_API int mk_set_tuning(uint32_t key, uint32_t value);

/* Launch shapes of one handle's tick (no reference counterpart).  0 in any
 * field means the built-in default (for solve_items: every block). */
typedef struct MkTuning {
    uint32_t sort_items;          /* keys per thread of the collider sort's 256-thread onesweep tile: 2, 4, 6,
                                     8, 11 or 16, or 32 for 512 threads x 16 (default by size: 8 up to 64k keys,
                                     11 up to 2M, else 32) */
    uint32_t sort_ctas_per_sm;    /* onesweep CTAs per SM (default 1 for the 8,192-key tile, 2 for 11 or 16
                                     keys, 3 for 8, else 6) */
    uint32_t append_ctas_per_sm;  /* CTAs per SM of the ordered-append kernels (default 8) */
    uint32_t solve_items;         /* 0 (default): every SM's block joins the cooperative solve; n > 0: only
                                     enough blocks for n contacts (and 4n bodies) per thread */
    uint32_t morton_mode;         /* the broadphase's key mode (MK_MORTON_*; the creation config's until
                                     tuned): start from mk_get_handle_tuning, since 0 is MK_MORTON_63 */
} MkTuning;
MK_API int mk_get_handle_tuning(const MkHandle* handle, MkTuning* out);
/* Applies a tuning; the tick's CUDA graphs are captured again. */
MK_API int mk_set_handle_tuning(MkHandle* handle, const MkTuning* tuning, MkError* err);
/* Autotuner: from the handle's current state, times the next `ticks` ticks
 * (graphs uploaded first) for each candidate shape, varying one field at a time over
 * two sweeps (the launch shapes and, for a handle in MK_MORTON_39 or
 * MK_MORTON_30_ADAPTIVE, the key mode between those two), restoring the state
 * before every candidate; a change is kept only
 * when it is at least 2% faster.  The fastest
 * tuning is applied and the state restored again; *best_ms_per_tick
 * receives its time.  The handle must not be in use meanwhile. */
MK_API int mk_autotune(MkHandle* handle, uint32_t ticks, MkTuning* best, double* best_ms_per_tick,
                       MkError* err);

/* Library identity: returns "mechanic_b200 <version> sm_100a". */
MK_API const char* mk_version(void);

/* Last CUDA error text seen by this thread (empty when none). */
MK_API const char* mk_last_error(void);

/* ---------------------------------------------------------------------------
 * Stream-ordered device operations (device pointers in, device pointers out).
 * They are the building blocks of the tick and are exported for callers that
 * keep their own buffers.  `stream` is a cudaStream_t (NULL = default stream).
 * ------------------------------------------------------------------------- */

/* Scratch bytes mk_op_sort_keys needs for n entries. */
MK_API uint64_t mk_op_sort_scratch_bytes(uint32_t n);

/* Stable LSD onesweep radix sort of 63-bit keys with 32-bit values
 * (replaces the bitonic sort_local_initial / sort_global_step /
 * sort_local_merge passes, lbvh.wgsl:132-217).  Equal keys keep input order,
 * which is the reference's (code, index) tie-break when values are indices.
 * `scratch` must hold mk_op_sort_scratch_bytes(n) bytes, 256-byte aligned.
 * Results land in keys_out / values_out; inputs are left unchanged.  Inputs
 * and outputs must not overlap (MK_ERR_INVALID_ARGUMENT otherwise). */
MK_API int mk_op_sort_keys(const uint64_t* keys_in, const uint32_t* values_in,
                    uint64_t* keys_out, uint32_t* values_out, uint32_t n,
                    uint32_t key_bits, void* scratch, uint64_t scratch_bytes,
                    void* stream);

/* The same sort for callers that cannot allocate device memory when they
 * need it (allocator and memory-pool hooks that must not recurse into the
 * allocator, embedders with a fixed memory budget).  No counterpart in the
 * reference.  Its scratch is a static device array owned by the library
 * (about 14 MB on every GPU that loads it, kept until exit), so only inputs
 * and outputs are passed and nothing is allocated.  It launches kernels on
 * `stream`, so it must not be called from inside a CUDA host function
 * (cudaLaunchHostFunc, stream callbacks), where no CUDA call is allowed.  At
 * most MK_STATIC_SORT_MAX_KEYS keys; larger n, or inputs that overlap the
 * outputs, return MK_ERR_INVALID_ARGUMENT with the reason in mk_last_error().
 * The first call on each device (with it current) looks up the array's
 * device address and keeps it: make that call before any stream capture, and
 * make no call after cudaDeviceReset in the same process (the kept address
 * belongs to the context the reset destroyed).  All calls share the array,
 * so calls that overlap on the GPU race and must be ordered by the caller. */
#define MK_STATIC_SORT_MAX_KEYS 524288u
MK_API int mk_op_sort_keys_static(const uint64_t* keys_in, const uint32_t* values_in,
                                  uint64_t* keys_out, uint32_t* values_out, uint32_t n,
                                  uint32_t key_bits, void* stream);

/* Batched OBB separating-axis test of collision.wgsl:393-486 for `count`
 * pairs of world boxes.  Each box is four float4 rows:
 * {center.xyz, half_x}, {axis_x.xyz, half_y}, {axis_y.xyz, half_z},
 * {axis_z.xyz, unused}.  Writes per pair: normal.xyz + penetration (float4)
 * and a feature word (axis index 0..14 | near_face_axes << 8 | early-exit bit 16). */
MK_API int mk_op_obb_sat(const float* boxes_a, const float* boxes_b, uint32_t count,
                  float* normal_penetration, uint32_t* features, void* stream);

/* Learned contact warm start (no reference counterpart).  With
 * contact_tolerance > 0 every tick records 16 inputs per active contact at
 * the start of the contact solve (relative normal velocity, tangential
 * speed, depth rate, normal, inverse-mass share, cached impulse, bias,
 * cylinder-ground and ground flags, cold step, log and value of the impulse
 * denominator D); the network maps them to the converged impulse x D.
 * mk_set_warm_start_network loads mk_mlp_param_count() parameters (host
 * memory); with warm_start = MK_WARM_LEARNED the learned start then runs
 * beside the cached one and the lower residual after one pass continues.
 * mk_read_warm_start_samples copies the last tick's inputs (count x 16
 * floats) and targets (the converged impulse x D, count floats) into host
 * memory; *count receives the number of active contacts, of which at most
 * capacity rows are written. */
MK_API int mk_set_warm_start_network(MkHandle* handle, const float* params, uint32_t count, MkError* err);
MK_API int mk_read_warm_start_samples(MkHandle* handle, float* features, float* targets, uint32_t capacity,
                                      uint32_t* count, MkError* err);

/* Learned closure preconditioner (no reference counterpart).  With
 * closure_mode = MK_CLOSURE_PCG_RESIDUAL and preconditioner = MK_PRECOND_LEARNED
 * the network maps 16 inputs per 2 x 2 block of consecutive closure
 * coordinates (normalised coupling, log diagonal ratio, off-block row sums
 * of J^T J against ones and alternating signs, pair flag) to (y0, y1, y2),
 * the block of S M^-1 S (S = diag(sqrt(diag(J^T J)))) being t11 = e^y0,
 * t22 = e^y1, t12 = 0.999 tanh(y2) sqrt(t11 t22), positive definite by
 * construction; a block whose output is not finite keeps the plain 2 x 2
 * inverse.  MK_BUF_CLOSURE_BLOCK_OUTPUTS holds the (t11, t12, t22) used.
 * Loads mk_mlp_param_count() parameters from host memory. */
MK_API int mk_set_preconditioner_network(MkHandle* handle, const float* params, uint32_t count, MkError* err);

/* ---------------------------------------------------------------------
 * The learned parts' network (no reference counterpart): 16 inputs (input
 * slot 15 is replaced by the constant 1 that carries the first layer's
 * bias), two hidden layers of 64 with ReLU, 16 outputs.  Parameters are one
 * f32 device array of mk_mlp_param_count() floats, row-major [out][in]:
 * W1 64x16 | W2 64x64 | W3 16x64 | b2 64 | b3 16.  The kernels compute with
 * bf16 weights and activations on the tcgen05 tensor cores, f32 accumulation.
 * All pointers are device pointers; x and targets rows are 16 floats,
 * 16-byte aligned.  Waits inside the kernels are bounded: a timeout sets
 * MK_DEVICE_WAIT_TIMEOUT_FLAG in *error_flags (device memory). */
MK_API uint32_t mk_mlp_param_count(void);
MK_API uint64_t mk_op_mlp_scratch_bytes(uint32_t max_samples);
/* y[n][y_cols] = net(x[n][16]), 1 <= y_cols <= 16. */
MK_API int mk_op_mlp_forward(const float* params, const float* x, uint32_t n, float* y, uint32_t y_cols,
                             void* scratch, uint64_t scratch_bytes, uint32_t* error_flags, void* stream);
/* Gradient of L = (1/n) sum_s sum_o out_weights[o] (y_so - targets_so)^2 with respect to the
 * parameters, into grad[mk_mlp_param_count() + 1] (L in the last slot). */
MK_API int mk_op_mlp_gradient(const float* params, const float* x, const float* targets,
                              const float* out_weights, uint32_t n, float* grad, void* scratch,
                              uint64_t scratch_bytes, uint32_t* error_flags, void* stream);
/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8) over consecutive batches of `batch` samples,
 * cycling through the n samples; losses (device, optional) receives each step's batch loss. */
MK_API int mk_op_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* targets,
                           const float* out_weights, uint32_t n, uint32_t batch, uint32_t steps, float lr,
                           uint32_t first_step, float* losses, void* scratch, uint64_t scratch_bytes,
                           uint32_t* error_flags, void* stream);

/* ---------------------------------------------------------------------
 * Self-test of the bounded device waits (no reference counterpart: the
 * reference's waits, the storageBarrier refit of lbvh.wgsl:290-319, assume
 * arrival).  Every spin-wait in this library's kernels gives up after an
 * iteration limit, raises MK_DEVICE_WAIT_TIMEOUT_FLAG and returns.  This
 * call runs the same device wait functions on a wait that nothing can
 * satisfy, with `spin_limit` (1..65536) polls instead of the kernels' 2^20:
 * a grid barrier expecting one block more than were launched, an ordered-
 * append look-back tile whose predecessor never publishes, or an mbarrier
 * no thread arrives on.  It allocates a few bytes of device memory on the
 * current device, runs on its own stream and returns once the probe ended. */
enum {
    MK_WAIT_PROBE_GRID_BARRIER = 0,
    MK_WAIT_PROBE_LOOKBACK = 1,
    MK_WAIT_PROBE_MBARRIER = 2,
};
typedef struct MkWaitProbe {
    uint32_t error_flags;       /* MK_DEVICE_WAIT_TIMEOUT_FLAG when the wait gave up */
    uint32_t blocks_launched;
    uint32_t blocks_finished;   /* blocks that reached the end of the probe kernel */
    uint32_t pad;
    uint64_t lookback_prefix;   /* look-back probe: the prefix the tile went on with (0) */
    double elapsed_ms;          /* device time of the probe kernel */
} MkWaitProbe;
MK_API int mk_selftest_bounded_wait(uint32_t which, uint32_t spin_limit, MkWaitProbe* out, MkError* err);

#ifdef __cplusplus
}
#endif

#endif /* MECHANIC_B200_H */
