/*
 * oracle.h — CPU restatement of Mechanic's rigid-body step (TEST
 * INFRASTRUCTURE ONLY).
 *
 * This library is the checker, never the product: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline / reference legs of
 * bench.py load it.  The product path (mechanic_b200) never links, loads or
 * falls back to it.
 *
 * It restates, in the reference's operation order, the WGSL kernels of
 * crates/mechanic-gpu/src/kernels/{physics,lbvh,collision,mechanism,
 * articulated,closure,bearings,snapshot}.wgsl and the CPU narrowphase of
 * crates/mechanic-gpu/src/collision.rs.  It is compiled twice over one
 * template: FP32 (bit-exact parity target, -ffp-contract=off) and FP64
 * (error reporting).
 *
 * Parity pinning: the reference (Rust + WGSL through wgpu) cannot be built or
 * run here, and it ships no golden kernel outputs.  The restatement is pinned
 * against the reference's own known-answer tests (collision.rs:185-233,
 * compile.rs:1011-1142, abi.rs:298-358) and its behavioural tests; kernel-level
 * parity beyond those is "parity unpinned" against the reference itself and is
 * pinned against this restatement.
 */
#ifndef MECHANIC_ORACLE_H
#define MECHANIC_ORACLE_H

#include <stdint.h>
#include "../include/mechanic_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrWorld OrWorld;

/* precision: 32 or 64.  pair_capacity 0 => MK_DEFAULT_MAX_CONTACT_PAIRS. */
OrWorld* or_create(const MkCreation* creation, const MkConfig* config,
                   int precision, uint32_t pair_capacity);
void or_destroy(OrWorld* world);
void or_set_threads(int threads);
int or_get_threads(void);

/* One full tick (device.rs:859-961). */
int or_step(OrWorld* world, uint64_t tick_index);

enum {
    OR_COUNT_PAIRS = 0, OR_COUNT_CONTACTS = 1, OR_COUNT_ACTIVE = 2,
    OR_COUNT_BODIES = 3, OR_COUNT_COLLIDERS = 4, OR_COUNT_MANIFOLD = 5,
    OR_COUNT_COORDINATES = 6, OR_COUNT_BEARINGS = 7
};
uint64_t or_count(const OrWorld* world, int what);

void or_get_state(const OrWorld* world, GpuTransform* transforms, GpuVelocity* velocities);
void or_get_state_f64(const OrWorld* world, double* pos4, double* rot4, double* lin4, double* ang4);
void or_set_state(OrWorld* world, const GpuTransform* transforms, const GpuVelocity* velocities);
void or_get_diagnostics(const OrWorld* world, GpuDiagnostics* out);
void or_get_pairs(const OrWorld* world, GpuPair* out);
void or_get_contacts(const OrWorld* world, GpuContact* out);
void or_get_contacts_f64(const OrWorld* world, double* rows16);
void or_get_contact_keys(const OrWorld* world, uint64_t* out);
void or_get_features(const OrWorld* world, uint32_t* out);
void or_get_active(const OrWorld* world, uint32_t* out);
void or_get_collider_keys(const OrWorld* world, uint64_t* out);
void or_get_sorted(const OrWorld* world, uint64_t* keys, uint32_t* values);
void or_get_aabbs(const OrWorld* world, float* out8);
void or_get_world_masses(const OrWorld* world, float* out12);
void or_get_snapshot(const OrWorld* world, uint32_t slot, GpuTransform* out);
void or_get_coordinates(const OrWorld* world, GpuMechanismCoordinate* out);
void or_set_coordinates(OrWorld* world, const GpuMechanismCoordinate* in);
void or_get_links(const OrWorld* world, GpuLinkState* out);

/* Manifold cache as the list of entries touched on the last tick, sorted by
 * (collider_a, collider_b); each entry uses the GpuContact layout
 * (metadata = body a, body b, collider a, collider b). */
uint32_t or_get_manifold(const OrWorld* world, GpuContact* out, uint32_t capacity);
void or_set_manifold(OrWorld* world, const GpuContact* rows, uint32_t count, uint64_t last_tick);

/* Karras topology (lbvh.wgsl:219-278) over the sorted keys of the last
 * tick: children[2*(C-1)], leaves offset by C-1. */
void or_get_karras(const OrWorld* world, uint32_t* children);

/* ---- function-level restatements used by known-answer tests ---------- */

/* collision.wgsl:393-486 on explicit world boxes (16 floats each:
 * center.xyz+hx, axis_x.xyz+hy, axis_y.xyz+hz, axis_z.xyz+0).
 * Returns feature word (axis 0..14 | near << 8 | early-exit << 16). */
uint32_t or_obb_sat_f32(const float* box_a, const float* box_b, float* normal_penetration);

/* collision.wgsl:266-287 on explicit world boxes. */
void or_contact_point_f32(const float* box_a, const float* box_b, const float* normal, float* point3);

/* collision.rs:43-64 (CPU SAT: A axes then B axes, threshold -1e-6).
 * Returns 1 with normal/penetration, or 0 when separated. */
int or_cpu_obb_sat(const float* center_a, const float* quat_a, const float* half_a,
                   const float* center_b, const float* quat_b, const float* half_b,
                   float* normal_penetration);

/* collision.rs:68-103: returns point count (<= 4), points in out (3 each). */
int or_cpu_contact_manifold(const float* center_a, const float* quat_a, const float* half_a,
                            const float* center_b, const float* quat_b, const float* half_b,
                            float* normal_penetration, float* points);

uint32_t or_morton30(float x, float y, float z);   /* lbvh.wgsl:84-98 */
uint64_t or_morton63(float x, float y, float z, float lx, float ly, float lz, float scale);   /* 21 bits/axis over the centre bounds (lo, scale) */
uint64_t or_morton48(float x, float y, float z, float lx, float ly, float lz, float scale);   /* 16 bits/axis over the centre bounds (lo, scale) */
uint64_t or_morton39(float x, float y, float z, float lx, float ly, float lz, float scale);   /* 13 bits/axis over the centre bounds (lo, scale) */
uint64_t or_morton30a(float x, float y, float z, float lx, float ly, float lz, float scale);  /* 10 bits/axis over the centre bounds (lo, scale) */

#ifdef __cplusplus
}
#endif

#endif
