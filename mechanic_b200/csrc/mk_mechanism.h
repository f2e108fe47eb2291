// mk_mechanism.h — articulated passes (bearing projection, coordinate
// advance, forward kinematics, loop closure, velocity reconstruction,
// validation) of the B200 tick.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "mk_internal.h"

namespace mk {

struct MechParams {
    uint32_t body_count = 0, bearing_count = 0, coordinate_count = 0, max_depth = 0, closure_count = 0;
    uint32_t jump_rounds = 0;        // ceil(log2(max_depth)), at least 1 when max_depth > 0 (device.rs:2103-2111)
    uint32_t final_is_a = 1;         // links_a holds the final FK pass when jump_rounds is even
    uint32_t iterations = 8;
    uint32_t closure_mode = 0;
    uint32_t has_dynamic_root = 0;
    uint32_t serial_contacts = 0;    // dynamic root and <= 64 bearings (device.rs:1370-1373)
    float dt = 1.0f / 60.0f, ang_damp = 0.98f;
    // closure topology (host-derived, static)
    uint32_t closures = 0;           // closure bearings
    uint32_t slots = 0;              // joints on closure branches, over all closures
    uint32_t long_coords = 0;        // closure coordinates with more than kLongList slots
    uint32_t long_chunks = 0;        // chunks of at most kLongList slots over those coordinates' runs
    uint32_t wide_closures = 0;      // closures average 32 slots or more: a warp walks each
    uint32_t closure_coords = 0;     // distinct coordinates on closure branches
    uint32_t closure_bodies = 0;     // bodies of components that contain a closure
    // MK_CLOSURE_PCG_RESIDUAL
    float closure_tol = 1.0e-5f;     // relative PCG residual per Newton step
    uint32_t closure_max_it = 256;   // PCG iterations per Newton step
    uint32_t learned_precond = 0;    // blocks corrected by the preconditioner network
    uint32_t precond = 0;            // MK_PRECOND_*
    uint32_t blocks = 0;             // 2 x 2 preconditioner blocks: ceil(closure_coords / 2)
    uint32_t loops = 0;              // per-loop preconditioner blocks (<= kMaxLoop coordinates each)
};

// Outcome of the closure solve of one tick (MK_CLOSURE_PCG_RESIDUAL).
struct ClosureState {
    uint32_t done;                   // converged at an earlier Newton step
    uint32_t live_blocks;            // blocks the network runs on this step (0 once converged)
    uint32_t newton_steps;
    uint32_t pcg_iterations;
    uint32_t learned_blocks;         // blocks that used the network's correction (summed over steps)
    uint32_t rejected_blocks;        // blocks whose correction was not positive definite
    double max_relative_residual;    // worst final ||r|| / ||r0|| over the Newton steps
};

struct MechBuffers {
    GpuBearing* bearings = nullptr;             // J
    GpuMechanismBody* bodies = nullptr;         // B
    GpuMechanismCoordinate* coords = nullptr;   // Q
    GpuMechanismDrive* drives = nullptr;        // Q
    uint32_t* preorder = nullptr;               // B
    GpuLinkState* links_a = nullptr;            // B
    GpuLinkState* links_b = nullptr;            // B
    GpuLinkState* links_final = nullptr;        // alias of a or b
    int32_t* deltas = nullptr;                  // 6 per body (bearing projection)
    // reconstruct_body_velocities by depth level (level l: bodies [off[l], off[l+1]))
    float4* bear_cache = nullptr;               // 9 float4 per bearing: pose-only parts of its projection rows
    uint32_t* level_bodies = nullptr;
    const uint32_t* level_offsets = nullptr;    // host memory owned by the handle, level_count + 1 entries
    uint32_t level_count = 0;
    // closure loop
    uint32_t* cl_bearings = nullptr;            // closure bearing rows
    uint32_t* cl_slot_off = nullptr;            // closures + 1: slots of closure k (branch a, then branch b)
    uint32_t* cl_split = nullptr;               // first branch-b slot of closure k
    uint32_t* slot_body = nullptr;              // child body of the joint of each slot
    uint32_t* cq_coords = nullptr;              // coordinates on closure branches (ascending)
    uint32_t* cq_off = nullptr;                 // closure_coords + 1: CSR into cq_slots
    uint32_t* cq_slots = nullptr;               // slots of each coordinate, in serial accumulation order
    uint32_t* cb_bodies = nullptr;              // bodies of closure components
    float* slot_g = nullptr;                    // per-slot gradient / operator contributions, stored at the
    float* slot_d = nullptr;                    // slot's position in cq_slots (each coordinate's run contiguous)
    uint32_t* slot_pos = nullptr;               // position of each slot in cq_slots
    uint32_t* long_q = nullptr;                 // closure coordinates (positions) with long slot lists
    uint32_t* long_chunk_off = nullptr;         // long_coords + 1: each long coordinate's first chunk
    uint32_t* chunk_long = nullptr;             // per chunk: its long coordinate (index into long_q)
    float* chunk_g = nullptr;                   // per chunk: its partial sums
    float* chunk_d = nullptr;
    float* grad = nullptr;                      // Q (closure.wgsl:46-49 accumulators)
    float* diag = nullptr;                      // Q
    float* pcg = nullptr;                       // 5 x Q: sol, res, pre, dir, op (closure.wgsl:51-60)
    uint32_t* grid_barrier = nullptr;           // arrival word of the grid-wide closure loop (zero at rest)
    uint32_t* loop_state = nullptr;             // 12 steps x 2: largest residuals (um, udeg), zeroed per tick
    float* chunk_part = nullptr;                // 2 x chunks of 1,024 closure coordinates: dot-product sums
    double* chunk_part_d = nullptr;             // the same in FP64 (closure PCG to a residual)
    uint32_t readback_iterations = 0;
    double readback_residual = 0.0;
    // MK_CLOSURE_PCG_RESIDUAL
    uint32_t* slot_closure = nullptr;           // closure of each slot
    float4* slot_v = nullptr;                   // 2 per slot: the joint's Jacobian column (position, axis rows)
    float4* blk_m = nullptr;                    // per block: preconditioner inverse (m11, m12, m22, -)
    float4* blk_feat = nullptr;                 // 4 per block: network inputs
    float* blk_out = nullptr;                   // 3 per block: network outputs of the current step
    float* blk_hist = nullptr;                  // 12 steps x blocks x 3: outputs used at each Newton step
    float* probe = nullptr;                     // 2 x Q: A * ones, A * alternating signs
    ClosureState* cstate = nullptr;
    float* precond_params = nullptr;            // preconditioner network parameters (mlp::kParams)
    uint32_t* loop_off = nullptr;               // loops + 1: offsets into loop_q
    uint32_t* loop_q = nullptr;                 // closure-coordinate positions of each loop block
    float* loop_l = nullptr;                    // 36 per loop: Cholesky factor (lower, row-major packed)
    void* mlp_scratch = nullptr;
};

MechParams make_mech_params(const MkCreation* cr, const StepParams& p, uint32_t iterations, uint32_t closure_mode,
                            float closure_tol, uint32_t closure_max_it, uint32_t precond);
// Host-side closure topology and depth levels; fills the counts in `p`.
struct MechTopology {
    std::vector<uint32_t> level_bodies, level_offsets;
    std::vector<uint32_t> cl_bearings, cl_slot_off, cl_split, slot_body, cq_coords, cq_off, cq_slots, cb_bodies;
    std::vector<uint32_t> slot_closure, slot_pos, long_q, long_chunk_off, chunk_long;
    std::vector<uint32_t> loop_off, loop_q;
};
MechTopology derive_topology(const MkCreation* cr, MechParams& p);
// Reference-mode closure loop: 0 = by size, 1 = one block, 2 = the whole grid.
void set_closure_grid(uint32_t mode);
uint32_t closure_grid_mode();
// Regions of the mechanism buffers to clear at the start of every tick.
void mechanism_tick_clears(const MechBuffers& m, const MechParams& p, void** ptr, uint64_t* bytes, uint32_t* count);
void carve_mechanism(MechBuffers& m, const MechParams& p, uint32_t B, uint32_t J, uint32_t Q,
                     const std::function<char*(uint64_t)>& take);
bool upload_mechanism(MechBuffers& m, const MechParams& p, const MechTopology& topo, const MkCreation* cr,
                      cudaStream_t s, MkError* err);
cudaError_t enqueue_mechanism(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
bool pcg_residual_mode(const MechParams& p);
cudaError_t enqueue_contact_solver_with_bearings(MechBuffers& m, const StepBuffers& b, const StepParams& sp,
                                                 const MechParams& p, const StepLaunch& l, int parity, cudaStream_t s);
cudaError_t enqueue_post_contact(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
void enqueue_validate_state(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
void enqueue_validate_bearings(MechBuffers& m, const StepBuffers& b, const MechParams& p, bool mechanism_active,
                               cudaStream_t s);
void read_mechanism_readback(const MechBuffers& m, const MechParams& p, const GpuDiagnostics& d,
                             const ClosureState* cs, MkTickReadback* out);
// bytes of network scratch the learned preconditioner needs (0 without it)
uint64_t mechanism_mlp_scratch_bytes(const MechParams& p);

}  // namespace mk
