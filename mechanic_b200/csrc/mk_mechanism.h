// mk_mechanism.h — articulated passes (bearing projection, coordinate
// advance, forward kinematics, loop closure, velocity reconstruction,
// validation) of the B200 tick.
#pragma once

#include <cstdint>
#include <functional>

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
};

struct MechBuffers {
    GpuBearing* bearings = nullptr;             // J
    GpuMechanismBody* bodies = nullptr;         // B
    GpuMechanismCoordinate* coords = nullptr;   // Q
    GpuMechanismDrive* drives = nullptr;        // Q
    uint32_t* preorder = nullptr;               // B
    uint32_t* level_offsets = nullptr;          // depth levels of the preorder (max_depth + 2)
    uint32_t* level_bodies = nullptr;           // bodies grouped by depth
    GpuLinkState* links_a = nullptr;            // B
    GpuLinkState* links_b = nullptr;            // B
    GpuLinkState* links_final = nullptr;        // alias of a or b
    int32_t* deltas = nullptr;                  // 6 per body (bearing projection)
    float* closure_grad = nullptr;              // Q (float CAS accumulators, closure.wgsl:46-49)
    float* closure_diag = nullptr;              // Q
    uint32_t* closure_state = nullptr;          // 2 words + flags
    float* pcg = nullptr;                       // Q x 8 (PcgRow, closure.wgsl:51-60)
    double* reduce = nullptr;                   // FP64 reduction scratch
    uint32_t* closure_bearings = nullptr;       // indices of closure bearings
    uint32_t* readback = nullptr;               // host-visible iteration count / residual bits
    uint32_t readback_iterations = 0;
    double readback_residual = 0.0;
};

MechParams make_mech_params(const MkCreation* cr, const StepParams& p, uint32_t iterations, uint32_t closure_mode);
void carve_mechanism(MechBuffers& m, uint32_t B, uint32_t J, uint32_t Q, const std::function<char*(uint64_t)>& take);
bool upload_mechanism(MechBuffers& m, const MkCreation* cr, cudaStream_t s, MkError* err);
void enqueue_mechanism_prelude(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
cudaError_t enqueue_mechanism(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
cudaError_t enqueue_contact_solver_with_bearings(MechBuffers& m, const StepBuffers& b, const StepParams& sp,
                                                 const MechParams& p, const StepLaunch& l, int parity, cudaStream_t s);
cudaError_t enqueue_post_contact(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
void enqueue_validate_state(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s);
void enqueue_validate_bearings(MechBuffers& m, const StepBuffers& b, const MechParams& p, bool mechanism_active,
                               cudaStream_t s);
void read_mechanism_readback(const MechBuffers& m, MkTickReadback* out);

}  // namespace mk
