// mk_mechanism.cu — articulated passes of the tick.
//
// bearings.wgsl:48-102 (residual validation) is implemented here; the
// articulated solver passes (articulated.wgsl, mechanism.wgsl, closure.wgsl)
// report cudaErrorNotSupported until they land, so a creation with a
// mechanism fails loudly at mk_create instead of stepping without joints.
#include <cstdio>
#include <cstring>
#include <vector>

#include "mk_device.cuh"
#include "mk_mechanism.h"

namespace mk {

MechParams make_mech_params(const MkCreation* cr, const StepParams& p, uint32_t iterations, uint32_t closure_mode) {
    MechParams m;
    m.body_count = cr->body_count;
    m.bearing_count = cr->bearing_count;
    m.coordinate_count = cr->coordinate_count;
    m.max_depth = cr->max_depth;
    m.closure_count = cr->closure_count;
    uint32_t covered = 1, rounds = 0;
    while (covered < cr->max_depth) { covered *= 2; ++rounds; }
    if (cr->max_depth > 0 && rounds == 0) rounds = 1;
    m.jump_rounds = rounds;
    m.final_is_a = (rounds % 2 == 0) ? 1u : 0u;
    m.iterations = iterations;
    m.closure_mode = closure_mode;
    m.has_dynamic_root = cr->has_dynamic_root;
    m.serial_contacts = (cr->has_dynamic_root && cr->bearing_count <= 64) ? 1u : 0u;
    m.dt = p.dt;
    m.ang_damp = p.ang_damp;
    return m;
}

void carve_mechanism(MechBuffers& m, uint32_t B, uint32_t J, uint32_t Q, const std::function<char*(uint64_t)>& take) {
    B = B ? B : 1;
    J = J ? J : 1;
    Q = Q ? Q : 1;
    m.bearings = reinterpret_cast<GpuBearing*>(take(sizeof(GpuBearing) * (uint64_t)J));
    m.bodies = reinterpret_cast<GpuMechanismBody*>(take(sizeof(GpuMechanismBody) * (uint64_t)B));
    m.coords = reinterpret_cast<GpuMechanismCoordinate*>(take(sizeof(GpuMechanismCoordinate) * (uint64_t)Q));
    m.drives = reinterpret_cast<GpuMechanismDrive*>(take(sizeof(GpuMechanismDrive) * (uint64_t)Q));
    m.preorder = reinterpret_cast<uint32_t*>(take(4ull * B));
    m.links_a = reinterpret_cast<GpuLinkState*>(take(sizeof(GpuLinkState) * (uint64_t)B));
    m.links_b = reinterpret_cast<GpuLinkState*>(take(sizeof(GpuLinkState) * (uint64_t)B));
    m.deltas = reinterpret_cast<int32_t*>(take(24ull * B));
}

bool upload_mechanism(MechBuffers& m, const MkCreation* cr, cudaStream_t s, MkError* err) {
    cudaError_t e = cudaSuccess;
    if (cr->bearing_count)
        e = cudaMemcpyAsync(m.bearings, cr->bearings, sizeof(GpuBearing) * cr->bearing_count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && cr->mechanism_bodies)
        e = cudaMemcpyAsync(m.bodies, cr->mechanism_bodies, sizeof(GpuMechanismBody) * cr->body_count,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && cr->preorder)
        e = cudaMemcpyAsync(m.preorder, cr->preorder, 4ull * cr->body_count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && cr->coordinate_count) {
        std::vector<GpuMechanismDrive> d(cr->coordinate_count);
        if (cr->drives) {
            std::memcpy(d.data(), cr->drives, sizeof(GpuMechanismDrive) * cr->coordinate_count);
        } else {
            for (auto& r : d) {   // GpuMechanismDrive::PASSIVE (abi.rs:266-275)
                std::memset(&r, 0, sizeof(r));
                r.min_angle = -INFINITY;
                r.max_angle = INFINITY;
            }
        }
        e = cudaMemcpyAsync(m.drives, d.data(), sizeof(GpuMechanismDrive) * d.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) {
        if (err) {
            std::memset(err, 0, sizeof(*err));
            err->code = MK_ERR_DEVICE_FAILURE;
            std::snprintf(err->message, sizeof(err->message), "upload mechanism: %s", cudaGetErrorString(e));
        }
        return false;
    }
    m.links_final = nullptr;
    return true;
}

void enqueue_mechanism_prelude(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s) {
    (void)b;
    cudaMemsetAsync(m.deltas, 0, 24ull * (p.body_count ? p.body_count : 1), s);
}

cudaError_t enqueue_mechanism(MechBuffers&, const StepBuffers&, const MechParams&, cudaStream_t) {
    return cudaErrorNotSupported;
}

cudaError_t enqueue_contact_solver_with_bearings(MechBuffers&, const StepBuffers&, const StepParams&,
                                                 const MechParams&, const StepLaunch&, int, cudaStream_t) {
    return cudaErrorNotSupported;
}

cudaError_t enqueue_post_contact(MechBuffers&, const StepBuffers&, const MechParams&, cudaStream_t) {
    return cudaErrorNotSupported;
}

void enqueue_validate_state(MechBuffers&, const StepBuffers&, const MechParams&, cudaStream_t) {}

// bearings.wgsl:48-66
__device__ __forceinline__ void record_residual(GpuDiagnostics* d, f3 anchor_a, f3 anchor_b, f3 axis_a, f3 axis_b,
                                                bool closure) {
    const uint32_t um = round_u32(length(anchor_a - anchor_b) * 1000000.0f);
    const float deg = atan2_cr(length(cross(axis_a, axis_b)), clampf(dot(axis_a, axis_b), -1.0f, 1.0f)) * 57.295779513f;
    const uint32_t udeg = round_u32(deg * 1000000.0f);
    atomicMax(&d->max_anchor_micrometers, um);
    atomicMax(&d->max_axis_microdegrees, udeg);
    if (closure && (um > 10u || udeg > 1000u)) atomicOr(&d->error_flags, MK_CONSTRAINT_NON_CONVERGENCE_FLAG);
}

// bearings.wgsl:68-102 (world poses, or the final mechanism links).
__global__ void k_validate_bearings(const GpuBearing* __restrict__ bearings, uint32_t J, const float4* pos,
                                    const float4* rot, const GpuLinkState* links, GpuDiagnostics* diag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J) return;
    const GpuBearing br = bearings[i];
    const uint32_t a = br.metadata[0], c = br.metadata[1];
    float4 pa, qa, pc, qc;
    if (links) {
        pa = *reinterpret_cast<const float4*>(links[a].position);
        qa = *reinterpret_cast<const float4*>(links[a].rotation);
        pc = *reinterpret_cast<const float4*>(links[c].position);
        qc = *reinterpret_cast<const float4*>(links[c].rotation);
    } else {
        pa = pos[a]; qa = rot[a]; pc = pos[c]; qc = rot[c];
    }
    const f3 anchor_a = xyz(pa) + quat_rotate(qa, mkf3(br.local_anchor_a[0], br.local_anchor_a[1], br.local_anchor_a[2]));
    const f3 anchor_b = xyz(pc) + quat_rotate(qc, mkf3(br.local_anchor_b[0], br.local_anchor_b[1], br.local_anchor_b[2]));
    const f3 axis_a = normalize(quat_rotate(qa, mkf3(br.local_axis_a[0], br.local_axis_a[1], br.local_axis_a[2])));
    const f3 axis_b = normalize(quat_rotate(qc, mkf3(br.local_axis_b[0], br.local_axis_b[1], br.local_axis_b[2])));
    record_residual(diag, anchor_a, anchor_b, axis_a, axis_b, br.metadata[3] != 0u);
}

void enqueue_validate_bearings(MechBuffers& m, const StepBuffers& b, const MechParams& p, bool mechanism_active,
                               cudaStream_t s) {
    if (p.bearing_count == 0) return;
    k_validate_bearings<<<(p.bearing_count + 255) / 256, 256, 0, s>>>(m.bearings, p.bearing_count, b.pos, b.rot,
                                                                       mechanism_active ? m.links_final : nullptr,
                                                                       b.diag);
}

void read_mechanism_readback(const MechBuffers& m, MkTickReadback* out) {
    out->closure_iterations = m.readback_iterations;
    out->closure_relative_residual = m.readback_residual;
}

}  // namespace mk
