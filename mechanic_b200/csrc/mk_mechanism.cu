// mk_mechanism.cu — articulated passes of the tick.
//
// Stage map (reference kernel -> this file), in the dispatch order of
// device.rs:963-1155:
//   articulated.wgsl project_bearing_velocities :287-316   -> k_project_bearings
//   articulated.wgsl apply_velocity_deltas :318-337        -> k_apply_mdeltas
//   articulated.wgsl advance_coordinates :366-415          -> k_advance_coordinates
//   mechanism.wgsl prepare_links / jump_* :72-149          -> k_prepare_links / k_jump (list-restricted)
//   closure.wgsl evaluate / finalize / solve_closure_pcg   -> k_closure_loop (one block, all 12 Newton steps)
//   mechanism.wgsl publish_* :151-185                      -> k_publish
//   articulated.wgsl reconstruct_body_velocities :431-456  -> k_reconstruct_level (one launch per depth)
//   articulated.wgsl capture_coordinates :417-429          -> k_capture_coordinates
//   articulated.wgsl validate_articulated_state :458-484   -> k_validate_state
//   bearings.wgsl validate_* :68-102                       -> k_validate_bearings
//   articulated.wgsl project_bearing_velocities_serial     -> k_project_bearings_serial
//
// The serial reconstruction becomes level-synchronous (every body of depth
// d after all of depth d-1: the same arithmetic per body, so the same bits).
// The closure accumulators are gathered per coordinate from per-joint slots
// in the serial accumulation order instead of float atomics.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "mk_device.cuh"
#include "mk_mechanism.h"
#include "mk_mlp.h"

namespace mk {

constexpr uint32_t kMBlock = 256;
constexpr uint32_t kClosureThreads = 1024;
constexpr uint32_t kClosureSteps = 12;     // device.rs:974
constexpr uint32_t kClosureRounds = 8;     // closure.wgsl:356
constexpr uint32_t kMaxLoop = 8;           // coordinates of one per-loop preconditioner block (storage)
// A closure constrains 5 directions (3 of position, 2 of its hinge axis), so a
// loop's J^T J has rank at most 5: a block of more of its coordinates is
// singular (its Cholesky then hangs on the ridge alone, and the preconditioned
// iteration diverged on 16-body loops).  Loops are cut into pieces of 5.
constexpr uint32_t kLoopPiece = 5;
constexpr uint32_t kBearingCache = 9;     // float4 per bearing in the projection cache
constexpr uint32_t kLongList = 256;        // slot runs longer than this are summed in chunks of this many

// ----------------------------------------------------------------- host side
MechParams make_mech_params(const MkCreation* cr, const StepParams& p, uint32_t iterations, uint32_t closure_mode,
                            float closure_tol, uint32_t closure_max_it, uint32_t learned_precond) {
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
    m.serial_contacts = (cr->max_depth > 0 && cr->has_dynamic_root && cr->bearing_count <= 64) ? 1u : 0u;
    m.dt = p.dt;
    m.ang_damp = p.ang_damp;
    m.closure_tol = closure_tol > 0.0f ? closure_tol : 1.0e-5f;
    m.closure_max_it = closure_max_it ? closure_max_it : 256u;
    m.learned_precond = (closure_mode == MK_CLOSURE_PCG_RESIDUAL && learned_precond == MK_PRECOND_LEARNED) ? 1u : 0u;
    m.precond = learned_precond;
    return m;
}

bool pcg_residual_mode(const MechParams& p) { return p.closure_mode == MK_CLOSURE_PCG_RESIDUAL && p.closures > 0; }

MechTopology derive_topology(const MkCreation* cr, MechParams& p) {
    MechTopology t;
    const uint32_t B = cr->body_count;
    if (cr->max_depth == 0 || !cr->mechanism_bodies) return t;
    const GpuMechanismBody* mb = cr->mechanism_bodies;
    // depth levels 1..max_depth (roots are skipped by the reconstruction)
    t.level_offsets.assign(cr->max_depth + 2, 0);
    for (uint32_t i = 0; i < B; ++i)
        if (!mb[i].metadata[3] && mb[i].traversal[1] <= cr->max_depth) ++t.level_offsets[mb[i].traversal[1] + 1];
    for (size_t l = 1; l < t.level_offsets.size(); ++l) t.level_offsets[l] += t.level_offsets[l - 1];
    t.level_bodies.resize(t.level_offsets.back());
    std::vector<uint32_t> fill(t.level_offsets.begin(), t.level_offsets.end() - 1);
    for (uint32_t i = 0; i < B; ++i)
        if (!mb[i].metadata[3] && mb[i].traversal[1] <= cr->max_depth) t.level_bodies[fill[mb[i].traversal[1]]++] = i;
    // closure branches: walk each endpoint to its root (closure.wgsl:154-192)
    std::map<uint32_t, std::vector<uint32_t>> coord_slots;
    std::vector<uint8_t> closure_root(B, 0);
    t.cl_slot_off.push_back(0);
    for (uint32_t j = 0; j < cr->bearing_count; ++j) {
        const GpuBearing& br = cr->bearings[j];
        if (br.metadata[3] == 0) continue;
        t.cl_bearings.push_back(j);
        for (int side = 0; side < 2; ++side) {
            if (side == 1) t.cl_split.push_back((uint32_t)t.slot_body.size());
            uint32_t body = br.metadata[side];
            for (uint32_t guard = 0; guard <= B && body < B; ++guard) {
                if (mb[body].metadata[3] != 0) { closure_root[body] = 1; break; }
                const uint32_t coord = cr->bearings[mb[body].metadata[1]].metadata[2];
                coord_slots[coord].push_back((uint32_t)t.slot_body.size());
                t.slot_body.push_back(body);
                body = mb[body].metadata[0];
            }
        }
        t.cl_slot_off.push_back((uint32_t)t.slot_body.size());
    }
    t.cq_off.push_back(0);
    for (auto& kv : coord_slots) {
        t.cq_coords.push_back(kv.first);
        for (uint32_t sl : kv.second) t.cq_slots.push_back(sl);
        t.cq_off.push_back((uint32_t)t.cq_slots.size());
    }
    // bodies whose root carries a closure: the only links the closure loop changes
    if (!t.cl_bearings.empty()) {
        for (uint32_t i = 0; i < B; ++i) {
            uint32_t body = i;
            for (uint32_t guard = 0; guard <= B && mb[body].metadata[3] == 0; ++guard) body = mb[body].metadata[0];
            if (closure_root[body]) t.cb_bodies.push_back(i);
        }
    }
    // slot values are stored at their position in cq_slots, so each coordinate reads its
    // run contiguously; runs longer than kLongList (coordinates near the root of a large
    // loop lattice carry a slot of nearly every closure) are summed in chunks
    t.slot_pos.assign(t.slot_body.size(), 0u);
    for (uint32_t i = 0; i < (uint32_t)t.cq_slots.size(); ++i) t.slot_pos[t.cq_slots[i]] = i;
    t.long_chunk_off.push_back(0);
    for (uint32_t q = 0; q + 1 < (uint32_t)t.cq_off.size(); ++q) {
        const uint32_t n = t.cq_off[q + 1] - t.cq_off[q];
        if (n <= kLongList) continue;
        const uint32_t w = (uint32_t)t.long_q.size();
        t.long_q.push_back(q);
        for (uint32_t c = 0; c < (n + kLongList - 1) / kLongList; ++c) t.chunk_long.push_back(w);
        t.long_chunk_off.push_back((uint32_t)t.chunk_long.size());
    }
    p.long_coords = (uint32_t)t.long_q.size();
    p.wide_closures = (!t.cl_bearings.empty() && t.slot_body.size() >= 32ull * t.cl_bearings.size()) ? 1u : 0u;
    p.long_chunks = (uint32_t)t.chunk_long.size();
    t.slot_closure.resize(t.slot_body.size());
    for (size_t k = 0; k + 1 < t.cl_slot_off.size(); ++k)
        for (uint32_t sl = t.cl_slot_off[k]; sl < t.cl_slot_off[k + 1]; ++sl) t.slot_closure[sl] = (uint32_t)k;
    p.closures = (uint32_t)t.cl_bearings.size();
    p.slots = (uint32_t)t.slot_body.size();
    p.closure_coords = (uint32_t)t.cq_coords.size();
    p.closure_bodies = (uint32_t)t.cb_bodies.size();
    p.blocks = (p.closure_coords + 1) / 2;
    // per-loop blocks: each closure coordinate joins the block of the first closure that
    // contains it; loops longer than kLoopPiece are cut into consecutive pieces
    {
        std::map<uint32_t, uint32_t> position;
        for (uint32_t q = 0; q < t.cq_coords.size(); ++q) position[t.cq_coords[q]] = q;
        std::vector<uint8_t> taken(t.cq_coords.size(), 0);
        t.loop_off.push_back(0);
        for (size_t k = 0; k + 1 < t.cl_slot_off.size(); ++k) {
            std::vector<uint32_t> qs;
            for (uint32_t sl = t.cl_slot_off[k]; sl < t.cl_slot_off[k + 1]; ++sl) {
                const uint32_t coord = cr->bearings[mb[t.slot_body[sl]].metadata[1]].metadata[2];
                auto it = position.find(coord);
                if (it == position.end() || taken[it->second]) continue;
                taken[it->second] = 1;
                qs.push_back(it->second);
            }
            std::sort(qs.begin(), qs.end());
            for (size_t i = 0; i < qs.size(); i += kLoopPiece) {
                for (size_t j = i; j < std::min<size_t>(qs.size(), i + kLoopPiece); ++j) t.loop_q.push_back(qs[j]);
                t.loop_off.push_back((uint32_t)t.loop_q.size());
            }
        }
        p.loops = (uint32_t)t.loop_off.size() - 1;
    }
    return t;
}

void carve_mechanism(MechBuffers& m, const MechParams& p, uint32_t B, uint32_t J, uint32_t Q,
                     const std::function<char*(uint64_t)>& take) {
    B = B ? B : 1;
    J = J ? J : 1;
    Q = Q ? Q : 1;
    auto u32 = [&](uint64_t n) { return reinterpret_cast<uint32_t*>(take(4ull * (n ? n : 1))); };
    auto f32 = [&](uint64_t n) { return reinterpret_cast<float*>(take(4ull * (n ? n : 1))); };
    m.bearings = reinterpret_cast<GpuBearing*>(take(sizeof(GpuBearing) * (uint64_t)J));
    m.bodies = reinterpret_cast<GpuMechanismBody*>(take(sizeof(GpuMechanismBody) * (uint64_t)B));
    m.coords = reinterpret_cast<GpuMechanismCoordinate*>(take(sizeof(GpuMechanismCoordinate) * (uint64_t)Q));
    m.drives = reinterpret_cast<GpuMechanismDrive*>(take(sizeof(GpuMechanismDrive) * (uint64_t)Q));
    m.preorder = u32(B);
    m.links_a = reinterpret_cast<GpuLinkState*>(take(sizeof(GpuLinkState) * (uint64_t)B));
    m.links_b = reinterpret_cast<GpuLinkState*>(take(sizeof(GpuLinkState) * (uint64_t)B));
    m.deltas = reinterpret_cast<int32_t*>(take(24ull * B));
    m.bear_cache = reinterpret_cast<float4*>(take(16ull * kBearingCache * (J ? J : 1)));
    m.level_bodies = u32(B);
    m.cl_bearings = u32(p.closures);
    m.cl_slot_off = u32(p.closures + 1);
    m.cl_split = u32(p.closures);
    m.slot_body = u32(p.slots);
    m.cq_coords = u32(p.closure_coords);
    m.cq_off = u32(p.closure_coords + 1);
    m.cq_slots = u32(p.slots);
    m.cb_bodies = u32(p.closure_bodies);
    m.slot_g = f32(p.slots);
    m.slot_d = f32(p.slots);
    m.slot_pos = u32(p.slots);
    m.long_q = u32(p.long_coords);
    m.long_chunk_off = u32(p.long_coords + 1);
    m.chunk_long = u32(p.long_chunks);
    m.chunk_g = f32(p.long_chunks);
    m.chunk_d = f32(p.long_chunks);
    m.grad = f32(Q);
    m.diag = f32(Q);
    m.pcg = f32(5ull * Q);
    m.grid_barrier = u32(64);   // its own 256-byte line
    m.loop_state = u32(2ull * kClosureSteps);
    m.chunk_part = f32(2ull * ((p.closure_coords + kClosureThreads - 1) / kClosureThreads));
    m.chunk_part_d = reinterpret_cast<double*>(take(16ull * ((p.closure_coords + kClosureThreads - 1) / kClosureThreads + 1)));
    m.links_final = p.final_is_a ? m.links_a : m.links_b;
    m.slot_v = reinterpret_cast<float4*>(take(32ull * (p.slots ? p.slots : 1)));   // Jacobian columns
    if (pcg_residual_mode(p)) {
        m.slot_closure = u32(p.slots);
        m.blk_m = reinterpret_cast<float4*>(take(16ull * (p.blocks ? p.blocks : 1)));
        m.blk_feat = reinterpret_cast<float4*>(take(64ull * (p.blocks ? p.blocks : 1)));
        m.blk_out = f32(3ull * p.blocks);
        m.blk_hist = f32(3ull * kClosureSteps * p.blocks);
        m.probe = f32(2ull * Q);
        m.cstate = reinterpret_cast<ClosureState*>(take(sizeof(ClosureState)));
        if (p.learned_precond) {
            m.precond_params = f32(mlp::kParams + 16);
            m.mlp_scratch = take(mlp::scratch_bytes(0));
        }
        m.loop_off = u32(p.loops + 1);
        m.loop_q = u32(p.closure_coords);
        m.loop_l = f32(36ull * p.loops);
    }
}

template <class T>
static cudaError_t put(T* dst, const std::vector<T>& v, cudaStream_t s) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s);
}

bool upload_mechanism(MechBuffers& m, const MechParams& p, const MechTopology& t, const MkCreation* cr,
                      cudaStream_t s, MkError* err) {
    cudaError_t e = cudaSuccess;
    if (cr->bearing_count)
        e = cudaMemcpyAsync(m.bearings, cr->bearings, sizeof(GpuBearing) * cr->bearing_count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && cr->mechanism_bodies)
        e = cudaMemcpyAsync(m.bodies, cr->mechanism_bodies, sizeof(GpuMechanismBody) * cr->body_count,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && cr->preorder)
        e = cudaMemcpyAsync(m.preorder, cr->preorder, 4ull * cr->body_count, cudaMemcpyHostToDevice, s);
    std::vector<GpuMechanismDrive> d(cr->coordinate_count);
    if (cr->coordinate_count) {
        if (cr->drives) {
            std::memcpy(d.data(), cr->drives, sizeof(GpuMechanismDrive) * cr->coordinate_count);
        } else {
            for (auto& r : d) {   // GpuMechanismDrive::PASSIVE (abi.rs:266-275)
                std::memset(&r, 0, sizeof(r));
                r.min_angle = -INFINITY;
                r.max_angle = INFINITY;
            }
        }
        if (e == cudaSuccess) e = put(m.drives, d, s);
    }
    if (e == cudaSuccess) e = put(m.level_bodies, t.level_bodies, s);
    if (e == cudaSuccess) e = put(m.cl_bearings, t.cl_bearings, s);
    if (e == cudaSuccess) e = put(m.cl_slot_off, t.cl_slot_off, s);
    if (e == cudaSuccess) e = put(m.cl_split, t.cl_split, s);
    if (e == cudaSuccess && m.slot_closure) e = put(m.slot_closure, t.slot_closure, s);
    if (e == cudaSuccess && m.loop_off) e = put(m.loop_off, t.loop_off, s);
    if (e == cudaSuccess && m.loop_q) e = put(m.loop_q, t.loop_q, s);
    if (e == cudaSuccess && m.precond_params) e = mlp::pack(m.precond_params, m.mlp_scratch, s);
    if (e == cudaSuccess) e = put(m.slot_body, t.slot_body, s);
    if (e == cudaSuccess) e = put(m.cq_coords, t.cq_coords, s);
    if (e == cudaSuccess) e = put(m.cq_off, t.cq_off, s);
    if (e == cudaSuccess) e = put(m.cq_slots, t.cq_slots, s);
    if (e == cudaSuccess) e = put(m.slot_pos, t.slot_pos, s);
    if (e == cudaSuccess && !t.long_q.empty()) e = put(m.long_q, t.long_q, s);
    if (e == cudaSuccess && !t.long_q.empty()) e = put(m.long_chunk_off, t.long_chunk_off, s);
    if (e == cudaSuccess && !t.chunk_long.empty()) e = put(m.chunk_long, t.chunk_long, s);
    if (e == cudaSuccess) e = put(m.cb_bodies, t.cb_bodies, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    (void)p;
    if (e != cudaSuccess) {
        if (err) {
            std::memset(err, 0, sizeof(*err));
            err->code = MK_ERR_DEVICE_FAILURE;
            std::snprintf(err->message, sizeof(err->message), "upload mechanism: %s", cudaGetErrorString(e));
        }
        return false;
    }
    return true;
}

// --------------------------------------------------------------- device math
__device__ __forceinline__ f3 r3(const float* v) { return mkf3(v[0], v[1], v[2]); }
__device__ __forceinline__ float4 r4(const float* v) { return make_float4(v[0], v[1], v[2], v[3]); }

// articulated.wgsl:94-102: world inverse inertia from the body-frame rows.
__device__ __forceinline__ f3 wii(const StepBuffers& b, uint32_t body, f3 v) {
    const float4 r = b.rot[body];
    const f3 l = quat_rotate(conjq(r), v);
    const float4* m = b.mass + 4ull * body;
    const f3 lr = xyz(m[1]) * l.x + xyz(m[2]) * l.y + xyz(m[3]) * l.z;
    return quat_rotate(r, lr);
}
__device__ __forceinline__ float inv_mass(const StepBuffers& b, uint32_t body) { return b.mass[4ull * body].x; }

// One body's fixed-point deltas summed in registers: a row's contribution is
// converted as add_mdelta does and the integer sums wrap as the atomics do,
// so one atomic per component gives the same totals as one per row.
struct MDelta {
    uint32_t v[6];
};
__device__ __forceinline__ void mdelta_add(MDelta& acc, f3 l, f3 a) {
    const float s = 1048576.0f;
    acc.v[0] += (uint32_t)fixed_i32(l.x * s);
    acc.v[1] += (uint32_t)fixed_i32(l.y * s);
    acc.v[2] += (uint32_t)fixed_i32(l.z * s);
    acc.v[3] += (uint32_t)fixed_i32(a.x * s);
    acc.v[4] += (uint32_t)fixed_i32(a.y * s);
    acc.v[5] += (uint32_t)fixed_i32(a.z * s);
}
__device__ __forceinline__ void mdelta_flush(int32_t* deltas, uint32_t body, const MDelta& acc) {
    int32_t* d = deltas + 6ull * body;
#pragma unroll
    for (int c = 0; c < 6; ++c)
        if (acc.v[c]) atomicAdd(d + c, (int32_t)acc.v[c]);
}

__device__ __forceinline__ void add_mdelta(int32_t* deltas, uint32_t body, f3 l, f3 a) {   // :104-112
    const float s = 1048576.0f;
    int32_t* d = deltas + 6ull * body;
    atomicAdd(d + 0, fixed_i32(l.x * s));
    atomicAdd(d + 1, fixed_i32(l.y * s));
    atomicAdd(d + 2, fixed_i32(l.z * s));
    atomicAdd(d + 3, fixed_i32(a.x * s));
    atomicAdd(d + 4, fixed_i32(a.y * s));
    atomicAdd(d + 5, fixed_i32(a.z * s));
}

__device__ __forceinline__ void hinge_tangents(const StepBuffers& b, uint32_t a, uint32_t c, const GpuBearing& br,
                                               f3& ta, f3& tb) {
    const f3 axa = normalize(quat_rotate(b.rot[a], r3(br.local_axis_a)));
    const f3 axb = normalize(quat_rotate(b.rot[c], r3(br.local_axis_b)));
    const f3 hinge = normalize(axa + axb);
    const f3 helper = fabsf(hinge.x) > 0.8f ? mkf3(0, 1, 0) : mkf3(1, 0, 0);
    ta = normalize(cross(hinge, helper));
    tb = cross(hinge, ta);
}

// The parts of a bearing's five rows that depend on the poses only: they stay
// fixed over a set of projection passes (the poses change at the forward
// kinematics, not between passes), so they are computed once per set, with the
// same expressions as the rows would compute them.  9 float4 per bearing:
// {arm_a, 1/m_a} {arm_b, 1/m_b} {den0, den1, den2, -} {t_a, den3} {t_b, den4}
// {I_a t_a} {I_b t_a} {I_a t_b} {I_b t_b}: arms of the three linear rows (world
// axes), hinge tangents of the two angular rows, world inverse inertia products
// and the rows' denominators.
__global__ void __launch_bounds__(kMBlock) k_bearing_cache(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.bearing_count) return;
    const GpuBearing br = m.bearings[j];
    const uint32_t a = br.metadata[0], c = br.metadata[1];
    const f3 arm_a = quat_rotate(b.rot[a], r3(br.local_anchor_a)), arm_b = quat_rotate(b.rot[c], r3(br.local_anchor_b));
    const float ima = inv_mass(b, a), imb = inv_mass(b, c);
    float den[5];
#pragma unroll
    for (uint32_t row = 0; row < 3; ++row) {
        const f3 d = row == 0 ? mkf3(1, 0, 0) : row == 1 ? mkf3(0, 1, 0) : mkf3(0, 0, 1);
        const f3 ang_a = cross(arm_a, d), ang_b = cross(arm_b, d);
        den[row] = ima + imb + dot(ang_a, wii(b, a, ang_a)) + dot(ang_b, wii(b, c, ang_b));
    }
    f3 ta, tb;
    hinge_tangents(b, a, c, br, ta, tb);
    const f3 ia3 = wii(b, a, ta), ib3 = wii(b, c, ta), ia4 = wii(b, a, tb), ib4 = wii(b, c, tb);
    den[3] = dot(ta, ia3 + ib3);
    den[4] = dot(tb, ia4 + ib4);
    float4* o = m.bear_cache + (uint64_t)kBearingCache * j;
    o[0] = f4(arm_a, ima);
    o[1] = f4(arm_b, imb);
    o[2] = make_float4(den[0], den[1], den[2], 0.0f);
    o[3] = f4(ta, den[3]);
    o[4] = f4(tb, den[4]);
    o[5] = f4(ia3, 0.0f);
    o[6] = f4(ib3, 0.0f);
    o[7] = f4(ia4, 0.0f);
    o[8] = f4(ib4, 0.0f);
}

// articulated.wgsl:114-155, 287-316
// One bearing per group of kRowLanes lanes, one row per lane (three linear,
// two angular); the rows' fixed-point deltas are summed over the group by
// shuffles (integer sums: the same totals in any order) and one lane flushes
// them.  Every row reads the velocities of before the pass (Jacobi); the
// pose-only parts come from the set's bearing cache.
constexpr uint32_t kRowLanes = 8;
__global__ void __launch_bounds__(kMBlock) k_project_bearings(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = g / kRowLanes, row = g % kRowLanes;
    const bool live = j < p.bearing_count;   // whole groups share this (the grid covers whole groups)
    MDelta da{}, dc{};
    uint32_t a = 0, c = 0;
    if (live) {
        const uint4 meta = *reinterpret_cast<const uint4*>(m.bearings[j].metadata);
        a = meta.x;
        c = meta.y;
        const float4* cache = m.bear_cache + (uint64_t)kBearingCache * j;
        if (row < 3) {
            const float4 ca = __ldg(cache), cb = __ldg(cache + 1), cd = __ldg(cache + 2);
            const f3 arm_a = xyz(ca), arm_b = xyz(cb);
            const f3 va = xyz(b.lin[a]) + cross(xyz(b.ang[a]), arm_a);
            const f3 vb = xyz(b.lin[c]) + cross(xyz(b.ang[c]), arm_b);
            const f3 rel = vb - va;
            const float ima = ca.w, imb = cb.w;
            const f3 d = row == 0 ? mkf3(1, 0, 0) : row == 1 ? mkf3(0, 1, 0) : mkf3(0, 0, 1);
            const float den = row == 0 ? cd.x : row == 1 ? cd.y : cd.z;
            if (!(den <= 1.0e-12f)) {
                const f3 imp = d * (0.5f * dot(rel, d) / den);
                mdelta_add(da, imp * ima, wii(b, a, cross(arm_a, imp)));
                mdelta_add(dc, -imp * imb, wii(b, c, cross(arm_b, -imp)));
            }
        } else if (row < 5) {
            const float4 ax = __ldg(cache + row);   // {t_a, den3} or {t_b, den4}
            const f3 ia = xyz(__ldg(cache + (row == 3 ? 5 : 7))), ib = xyz(__ldg(cache + (row == 3 ? 6 : 8)));
            const f3 rang = xyz(b.ang[c]) - xyz(b.ang[a]);
            const f3 axis = xyz(ax);
            const float den = ax.w;
            if (!(den <= 1.0e-12f)) {
                const float imp = 0.5f * dot(rang, axis) / den;
                mdelta_add(da, mkf3(0, 0, 0), ia * imp);
                mdelta_add(dc, mkf3(0, 0, 0), -ib * imp);
            }
        }
    }
#pragma unroll
    for (uint32_t o = kRowLanes / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            da.v[q] += __shfl_down_sync(0xffffffffu, da.v[q], o, kRowLanes);
            dc.v[q] += __shfl_down_sync(0xffffffffu, dc.v[q], o, kRowLanes);
        }
    }
    if (live && row == 0) {
        mdelta_flush(m.deltas, a, da);
        mdelta_flush(m.deltas, c, dc);
    }
}

// articulated.wgsl:318-337
__global__ void __launch_bounds__(kMBlock) k_apply_mdeltas(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.body_count) return;
    int2* d2 = reinterpret_cast<int2*>(m.deltas + 6ull * i);
    const int2 x0 = d2[0], x1 = d2[1], x2 = d2[2];
    if ((x0.x | x0.y | x1.x | x1.y | x2.x | x2.y) == 0) {
        // most bodies have no bearing: their apply changes no bit unless a
        // velocity holds -0.0 or NaN, so only those are written
        if (zero_apply_is_identity(b.lin[i]) && zero_apply_is_identity(b.ang[i])) return;
    } else {
        d2[0] = make_int2(0, 0);
        d2[1] = make_int2(0, 0);
        d2[2] = make_int2(0, 0);
    }
    const float s = 1048576.0f;
    const f3 ld = mkf3((float)x0.x, (float)x0.y, (float)x1.x) / s;
    const f3 ad = mkf3((float)x1.y, (float)x2.x, (float)x2.y) / s;
    b.lin[i] = f4(xyz(b.lin[i]) + ld, 0.0f);
    b.ang[i] = f4(xyz(b.ang[i]) + ad, 0.0f);
}

// articulated.wgsl:157-285: forward then backward sweeps with immediate updates.
__device__ void project_row_immediate(const StepBuffers& b, const MechBuffers& m, uint32_t j) {
    const GpuBearing br = m.bearings[j];
    const uint32_t a = br.metadata[0], c = br.metadata[1];
    const f3 arm_a = quat_rotate(b.rot[a], r3(br.local_anchor_a)), arm_b = quat_rotate(b.rot[c], r3(br.local_anchor_b));
    const float ima = inv_mass(b, a), imb = inv_mass(b, c);
    const f3 dirs[3] = {mkf3(1, 0, 0), mkf3(0, 1, 0), mkf3(0, 0, 1)};
    for (int k = 0; k < 3; ++k) {
        const f3 va = xyz(b.lin[a]) + cross(xyz(b.ang[a]), arm_a);
        const f3 vb = xyz(b.lin[c]) + cross(xyz(b.ang[c]), arm_b);
        const f3 rel = vb - va, d = dirs[k];
        const f3 ang_a = cross(arm_a, d), ang_b = cross(arm_b, d);
        const float den = ima + imb + dot(ang_a, wii(b, a, ang_a)) + dot(ang_b, wii(b, c, ang_b));
        if (den <= 1.0e-12f) continue;
        const f3 imp = d * (dot(rel, d) / den);
        b.lin[a] = f4(xyz(b.lin[a]) + imp * ima, 0.0f);
        b.ang[a] = f4(xyz(b.ang[a]) + wii(b, a, cross(arm_a, imp)), 0.0f);
        b.lin[c] = f4(xyz(b.lin[c]) - imp * imb, 0.0f);
        b.ang[c] = f4(xyz(b.ang[c]) + wii(b, c, cross(arm_b, -imp)), 0.0f);
    }
    f3 ta, tb;
    hinge_tangents(b, a, c, br, ta, tb);
    const f3 tangents[2] = {ta, tb};
    for (int k = 0; k < 2; ++k) {
        const f3 rang = xyz(b.ang[c]) - xyz(b.ang[a]);
        const f3 axis = tangents[k];
        const f3 ia = wii(b, a, axis), ib = wii(b, c, axis);
        const float den = dot(axis, ia + ib);
        if (den <= 1.0e-12f) continue;
        const float imp = dot(rang, axis) / den;
        b.ang[a] = f4(xyz(b.ang[a]) + ia * imp, 0.0f);
        b.ang[c] = f4(xyz(b.ang[c]) - ib * imp, 0.0f);
    }
}

// Dispatched through indirect args that are zero without active contacts
// (collision.wgsl:747-749, device.rs:1101-1110).
__global__ void k_project_bearings_serial(StepBuffers b, MechBuffers m, MechParams p) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (b.counts->active == 0u) return;
    for (uint32_t j = 0; j < p.bearing_count; ++j) project_row_immediate(b, m, j);
    for (uint32_t j = p.bearing_count; j > 0; --j) project_row_immediate(b, m, j - 1);
}

// articulated.wgsl:339-364
__device__ __forceinline__ f3 permitted_axis(const StepBuffers& b, const MechBuffers& m, uint32_t body) {
    const GpuMechanismBody mb = m.bodies[body];
    const uint32_t parent = mb.metadata[0];
    const GpuBearing& br = m.bearings[mb.metadata[1]];
    f3 axis = normalize(quat_rotate(b.rot[parent], r3(br.local_axis_a)));
    if (mb.metadata[2] != 0u) axis = -normalize(quat_rotate(b.rot[parent], r3(br.local_axis_b)));
    return axis;
}
__device__ __forceinline__ float permitted_speed(const StepBuffers& b, const MechBuffers& m, uint32_t body) {
    const uint32_t parent = m.bodies[body].metadata[0];
    return dot(xyz(b.ang[body]) - xyz(b.ang[parent]), permitted_axis(b, m, body));
}
__device__ __forceinline__ float stabilized_speed(const StepBuffers& b, const MechBuffers& m, uint32_t body,
                                                  float speed) {
    const bool aligned = fabsf(permitted_axis(b, m, body).y) > 0.999f;
    return (aligned && fabsf(speed) < 0.005f) ? 0.0f : speed;
}

// articulated.wgsl:366-415
__global__ void __launch_bounds__(kMBlock) k_advance_coordinates(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body >= p.body_count || m.bodies[body].metadata[3] != 0u) return;
    const uint32_t c = m.bearings[m.bodies[body].metadata[1]].metadata[2];
    if (c == kInvalid) return;
    const float measured = permitted_speed(b, m, body) * p.ang_damp;
    const GpuMechanismDrive dr = m.drives[c];
    float speed = 0.0f;
    if (dr.mode == MK_DRIVE_MODE_PASSIVE) {
        speed = stabilized_speed(b, m, body, measured);
    } else {
        float desired = clampf(dr.target_speed, -dr.max_speed, dr.max_speed);
        if (dr.mode == MK_DRIVE_MODE_ANGLE) {
            const float err = dr.target_angle - m.coords[c].angle;
            const float brake = sqrtf(2.0f * dr.max_acceleration * fabsf(err));
            desired = sgnf(err) * mnf(brake, dr.max_speed);
            if (fabsf(err) < 0.0005f) desired = 0.0f;
        }
        const float budget = dr.max_acceleration * p.dt;
        speed = measured + clampf(desired - measured, -budget, budget);
    }
    float angle = m.coords[c].angle + speed * p.dt;
    if (angle < dr.min_angle) {
        angle = dr.min_angle;
        speed = 0.0f;
    } else if (angle > dr.max_angle) {
        angle = dr.max_angle;
        speed = 0.0f;
    }
    m.coords[c].angular_velocity = speed;
    m.coords[c].angle = angle;
}

// articulated.wgsl:417-429
__global__ void __launch_bounds__(kMBlock) k_capture_coordinates(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body >= p.body_count || m.bodies[body].metadata[3] != 0u) return;
    const uint32_t c = m.bearings[m.bodies[body].metadata[1]].metadata[2];
    if (c != kInvalid) m.coords[c].angular_velocity = stabilized_speed(b, m, body, permitted_speed(b, m, body));
}

// ------------------------------------------------------ forward kinematics
struct Link { float4 pos, rot; uint4 meta; };
__device__ __forceinline__ Link ld_link(const GpuLinkState* L, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(L + i);
    const float4 m = p[2];
    return {p[0], p[1], make_uint4(__float_as_uint(m.x), __float_as_uint(m.y), __float_as_uint(m.z), __float_as_uint(m.w))};
}
__device__ __forceinline__ void st_link(GpuLinkState* L, uint32_t i, const Link& v) {
    float4* p = reinterpret_cast<float4*>(L + i);
    p[0] = v.pos;
    p[1] = v.rot;
    p[2] = make_float4(__uint_as_float(v.meta.x), __uint_as_float(v.meta.y), __uint_as_float(v.meta.z),
                       __uint_as_float(v.meta.w));
}

// mechanism.wgsl:67-70
__device__ __forceinline__ float4 axis_rotation(f3 axis, float angle) {
    const float h = angle * 0.5f;
    const f3 v = normalize(axis) * sin_cr(h);
    return make_float4(v.x, v.y, v.z, cos_cr(h));
}

// mechanism.wgsl:72-108
__device__ __forceinline__ void prepare_link(const MechBuffers& m, uint32_t body) {
    const GpuMechanismBody mb = m.bodies[body];
    if (mb.metadata[3] != 0u) {
        st_link(m.links_a, body, {make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 1), make_uint4(body, 1, 0, 0)});
        return;
    }
    const GpuBearing& br = m.bearings[mb.metadata[1]];
    const float angle = m.coords[br.metadata[2]].angle;
    const float4 bind = r4(mb.bind_relative_rotation);
    float4 rr;
    f3 rp;
    if (mb.metadata[2] == 0u) {
        rr = quat_multiply(axis_rotation(r3(br.local_axis_a), angle), bind);
        rp = r3(br.local_anchor_a) - quat_rotate(rr, r3(br.local_anchor_b));
    } else {
        rr = quat_multiply(axis_rotation(r3(br.local_axis_b), -angle), bind);
        rp = r3(br.local_anchor_b) - quat_rotate(rr, r3(br.local_anchor_a));
    }
    st_link(m.links_a, body, {f4(rp, 0.0f), rr, make_uint4(mb.metadata[0], 0, 0, 0)});
}

// mechanism.wgsl:110-149
__device__ __forceinline__ void jump_link(const GpuLinkState* src, GpuLinkState* dst, uint32_t body) {
    const Link child = ld_link(src, body);
    if (child.meta.y != 0u) {
        st_link(dst, body, child);
        return;
    }
    const Link par = ld_link(src, child.meta.x);
    Link r;
    r.pos = f4(xyz(par.pos) + quat_rotate(par.rot, xyz(child.pos)), 0.0f);
    r.rot = normalize4(quat_multiply(par.rot, child.rot));
    r.meta = make_uint4(par.meta.x, par.meta.y, 0, 0);
    st_link(dst, body, r);
}

__global__ void __launch_bounds__(kMBlock) k_prepare_links(MechBuffers m, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body < p.body_count) prepare_link(m, body);
}
__global__ void __launch_bounds__(kMBlock) k_jump(const GpuLinkState* src, GpuLinkState* dst, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body < p.body_count) jump_link(src, dst, body);
}

// mechanism.wgsl:151-185
__global__ void __launch_bounds__(kMBlock) k_publish(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body >= p.body_count) return;
    const Link L = ld_link(m.links_final, body);
    const uint32_t root = L.meta.x;
    if (body == root) return;
    const float4 rq = b.rot[root];
    b.pos[body] = f4(xyz(b.pos[root]) + quat_rotate(rq, xyz(L.pos)), 0.0f);
    b.rot[body] = normalize4(quat_multiply(rq, L.rot));
}

// articulated.wgsl:431-456 for the bodies of one depth level.
__global__ void __launch_bounds__(kMBlock) k_reconstruct_level(StepBuffers b, MechBuffers m, uint32_t begin,
                                                               uint32_t end) {
    const uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= end) return;
    const uint32_t body = m.level_bodies[t];
    const GpuMechanismBody mb = m.bodies[body];
    const uint32_t parent = mb.metadata[0];
    const GpuBearing& br = m.bearings[mb.metadata[1]];
    const float4 rp = b.rot[parent], rb = b.rot[body];
    f3 axis = normalize(quat_rotate(rp, r3(br.local_axis_a)));
    f3 pa = quat_rotate(rp, r3(br.local_anchor_a));
    f3 ca = quat_rotate(rb, r3(br.local_anchor_b));
    if (mb.metadata[2] != 0u) {
        axis = -normalize(quat_rotate(rp, r3(br.local_axis_b)));
        pa = quat_rotate(rp, r3(br.local_anchor_b));
        ca = quat_rotate(rb, r3(br.local_anchor_a));
    }
    const float speed = m.coords[br.metadata[2]].angular_velocity;
    const f3 wp = xyz(b.ang[parent]);
    const f3 angular = wp + axis * speed;
    const f3 av = xyz(b.lin[parent]) + cross(wp, pa);
    b.lin[body] = f4(av - cross(angular, ca), 0.0f);
    b.ang[body] = f4(angular, 0.0f);
}

// articulated.wgsl:458-484
__global__ void __launch_bounds__(kMBlock) k_validate_state(StepBuffers b, MechBuffers m, MechParams p) {
    const uint32_t body = blockIdx.x * blockDim.x + threadIdx.x;
    if (body >= p.body_count) return;
    const float4 q = b.rot[body];
    const float rl = dot4(q, q);
    bool valid = finite4(b.pos[body]) && finite4(q) && finite4(b.lin[body]) && finite4(b.ang[body]) && rl > 0.5f &&
                 rl < 1.5f;
    const GpuMechanismBody mb = m.bodies[body];
    if (mb.metadata[3] == 0u) {
        const GpuMechanismCoordinate st = m.coords[m.bearings[mb.metadata[1]].metadata[2]];
        valid = valid && st.angle == st.angle && fabsf(st.angle) < kFloatMax && st.angular_velocity == st.angular_velocity &&
                fabsf(st.angular_velocity) < kFloatMax;
    }
    if (!valid) atomicOr(&b.diag->error_flags, MK_INVALID_NUMERIC_FLAG);
}

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
        const Link la = ld_link(links, a), lc = ld_link(links, c);
        pa = la.pos; qa = la.rot; pc = lc.pos; qc = lc.rot;
    } else {
        pa = pos[a]; qa = rot[a]; pc = pos[c]; qc = rot[c];
    }
    const f3 anchor_a = xyz(pa) + quat_rotate(qa, r3(br.local_anchor_a));
    const f3 anchor_b = xyz(pc) + quat_rotate(qc, r3(br.local_anchor_b));
    const f3 axis_a = normalize(quat_rotate(qa, r3(br.local_axis_a)));
    const f3 axis_b = normalize(quat_rotate(qc, r3(br.local_axis_b)));
    record_residual(diag, anchor_a, anchor_b, axis_a, axis_b, br.metadata[3] != 0u);
}

// ------------------------------------------------------------- closure loop
__device__ __forceinline__ float block_sum(float v, float* scratch) {
    // fixed tree order: warp shuffles, then warp 0 over the warp partials
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    __syncthreads();
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    float r = 0.0f;
    if (w == 0) {
        r = lane < (blockDim.x >> 5) ? scratch[lane] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (lane == 0) scratch[32] = r;
    }
    __syncthreads();
    return scratch[32];
}

// Dot products over the closure coordinates.  Up to kSerialDot coordinates
// one thread sums them in ascending coordinate order (the serial order of
// closure.wgsl:339-414, so small systems reproduce it bit for bit).  Larger
// systems sum per chunk of 1,024 coordinates: thread t of the chunk's block
// holds coordinate 1024 c + t, the block tree sums the chunk, and the chunk
// sums are added in chunk order -- the same result whether one block or the
// whole grid walks the chunks.
constexpr uint32_t kSerialDot = 512;
constexpr uint32_t kDotChunk = kClosureThreads;

// Sync of the closure loop: the block, or the whole cooperative grid.
template <bool kGrid>
__device__ __forceinline__ void loop_sync(uint32_t* barrier, uint32_t* error_flags) {
    if (kGrid) grid_barrier(barrier, error_flags, gridDim.x);
    else __syncthreads();
}

// Sums of the slot values of the closure coordinates whose runs are longer than
// kLongList slots (near the root of a large loop lattice a coordinate lies on a
// branch of nearly every closure: up to 176k slots).  Such a run is summed in two
// levels, so that no thread adds it alone: each chunk of kLongList consecutive
// slots serially, in parallel over the chunks, then the chunk sums serially in
// chunk order.  Runs of up to kLongList slots keep the one serial sum.  The
// accumulation order of the reference (CAS float atomics, closure.wgsl:128-192) is
// a race, so any fixed order is as faithful; the oracle restates this one.
// kEval: evaluation sums (a NaN gradient marks a slot without contribution, the
// diagonal summed beside it) into out_g / out_d; else plain sums into out_g.
template <bool kGrid, bool kEval>
__device__ void gather_long_runs(const MechBuffers& m, const MechParams& p, float* out_g, float* out_d,
                                 uint32_t* flags) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    for (uint32_t c = tid; c < p.long_chunks; c += nt) {
        const uint32_t w = m.chunk_long[c];
        const uint32_t q = m.long_q[w];
        const uint32_t begin = m.cq_off[q] + kLongList * (c - m.long_chunk_off[w]);
        const uint32_t end = min(begin + kLongList, m.cq_off[q + 1]);
        float g = 0.0f, d = 0.0f;
#pragma unroll 8
        for (uint32_t i = begin; i < end; ++i) {
            const float sg = __ldcg(m.slot_g + i);
            if (kEval) {
                if (sg == sg) { g += sg; d += __ldcg(m.slot_d + i); }
            } else {
                g += sg;
            }
        }
        m.chunk_g[c] = g;
        if (kEval) m.chunk_d[c] = d;
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    for (uint32_t w = tid; w < p.long_coords; w += nt) {
        float g = 0.0f, d = 0.0f;
        for (uint32_t c = m.long_chunk_off[w]; c < m.long_chunk_off[w + 1]; ++c) {
            g += __ldcg(m.chunk_g + c);
            if (kEval) d += __ldcg(m.chunk_d + c);
        }
        const uint32_t cc = m.cq_coords[m.long_q[w]];
        out_g[cc] = g;
        if (kEval) out_d[cc] = d;
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
}

// The chunked dot: `part` is this thread's term for the coordinate of chunk
// `c` it holds (0 when none); the block tree sum of the chunk goes to
// chunk_part[c].  Call for every chunk the block walks, all threads together.
__device__ __forceinline__ void chunk_dot(float part, float* chunk_part, uint32_t c, float* scratch) {
    const float s = block_sum(part, scratch);
    if (threadIdx.x == 0) chunk_part[c] = s;
}

// The total after a loop_sync: serial over the coordinates (small systems) or
// the chunk sums in chunk order, computed by thread 0 of every block and
// shared through scratch[32].
__device__ __forceinline__ float dot_total(uint32_t nq, const MechBuffers& m, const float* a, const float* bvec,
                                           const float* chunk_part, float* scratch) {
    if (threadIdx.x == 0) {
        float acc = 0.0f;
        if (nq <= kSerialDot) {
            for (uint32_t q = 0; q < nq; ++q) {
                const uint32_t c = m.cq_coords[q];
                acc += a[c] * bvec[c];
            }
        } else {
            const uint32_t chunks = (nq + kDotChunk - 1) / kDotChunk;
            for (uint32_t c = 0; c < chunks; ++c) acc += chunk_part[c];
        }
        scratch[32] = acc;
    }
    __syncthreads();
    const float r = scratch[32];
    __syncthreads();
    return r;
}

// slot_g[sl] = the slot's share of J^T J x: per closure the branch products
// (sums over its slots in slot order, branch a then b) and their transposes,
// from the stored Jacobian columns; closures strided over the block or grid.
__device__ __forceinline__ bool long_run(const MechBuffers& m, uint32_t q) { return m.cq_off[q + 1] - m.cq_off[q] > kLongList; }

__device__ __forceinline__ void closure_products(const MechBuffers& m, const MechParams& p, const float* x) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    for (uint32_t k = tid; k < p.closures; k += nt) {
        const uint32_t s0 = m.cl_slot_off[k], s1 = m.cl_slot_off[k + 1], split = m.cl_split[k];
        // branch a's and branch b's sums in registers (no indexed array), unrolled so
        // the columns' loads issue together; each sum keeps slot order
        f3 pp_a = mkf3(0, 0, 0), pa_a = mkf3(0, 0, 0), pp_b = mkf3(0, 0, 0), pa_b = mkf3(0, 0, 0);
#pragma unroll 4
        for (uint32_t sl = s0; sl < s1; ++sl) {
            const f3 pd = xyz(m.slot_v[2 * sl]), ad = xyz(m.slot_v[2 * sl + 1]);
            const float dv = x[__float_as_uint(m.slot_v[2 * sl].w)];
            const f3 tp = pd * dv, ta = ad * dv;
            if (sl < split) {
                pp_a = pp_a + tp;
                pa_a = pa_a + ta;
            } else {
                pp_b = pp_b + tp;
                pa_b = pa_b + ta;
            }
        }
        const f3 pp = pp_a + pp_b, pa = pa_a + pa_b;
#pragma unroll 4
        for (uint32_t sl = s0; sl < s1; ++sl)
            m.slot_g[m.slot_pos[sl]] = dot(xyz(m.slot_v[2 * sl]), pp) + 1.0f * dot(xyz(m.slot_v[2 * sl + 1]), pa);
    }
}

// Joint frame of `body` in its root's frame (closure.wgsl:168-181).
__device__ __forceinline__ void joint_frame(const MechBuffers& m, uint32_t body, f3& axis, f3& anchor, uint32_t& coord) {
    const GpuMechanismBody mb = m.bodies[body];
    const GpuBearing& tb = m.bearings[mb.metadata[1]];
    const Link pp = ld_link(m.links_final, mb.metadata[0]);
    if (mb.metadata[2] == 0u) {
        axis = normalize(quat_rotate(pp.rot, r3(tb.local_axis_a)));
        anchor = xyz(pp.pos) + quat_rotate(pp.rot, r3(tb.local_anchor_a));
    } else {
        axis = -normalize(quat_rotate(pp.rot, r3(tb.local_axis_b)));
        anchor = xyz(pp.pos) + quat_rotate(pp.rot, r3(tb.local_anchor_b));
    }
    coord = tb.metadata[2];
}

__device__ __forceinline__ void closure_frames(const MechBuffers& m, const GpuBearing& br, f3& anc_a, f3& anc_b,
                                               f3& ax_a, f3& ax_b) {
    const Link pa = ld_link(m.links_final, br.metadata[0]), pb = ld_link(m.links_final, br.metadata[1]);
    anc_a = xyz(pa.pos) + quat_rotate(pa.rot, r3(br.local_anchor_a));
    anc_b = xyz(pb.pos) + quat_rotate(pb.rot, r3(br.local_anchor_b));
    ax_a = normalize(quat_rotate(pa.rot, r3(br.local_axis_a)));
    ax_b = normalize(quat_rotate(pb.rot, r3(br.local_axis_b)));
}

__device__ __forceinline__ bool finite3(f3 v) {
    return v.x == v.x && v.y == v.y && v.z == v.z && fabsf(v.x) < kFloatMax && fabsf(v.y) < kFloatMax &&
           fabsf(v.z) < kFloatMax;
}

// The closure loop of device.rs:973-1020: 12 Newton steps of
// closure.wgsl:268-427 (evaluate, finalize, 8-round diagonal PCG, step the
// coordinates), each followed by forward kinematics of the closure
// components.  Accumulations go through per-joint slots summed per
// coordinate in the serial order; dot products as above.  kGrid = false runs
// it in one block (few closures: block syncs are nearly free); kGrid = true
// spreads closures, coordinate chunks and bodies over a cooperative grid with
// grid barriers in place of the block syncs (thousands of closures).  Both
// compute the same values.
// evaluate_closures (closure.wgsl:268-319) for closure k: its residual against the
// tolerance (lane 0 of the walkers records the step's maxima), then the slots
// first + i * step of its branches: the joint's Jacobian column and the slot's
// gradient and diagonal contributions (NaN: none).  With step 32 a warp walks
// one closure; every slot's arithmetic is the same whoever computes it.
__device__ __forceinline__ void evaluate_closure(const MechBuffers& m, uint32_t k, uint32_t* st, uint32_t* flags,
                                                 uint32_t Q, uint32_t first, uint32_t step) {
    const GpuBearing br = m.bearings[m.cl_bearings[k]];
    f3 aa, ab, xa, xb;
    closure_frames(m, br, aa, ab, xa, xb);
    const f3 rp = aa - ab, ra = xa - xb;
    const uint32_t s0 = m.cl_slot_off[k], s1 = m.cl_slot_off[k + 1], split = m.cl_split[k];
    bool active = true;
    if (!finite3(rp) || !finite3(ra)) {
        if (first == 0) {
            atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
            atomicMax(&st[0], 0xffffffffu);
            atomicMax(&st[1], 0xffffffffu);
        }
        active = false;
    } else {
        const uint32_t um = round_u32(length(rp) * 1000000.0f);
        // axis error as atan2(|a x b|, a . b): FP32 acos (closure.wgsl:295) reads 0
        // below ~3.5e-4 rad, blind to the 1000 micro-degree tolerance
        const float deg = atan2_cr(length(cross(xa, xb)), clampf(dot(xa, xb), -1.0f, 1.0f)) * 57.295779513f;
        const uint32_t ud = round_u32(deg * 1000000.0f);
        if (first == 0) {
            atomicMax(&st[0], um);
            atomicMax(&st[1], ud);
        }
        active = !(um <= 10u && ud <= 1000u);
    }
    for (uint32_t sl = s0 + first; sl < s1; sl += step) {
        float g = 0.0f, d = 0.0f;
        uint32_t valid = 0;
        // the slot's Jacobian column: the links do not move during the
        // step's PCG rounds, so closure.wgsl:194-266's recomputation in
        // every round gives these same floats (sign * v == v * sign)
        const bool side_a = sl < split;
        const f3 ea = side_a ? aa : ab, ex = side_a ? xa : xb;
        const float sign = side_a ? 1.0f : -1.0f;
        f3 axis, anchor;
        uint32_t coord;
        joint_frame(m, m.slot_body[sl], axis, anchor, coord);
        const f3 pd = cross(axis, ea - anchor) * sign;
        const f3 ad = cross(axis, ex) * sign;
        m.slot_v[2 * sl] = f4(pd, __uint_as_float(coord < Q ? coord : 0u));
        m.slot_v[2 * sl + 1] = f4(ad, 0.0f);
        if (active) {
            if (coord >= Q) {
                atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
            } else {
                g = dot(rp, pd) + 1.0f * dot(ra, ad);
                d = dot(pd, pd) + 1.0f * dot(ad, ad);
                if (g == g && d == d) valid = 1;
                else atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
            }
        }
        // NaN marks "no contribution" so the gather skips it
        m.slot_g[m.slot_pos[sl]] = valid ? g : __int_as_float(0x7fffffff);
        m.slot_d[m.slot_pos[sl]] = valid ? d : 0.0f;
    }
}

template <bool kGrid>
__global__ void __launch_bounds__(kClosureThreads) k_closure_loop(StepBuffers b, MechBuffers m, MechParams p) {
    __shared__ float s_red[33];
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gnt = gridDim.x * blockDim.x;
    const uint32_t NC = p.closures, NQ = p.closure_coords, NB = p.closure_bodies, Q = p.coordinate_count;
    const uint32_t chunks = (NQ + kDotChunk - 1) / kDotChunk;
    float* sol = m.pcg;
    float* res = m.pcg + Q;
    float* pre = m.pcg + 2ull * Q;
    float* dir = m.pcg + 3ull * Q;
    float* op = m.pcg + 4ull * Q;
    uint32_t* flags = &b.diag->error_flags;
    // per-step residual maxima (zeroed at the start of the tick) and chunk sums
    uint32_t* state = m.loop_state;
    float* part_a = m.chunk_part;
    float* part_b = m.chunk_part + chunks;
    bool converged_prev = false;
    uint32_t steps = 0, rounds = 0;
    for (uint32_t step = 0; step < kClosureSteps; ++step) {
        uint32_t* st = state + 2 * step;
        const bool evaluate = step == 0 || !converged_prev;
        // evaluate_closures (closure.wgsl:268-319): slot contributions
        if (evaluate) {
            if (p.wide_closures) {   // a warp per closure, its slots spread over the lanes
                const uint32_t lane = threadIdx.x & 31u;
                for (uint32_t k = gtid >> 5; k < NC; k += gnt >> 5) evaluate_closure(m, k, st, flags, Q, lane, 32u);
            } else {
                for (uint32_t k = gtid; k < NC; k += gnt) evaluate_closure(m, k, st, flags, Q, 0u, 1u);
            }
        }
        loop_sync<kGrid>(m.grid_barrier, flags);
        const bool unconverged = ld_relaxed_u32(&st[0]) > 10u || ld_relaxed_u32(&st[1]) > 1000u;
        if (unconverged) ++steps;
        if (evaluate && p.long_coords) gather_long_runs<kGrid, true>(m, p, m.grad, m.diag, flags);   // long runs first
        // gather per coordinate in the serial accumulation order, then the PCG's
        // initial vectors (solve_closure_pcg, closure.wgsl:333-427), chunk by chunk
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint32_t q = c * kDotChunk + threadIdx.x;
            float part = 0.0f;
            if (q < NQ) {
                float g = 0.0f, d = 0.0f;
                if (evaluate && long_run(m, q)) {
                    g = m.grad[m.cq_coords[q]];
                    d = m.diag[m.cq_coords[q]];
                } else if (evaluate) {
                    for (uint32_t i = m.cq_off[q]; i < m.cq_off[q + 1]; ++i) {
                        const float sg = m.slot_g[i];
                        if (sg == sg) { g += sg; d += m.slot_d[i]; }
                    }
                }
                const uint32_t cc = m.cq_coords[q];
                m.grad[cc] = g;
                m.diag[cc] = d;
                if (unconverged) {
                    float r = 0.0f, z = 0.0f;
                    if (d > 1.0e-12f) { r = -g; z = r / d; }
                    sol[cc] = 0.0f; res[cc] = r; pre[cc] = z; dir[cc] = z; op[cc] = 0.0f;
                    part = r * z;
                }
            }
            if (unconverged && NQ > kSerialDot) chunk_dot(part, part_a, c, s_red);
        }
        if (unconverged) {
            loop_sync<kGrid>(m.grid_barrier, flags);
            float rz = dot_total(NQ, m, res, pre, part_a, s_red);
            for (uint32_t round = 0; round < kClosureRounds; ++round) {
                // J^T J dir per closure: branch products then transposes
                // (closure.wgsl:194-266), from the step's stored columns
                closure_products(m, p, dir);
                loop_sync<kGrid>(m.grid_barrier, flags);
                if (p.long_coords) gather_long_runs<kGrid, false>(m, p, op, nullptr, flags);
                for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
                    const uint32_t q = c * kDotChunk + threadIdx.x;
                    float dpart = 0.0f;
                    if (q < NQ) {
                        float o = 0.0f;
                        if (long_run(m, q)) o = op[m.cq_coords[q]];
                        else
                            for (uint32_t i = m.cq_off[q]; i < m.cq_off[q + 1]; ++i) o += m.slot_g[i];
                        const uint32_t cc = m.cq_coords[q];
                        op[cc] = o;
                        dpart = dir[cc] * o;
                    }
                    if (NQ > kSerialDot) chunk_dot(dpart, part_b, c, s_red);
                }
                loop_sync<kGrid>(m.grid_barrier, flags);
                const float dop = dot_total(NQ, m, dir, op, part_b, s_red);
                const float alpha = fabsf(dop) > 1.0e-20f ? rz / dop : 0.0f;
                for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
                    const uint32_t q = c * kDotChunk + threadIdx.x;
                    float npart = 0.0f;
                    if (q < NQ) {
                        const uint32_t cc = m.cq_coords[q];
                        sol[cc] += alpha * dir[cc];
                        res[cc] -= alpha * op[cc];
                        const float d = m.diag[cc];
                        pre[cc] = 0.0f;
                        if (d > 1.0e-12f) pre[cc] = res[cc] / d;
                        npart = res[cc] * pre[cc];
                    }
                    if (NQ > kSerialDot) chunk_dot(npart, part_a, c, s_red);
                }
                loop_sync<kGrid>(m.grid_barrier, flags);
                const float nrz = dot_total(NQ, m, res, pre, part_a, s_red);
                const float beta = fabsf(rz) > 1.0e-20f ? nrz / rz : 0.0f;
                for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
                    const uint32_t q = c * kDotChunk + threadIdx.x;
                    if (q < NQ) {
                        const uint32_t cc = m.cq_coords[q];
                        dir[cc] = pre[cc] + beta * dir[cc];
                    }
                }
                rz = nrz;
                ++rounds;
                loop_sync<kGrid>(m.grid_barrier, flags);
            }
            // step every coordinate (coordinates off the closure branches add 0)
            for (uint32_t c = gtid; c < Q; c += gnt) {
                const float stp = clampf(0.35f * sol[c], -0.2f, 0.2f);
                if (stp == stp) m.coords[c].angle += stp;
                else atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
            }
            loop_sync<kGrid>(m.grid_barrier, flags);
            // forward kinematics of the closure components (mechanism.wgsl:72-149)
            for (uint32_t i = gtid; i < NB; i += gnt) prepare_link(m, m.cb_bodies[i]);
            loop_sync<kGrid>(m.grid_barrier, flags);
            bool a_src = true;
            for (uint32_t r = 0; r < p.jump_rounds; ++r) {
                for (uint32_t i = gtid; i < NB; i += gnt)
                    jump_link(a_src ? m.links_a : m.links_b, a_src ? m.links_b : m.links_a, m.cb_bodies[i]);
                loop_sync<kGrid>(m.grid_barrier, flags);
                a_src = !a_src;
            }
        }
        converged_prev = !unconverged;
    }
    if (gtid == 0) {
        atomicAdd(&b.diag->reserved_b, steps);
        atomicAdd(&b.diag->reserved_c, rounds);
    }
}

// ------------------------------------------------- closure PCG to a residual
// MK_CLOSURE_PCG_RESIDUAL: each Newton step of the closure loop solves
// (J^T J) dtheta = -g by preconditioned conjugate gradients until
// ||r|| <= closure_tol * ||r0|| (or closure_max_it iterations), with
// FP64 dot products and residual check (f32 vectors), instead of the
// reference's 8 diagonal-PCG rounds.  The preconditioner is block Jacobi
// over 2 x 2 blocks of consecutive closure coordinates (a whole loop's block
// would be the exact inverse of its independent component, leaving nothing
// to precondition); with the learned preconditioner the network's corrected
// block inverse replaces a block when it is positive definite.
//
// Each Newton step is two launches (evaluate, solve) with the network in
// between; a converged step sets `done` and the later launches return.

// Fixed-order FP64 block sum (1024 threads): per-thread partials, warp
// shuffle-down trees, then the same shuffle-down tree over the 32 warp sums,
// which every warp evaluates for itself (identical operands and order, so
// identical bits) instead of warp 0 publishing it through shared memory: two
// barriers per sum instead of four.
__device__ __forceinline__ double block_sum_d(double v, double* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    __syncthreads();   // the previous sum's readers are done with scratch
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    double r = lane < (blockDim.x >> 5) ? scratch[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    return __shfl_sync(0xffffffffu, r, 0);
}

// The FP64 dot product after a loop_sync: the chunk sums in chunk order (thread
// 0 of every block), shared through scratch[32].  Chunks of 1,024 coordinates
// with one coordinate per thread: up to 1,024 coordinates this is the block
// tree of the per-thread terms, and one block or the whole grid give the same.
__device__ __forceinline__ double chunk_total_d(const double* part, uint32_t chunks, double* scratch) {
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (uint32_t c = 0; c < chunks; ++c) acc += part[c];
        scratch[32] = acc;
    }
    __syncthreads();
    const double r = scratch[32];
    __syncthreads();
    return r;
}

// out[c] = (J^T J x)[c] for the closure coordinates, from the stored columns
// (the block, or with kGrid the whole cooperative grid).
template <bool kGrid>
__device__ void closure_apply(const MechBuffers& m, const MechParams& p, const float* x, float* out,
                              uint32_t* flags) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    closure_products(m, p, x);
    loop_sync<kGrid>(m.grid_barrier, flags);
    if (p.long_coords) gather_long_runs<kGrid, false>(m, p, out, nullptr, flags);
    for (uint32_t q = tid; q < p.closure_coords; q += nt) {
        if (long_run(m, q)) continue;
        float o = 0.0f;
        for (uint32_t i = m.cq_off[q]; i < m.cq_off[q + 1]; ++i) o += m.slot_g[i];
        out[m.cq_coords[q]] = o;
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
}

// (J^T J)[i][j] for two closure coordinates (positions qi, qj in the list).
__device__ __forceinline__ float closure_coupling(const MechBuffers& m, uint32_t qi, uint32_t qj) {
    float r = 0.0f;
    for (uint32_t a = m.cq_off[qi]; a < m.cq_off[qi + 1]; ++a) {
        const uint32_t sa = m.cq_slots[a];
        for (uint32_t bq = m.cq_off[qj]; bq < m.cq_off[qj + 1]; ++bq) {
            const uint32_t sb = m.cq_slots[bq];
            if (m.slot_closure[sa] != m.slot_closure[sb]) continue;
            r += dot(xyz(m.slot_v[2 * sa]), xyz(m.slot_v[2 * sb])) +
                 1.0f * dot(xyz(m.slot_v[2 * sa + 1]), xyz(m.slot_v[2 * sb + 1]));
        }
    }
    return r;
}

template <bool kGrid>
__global__ void __launch_bounds__(kClosureThreads) k_closure_eval(StepBuffers b, MechBuffers m, MechParams p,
                                                                  uint32_t step) {
    ClosureState* cs = m.cstate;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    const uint32_t NC = p.closures, NQ = p.closure_coords, Q = p.coordinate_count;
    uint32_t* flags = &b.diag->error_flags;
    if (step == 0) {
        if (tid == 0) *cs = ClosureState{0u, 0u, 0u, 0u, 0u, 0u, 0.0};
    } else if (ld_acquire_u32(&cs->done)) {
        return;
    }
    uint32_t* s_state = m.loop_state + 2 * step;   // largest residuals of this step (zeroed per tick)
    // slot columns and their gradient / diagonal contributions (closure.wgsl:268-319)
    for (uint32_t k = tid; k < NC; k += nt) {
        const GpuBearing br = m.bearings[m.cl_bearings[k]];
        f3 aa, ab, xa, xb;
        closure_frames(m, br, aa, ab, xa, xb);
        const f3 rp = aa - ab, ra = xa - xb;
        const uint32_t s0 = m.cl_slot_off[k], s1 = m.cl_slot_off[k + 1], split = m.cl_split[k];
        bool active = true;
        if (!finite3(rp) || !finite3(ra)) {
            atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
            atomicMax(&s_state[0], 0xffffffffu);
            atomicMax(&s_state[1], 0xffffffffu);
            active = false;
        } else {
            const uint32_t um = round_u32(length(rp) * 1000000.0f);
            const float deg = atan2_cr(length(cross(xa, xb)), clampf(dot(xa, xb), -1.0f, 1.0f)) * 57.295779513f;
            const uint32_t ud = round_u32(deg * 1000000.0f);
            atomicMax(&s_state[0], um);
            atomicMax(&s_state[1], ud);
            active = !(um <= 10u && ud <= 1000u);
        }
        for (uint32_t sl = s0; sl < s1; ++sl) {
            const bool side_a = sl < split;
            const f3 ea = side_a ? aa : ab, ex = side_a ? xa : xb;
            const float sign = side_a ? 1.0f : -1.0f;
            f3 axis, anchor;
            uint32_t coord;
            joint_frame(m, m.slot_body[sl], axis, anchor, coord);
            f3 pd = mkf3(0, 0, 0), ad = mkf3(0, 0, 0);
            float g = 0.0f, d = 0.0f;
            uint32_t valid = 0;
            if (coord >= Q) {
                atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
                coord = 0;
            } else {
                pd = cross(axis, ea - anchor) * sign;
                ad = cross(axis, ex) * sign;
                if (active) {
                    g = dot(rp, pd) + 1.0f * dot(ra, ad);
                    d = dot(pd, pd) + 1.0f * dot(ad, ad);
                    if (g == g && d == d) valid = 1;
                    else atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
                }
            }
            m.slot_v[2 * sl] = f4(pd, __uint_as_float(coord));
            m.slot_v[2 * sl + 1] = f4(ad, __uint_as_float(m.slot_closure[sl]));
            m.slot_g[m.slot_pos[sl]] = valid ? g : __int_as_float(0x7fffffff);
            m.slot_d[m.slot_pos[sl]] = valid ? d : 0.0f;
        }
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    if (p.long_coords) gather_long_runs<kGrid, true>(m, p, m.grad, m.diag, flags);
    for (uint32_t q = tid; q < NQ; q += nt) {
        const uint32_t c = m.cq_coords[q];
        if (!long_run(m, q)) {
            float g = 0.0f, d = 0.0f;
            for (uint32_t i = m.cq_off[q]; i < m.cq_off[q + 1]; ++i) {
                const float sg = m.slot_g[i];
                if (sg == sg) { g += sg; d += m.slot_d[i]; }
            }
            m.grad[c] = g;
            m.diag[c] = d;
        }
        // probe vectors: ones and alternating signs over the coordinate list
        m.pcg[c] = 1.0f;
        m.pcg[Q + c] = (q & 1u) ? -1.0f : 1.0f;
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    const bool unconverged = ld_relaxed_u32(&s_state[0]) > 10u || ld_relaxed_u32(&s_state[1]) > 1000u;
    // the 2 x 2 blocks and the network's inputs, for the preconditioners that use them
    const bool pair_blocks = p.precond == MK_PRECOND_LEARNED || p.precond == MK_PRECOND_PAIR_BLOCKS;
    // A * ones and A * alternating signs (block inputs of the network)
    if (pair_blocks) closure_apply<kGrid>(m, p, m.pcg, m.probe, flags);
    if (pair_blocks) closure_apply<kGrid>(m, p, m.pcg + Q, m.probe + Q, flags);
    // block entries (a, b, d) and the plain 2 x 2 inverse
    float* blk_b = m.pcg + 2ull * Q;   // coupling of each block (free until the solve)
    for (uint32_t blk = tid; pair_blocks && blk < p.blocks; blk += nt) {
        const uint32_t qi = 2 * blk, qj = qi + 1;
        const bool pair = qj < NQ;
        const float a = m.diag[m.cq_coords[qi]], d = pair ? m.diag[m.cq_coords[qj]] : 0.0f;
        const float bij = pair ? closure_coupling(m, qi, qj) : 0.0f;
        float4 inv = make_float4(a > 1.0e-12f ? 1.0f / a : 0.0f, 0.0f, d > 1.0e-12f ? 1.0f / d : 0.0f, 0.0f);
        if (pair && a > 1.0e-12f && d > 1.0e-12f) {
            const float det = a * d - bij * bij;
            if (det > 1.0e-6f * (a * d)) inv = make_float4(d / det, -bij / det, a / det, 0.0f);
        }
        m.blk_m[blk] = inv;
        blk_b[blk] = bij;
    }
    if (pair_blocks) loop_sync<kGrid>(m.grid_barrier, flags);
    // network inputs: the diagonal-normalised entries of J^T J around the block,
    // with the partner block (blk ^ 1) and the couplings to it recovered from
    // the two probes (exact when the loop's coordinates are these two blocks)
    for (uint32_t blk = tid; pair_blocks && blk < p.blocks; blk += nt) {
        float4 f[4] = {make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0),
                       make_float4(0, 0, 0, 1.0f)};
        const uint32_t qi = 2 * blk, qj = qi + 1;
        const uint32_t ci = m.cq_coords[qi];
        const bool pair = qj < NQ;
        const uint32_t cj = pair ? m.cq_coords[qj] : ci;
        const float a = m.diag[ci], d = pair ? m.diag[cj] : 0.0f, bij = blk_b[blk];
        const uint32_t pb = blk ^ 1u;
        const bool partner = pb < p.blocks && 2 * pb + 1 < NQ;
        if (pair && partner && a > 1.0e-12f && d > 1.0e-12f) {
            const float pa = m.diag[m.cq_coords[2 * pb]], pd = m.diag[m.cq_coords[2 * pb + 1]];
            if (pa > 1.0e-12f && pd > 1.0e-12f) {
                const float s1i = m.probe[ci] - a - bij, ssi = m.probe[Q + ci] - a + bij;
                const float s1j = m.probe[cj] - bij - d, ssj = m.probe[Q + cj] - bij + d;
                const float sa = sqrtf(a), sd = sqrtf(d), spa = sqrtf(pa), spd = sqrtf(pd);
                f[0] = make_float4(bij / (sa * sd), blk_b[pb] / (spa * spd), 0.5f * (s1i + ssi) / (sa * spa),
                                   0.5f * (s1i - ssi) / (sa * spd));
                f[1] = make_float4(0.5f * (s1j + ssj) / (sd * spa), 0.5f * (s1j - ssj) / (sd * spd), logf(a / d),
                                   1.0f);
            }
        }
        float4* fo = m.blk_feat + 4ull * blk;
        fo[0] = f[0]; fo[1] = f[1]; fo[2] = f[2]; fo[3] = f[3];
    }
    // per-loop blocks: Cholesky of J^T J on the loop's coordinates plus a ridge of
    // 1e-6 x the mean diagonal; a failed pivot leaves the block diagonal (Jacobi).
    // Across the grid the off-diagonal couplings (chains of dependent loads) are
    // computed first, one entry per thread, into the block's packed storage, and
    // one thread per loop then factors it; in one block the loop's thread
    // computes them itself (the extra sync and round trip cost more there).
    if (p.precond == MK_PRECOND_BLOCK_JACOBI) {
        if (kGrid) {
            constexpr uint32_t kOff = kMaxLoop * (kMaxLoop - 1) / 2;   // strict lower entries of a block
            for (uint32_t e = tid; e < p.loops * kOff; e += nt) {
                const uint32_t lp = e / kOff;
                uint32_t r = e % kOff, i = 1;
                while (r >= i) { r -= i; ++i; }   // (i, r): row i > column r
                const uint32_t o = m.loop_off[lp], n = m.loop_off[lp + 1] - o;
                if (i < n)
                    m.loop_l[36ull * lp + i * (i + 1) / 2 + r] = closure_coupling(m, m.loop_q[o + i], m.loop_q[o + r]);
            }
            loop_sync<kGrid>(m.grid_barrier, flags);
        }
        for (uint32_t lp = tid; lp < p.loops; lp += nt) {
            const uint32_t o = m.loop_off[lp], n = m.loop_off[lp + 1] - o;
            float a[kMaxLoop * (kMaxLoop + 1) / 2];
            float mean = 0.0f;
            for (uint32_t i = 0; i < n; ++i) mean += m.diag[m.cq_coords[m.loop_q[o + i]]];
            mean = n ? mean / (float)n : 0.0f;
            for (uint32_t i = 0; i < n; ++i)
                for (uint32_t j = 0; j <= i; ++j)
                    a[i * (i + 1) / 2 + j] = i == j  ? m.diag[m.cq_coords[m.loop_q[o + i]]] + 1.0e-6f * mean
                                             : kGrid ? m.loop_l[36ull * lp + i * (i + 1) / 2 + j]
                                                     : closure_coupling(m, m.loop_q[o + i], m.loop_q[o + j]);
            bool ok = mean > 1.0e-12f;
            for (uint32_t j = 0; j < n && ok; ++j) {
                float dj = a[j * (j + 1) / 2 + j];
                for (uint32_t k = 0; k < j; ++k) dj -= a[j * (j + 1) / 2 + k] * a[j * (j + 1) / 2 + k];
                if (!(dj > 0.0f)) { ok = false; break; }
                const float ljj = sqrtf(dj);
                a[j * (j + 1) / 2 + j] = ljj;
                for (uint32_t i = j + 1; i < n; ++i) {
                    float v = a[i * (i + 1) / 2 + j];
                    for (uint32_t k = 0; k < j; ++k) v -= a[i * (i + 1) / 2 + k] * a[j * (j + 1) / 2 + k];
                    a[i * (i + 1) / 2 + j] = v / ljj;
                }
            }
            float* l = m.loop_l + 36ull * lp;
            for (uint32_t i = 0; i < n; ++i)
                for (uint32_t j = 0; j <= i; ++j) {
                    float v = a[i * (i + 1) / 2 + j];
                    if (!ok) {   // Jacobi: L = diag(sqrt(a_ii))
                        const float dii = m.diag[m.cq_coords[m.loop_q[o + i]]];
                        v = (i == j) ? (dii > 1.0e-12f ? sqrtf(dii) : 0.0f) : 0.0f;
                    }
                    l[i * (i + 1) / 2 + j] = v;
                }
        }
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    if (tid == 0) {
        if (unconverged) {
            cs->live_blocks = p.blocks;
            ++cs->newton_steps;
        } else {
            cs->live_blocks = 0;
            st_release_u32(&cs->done, 1u);
        }
    }
}

template <bool kGrid>
__device__ __forceinline__ void precond_apply(const MechBuffers& m, const MechParams& p, const float* r, float* z,
                                              uint32_t* flags) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    if (p.precond == MK_PRECOND_DIAGONAL) {   // closure.wgsl:343-346, :396-400
        for (uint32_t q = tid; q < p.closure_coords; q += nt) {
            const uint32_t c = m.cq_coords[q];
            const float d = m.diag[c];
            z[c] = d > 1.0e-12f ? r[c] / d : 0.0f;
        }
        loop_sync<kGrid>(m.grid_barrier, flags);
        return;
    }
    if (p.precond == MK_PRECOND_BLOCK_JACOBI) {
        for (uint32_t lp = tid; lp < p.loops; lp += nt) {
            const uint32_t o = m.loop_off[lp], n = m.loop_off[lp + 1] - o;
            const float* l = m.loop_l + 36ull * lp;
            float y[kMaxLoop];
            for (uint32_t i = 0; i < n; ++i) {   // L y = r
                float v = r[m.cq_coords[m.loop_q[o + i]]];
                for (uint32_t k = 0; k < i; ++k) v -= l[i * (i + 1) / 2 + k] * y[k];
                const float lii = l[i * (i + 1) / 2 + i];
                y[i] = lii > 0.0f ? v / lii : 0.0f;
            }
            for (uint32_t ii = n; ii-- > 0;) {   // L^T z = y
                float v = y[ii];
                for (uint32_t k = ii + 1; k < n; ++k) v -= l[k * (k + 1) / 2 + ii] * y[k];
                const float lii = l[ii * (ii + 1) / 2 + ii];
                y[ii] = lii > 0.0f ? v / lii : 0.0f;
            }
            for (uint32_t i = 0; i < n; ++i) z[m.cq_coords[m.loop_q[o + i]]] = y[i];
        }
        loop_sync<kGrid>(m.grid_barrier, flags);
        return;
    }
    for (uint32_t blk = tid; blk < p.blocks; blk += nt) {
        const float4 mi = m.blk_m[blk];
        const uint32_t qi = 2 * blk, qj = qi + 1;
        const uint32_t ci = m.cq_coords[qi];
        if (qj < p.closure_coords) {
            const uint32_t cj = m.cq_coords[qj];
            const float ri = r[ci], rj = r[cj];
            z[ci] = mi.x * ri + mi.y * rj;
            z[cj] = mi.y * ri + mi.z * rj;
        } else {
            z[ci] = mi.x * r[ci];
        }
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
}

template <bool kGrid>
__global__ void __launch_bounds__(kClosureThreads) k_closure_pcg(StepBuffers b, MechBuffers m, MechParams p,
                                                                 uint32_t step) {
    __shared__ double s_red[33];
    ClosureState* cs = m.cstate;
    if (ld_acquire_u32(&cs->done)) return;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    const uint32_t NQ = p.closure_coords, NB = p.closure_bodies, Q = p.coordinate_count;
    const uint32_t chunks = (NQ + kDotChunk - 1) / kDotChunk;
    uint32_t* flags = &b.diag->error_flags;
    double* part_a = m.chunk_part_d;            // chunk sums of the FP64 dot products
    double* part_b = m.chunk_part_d + chunks;
    // one block over one chunk: a dot product's block sum is its total (the chunk-order
    // total is 0.0 + the chunk sums), and the sum's barriers order the loop's writes, so
    // neither the chunk sums in memory nor the sync that publishes them are needed
    const bool one = !kGrid && chunks == 1;
    double one_a = 0.0, one_b = 0.0;
    float* sol = m.pcg;
    float* res = m.pcg + Q;
    float* pre = m.pcg + 2ull * Q;
    float* dir = m.pcg + 3ull * Q;
    float* op = m.pcg + 4ull * Q;
    // learned blocks: T' = S M^-1 S with S = diag(sqrt(a), sqrt(d)), from the network's
    // (y0, y1, y2) as t11 = e^y0, t22 = e^y1, t12 = 0.999 tanh(y2) sqrt(t11 t22): positive
    // definite by construction (the check below only catches overflow and NaN)
    if (p.learned_precond) {
        uint32_t used = 0, rejected = 0;
        for (uint32_t blk = tid; blk < p.blocks; blk += nt) {
            const float y0 = fminf(fmaxf(m.blk_out[3 * blk], -30.0f), 30.0f);
            const float y1 = fminf(fmaxf(m.blk_out[3 * blk + 1], -30.0f), 30.0f);
            const float t11 = expf(y0), t22 = expf(y1);
            const float t12 = 0.999f * tanhf(m.blk_out[3 * blk + 2]) * sqrtf(t11 * t22);
            float* h = m.blk_hist + 3ull * ((uint64_t)step * p.blocks + blk);
            h[0] = t11; h[1] = t12; h[2] = t22;
            const uint32_t qi = 2 * blk, qj = qi + 1;
            const uint32_t ci = m.cq_coords[qi];
            const bool pair = qj < NQ;
            const float a = m.diag[ci], d = pair ? m.diag[m.cq_coords[qj]] : 0.0f;
            if (pair) {
                if (a > 1.0e-12f && d > 1.0e-12f && t11 > 0.0f && t22 > 0.0f &&
                    t11 * t22 - t12 * t12 > 1.0e-6f * (t11 * t22)) {
                    const float sa = sqrtf(a), sd = sqrtf(d);
                    m.blk_m[blk] = make_float4(t11 / a, t12 / (sa * sd), t22 / d, 0.0f);
                    ++used;
                } else {
                    ++rejected;
                }
            } else if (a > 1.0e-12f && t11 > 0.0f) {
                m.blk_m[blk] = make_float4(t11 / a, 0.0f, 0.0f, 0.0f);
                ++used;
            } else {
                ++rejected;
            }
        }
        if (used) atomicAdd(&cs->learned_blocks, used);
        if (rejected) atomicAdd(&cs->rejected_blocks, rejected);
        loop_sync<kGrid>(m.grid_barrier, flags);
    }
    // r = -g, x = 0, z = M^-1 r, p = z
    for (uint32_t q = tid; q < NQ; q += nt) {
        const uint32_t c = m.cq_coords[q];
        sol[c] = 0.0f;
        res[c] = -m.grad[c];
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    precond_apply<kGrid>(m, p, res, pre, flags);
    // coordinate loops that feed a dot product walk chunks of 1,024 coordinates
    // (thread t of the chunk's block holds coordinate 1024 c + t)
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const uint32_t q = c * kDotChunk + threadIdx.x;
        double prz = 0.0, prr = 0.0;
        if (q < NQ) {
            const uint32_t cc = m.cq_coords[q];
            dir[cc] = pre[cc];
            prz = (double)res[cc] * (double)pre[cc];
            prr = (double)res[cc] * (double)res[cc];
        }
        const double sz = block_sum_d(prz, s_red), sr = block_sum_d(prr, s_red);
        if (one) { one_a = sz; one_b = sr; }
        else if (threadIdx.x == 0) { part_a[c] = sz; part_b[c] = sr; }
    }
    if (!one) loop_sync<kGrid>(m.grid_barrier, flags);
    double rz = one ? 0.0 + one_a : chunk_total_d(part_a, chunks, s_red);
    const double rr0 = one ? 0.0 + one_b : chunk_total_d(part_b, chunks, s_red);
    double rr = rr0;
    const double tol2 = (double)p.closure_tol * (double)p.closure_tol;
    uint32_t it = 0;
    while (it < p.closure_max_it && rr > tol2 * rr0) {
        closure_apply<kGrid>(m, p, dir, op, flags);
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint32_t q = c * kDotChunk + threadIdx.x;
            double ppq = 0.0;
            if (q < NQ) {
                const uint32_t cc = m.cq_coords[q];
                ppq = (double)dir[cc] * (double)op[cc];
            }
            const double sq = block_sum_d(ppq, s_red);
            if (one) one_a = sq;
            else if (threadIdx.x == 0) part_a[c] = sq;
        }
        if (!one) loop_sync<kGrid>(m.grid_barrier, flags);
        const double pq = one ? 0.0 + one_a : chunk_total_d(part_a, chunks, s_red);
        const float alpha = fabs(pq) > 1.0e-30 ? (float)(rz / pq) : 0.0f;
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint32_t q = c * kDotChunk + threadIdx.x;
            double pr = 0.0;
            if (q < NQ) {
                const uint32_t cc = m.cq_coords[q];
                sol[cc] += alpha * dir[cc];
                res[cc] -= alpha * op[cc];
                pr = (double)res[cc] * (double)res[cc];
            }
            const double sr = block_sum_d(pr, s_red);
            if (one) one_b = sr;
            else if (threadIdx.x == 0) part_b[c] = sr;
        }
        if (!one) loop_sync<kGrid>(m.grid_barrier, flags);
        rr = one ? 0.0 + one_b : chunk_total_d(part_b, chunks, s_red);
        ++it;
        if (rr <= tol2 * rr0) break;
        precond_apply<kGrid>(m, p, res, pre, flags);
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint32_t q = c * kDotChunk + threadIdx.x;
            double pz = 0.0;
            if (q < NQ) {
                const uint32_t cc = m.cq_coords[q];
                pz = (double)res[cc] * (double)pre[cc];
            }
            const double sz = block_sum_d(pz, s_red);
            if (one) one_a = sz;
            else if (threadIdx.x == 0) part_a[c] = sz;
        }
        if (!one) loop_sync<kGrid>(m.grid_barrier, flags);
        const double nrz = one ? 0.0 + one_a : chunk_total_d(part_a, chunks, s_red);
        const float beta = fabs(rz) > 1.0e-300 ? (float)(nrz / rz) : 0.0f;
        for (uint32_t q = tid; q < NQ; q += nt) {
            const uint32_t cc = m.cq_coords[q];
            dir[cc] = pre[cc] + beta * dir[cc];
        }
        rz = nrz;
        loop_sync<kGrid>(m.grid_barrier, flags);
    }
    if (tid == 0) {
        cs->pcg_iterations += it;
        const double rel = rr0 > 0.0 ? sqrt(rr / rr0) : 0.0;
        if (rel > cs->max_relative_residual) cs->max_relative_residual = rel;
    }
    // step the closure coordinates (closure.wgsl:416-427)
    for (uint32_t q = tid; q < NQ; q += nt) {
        const uint32_t c = m.cq_coords[q];
        const float stp = clampf(0.35f * sol[c], -0.2f, 0.2f);
        if (stp == stp) m.coords[c].angle += stp;
        else atomicOr(flags, MK_INVALID_NUMERIC_FLAG);
    }
    loop_sync<kGrid>(m.grid_barrier, flags);
    // forward kinematics of the closure components (mechanism.wgsl:72-149)
    for (uint32_t i = tid; i < NB; i += nt) prepare_link(m, m.cb_bodies[i]);
    loop_sync<kGrid>(m.grid_barrier, flags);
    bool a_src = true;
    for (uint32_t r = 0; r < p.jump_rounds; ++r) {
        for (uint32_t i = tid; i < NB; i += nt)
            jump_link(a_src ? m.links_a : m.links_b, a_src ? m.links_b : m.links_a, m.cb_bodies[i]);
        loop_sync<kGrid>(m.grid_barrier, flags);
        a_src = !a_src;
    }
}

// --------------------------------------------------------------- launches
static inline uint32_t nblocks(uint32_t n) { return (n + kMBlock - 1) / kMBlock; }

// The pose-only parts of the bearing rows, before a set of projection passes.
static cudaError_t bearing_cache(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s) {
    if (p.bearing_count) k_bearing_cache<<<nblocks(p.bearing_count), kMBlock, 0, s>>>(b, m, p);
    return cudaGetLastError();
}

static cudaError_t bearing_projection_iteration(MechBuffers& m, const StepBuffers& b, const MechParams& p,
                                                cudaStream_t s) {
    // a group of kRowLanes lanes per bearing, in 64-thread blocks (8 bearings each)
    if (p.bearing_count) k_project_bearings<<<(p.bearing_count + 7) / 8, 64, 0, s>>>(b, m, p);
    k_apply_mdeltas<<<nblocks(p.body_count), kMBlock, 0, s>>>(b, m, p);
    return cudaGetLastError();
}

static cudaError_t forward_kinematics(MechBuffers& m, const MechParams& p, cudaStream_t s) {
    k_prepare_links<<<nblocks(p.body_count), kMBlock, 0, s>>>(m, p);
    bool a_src = true;
    for (uint32_t r = 0; r < p.jump_rounds; ++r) {
        k_jump<<<nblocks(p.body_count), kMBlock, 0, s>>>(a_src ? m.links_a : m.links_b, a_src ? m.links_b : m.links_a,
                                                         p);
        a_src = !a_src;
    }
    return cudaGetLastError();
}

static cudaError_t reconstruct(MechBuffers& m, const StepBuffers& b, cudaStream_t s) {
    for (uint32_t l = 1; l < m.level_count; ++l) {
        const uint32_t begin = m.level_offsets[l], end = m.level_offsets[l + 1];
        if (end > begin) k_reconstruct_level<<<nblocks(end - begin), kMBlock, 0, s>>>(b, m, begin, end);
    }
    return cudaGetLastError();
}

// Closure solves (the reference's loop and the PCG to a residual): one block
// below kGridClosures closures, the whole grid from there (both compute the
// same values); a tuning override.  Measured on five-body chains: one block is
// faster at 254 closures, even at 410, and the grid from about 1,000 (grid
// barriers cost more than a block's syncs until one closure per thread no
// longer fits).
constexpr uint32_t kGridClosures = 512;
static uint32_t g_closure_grid = 0;
void set_closure_grid(uint32_t mode) { g_closure_grid = mode <= 2u ? mode : 0u; }
uint32_t closure_grid_mode() { return g_closure_grid; }

// One co-resident 1,024-thread block per SM for the grid-wide closure kernels
// (cooperative launch: they sync with grid barriers).  `step` is passed when
// the kernel takes one (kNoStep: it does not).
constexpr uint32_t kNoStep = 0xffffffffu;
static cudaError_t launch_grid(const void* kernel, const StepBuffers& b, const MechBuffers& m, const MechParams& p,
                               uint32_t step, cudaStream_t s) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kClosureThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    StepBuffers bb = b;
    MechBuffers mm = m;
    MechParams pp = p;
    uint32_t st = step;
    void* args3[] = {&bb, &mm, &pp};
    void* args4[] = {&bb, &mm, &pp, &st};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((uint32_t)sms);
    cfg.blockDim = dim3(kClosureThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, kernel, step == kNoStep ? args3 : args4);
}

void mechanism_tick_clears(const MechBuffers& m, const MechParams& p, void** ptr, uint64_t* bytes, uint32_t* count) {
    *count = 0;
    if (p.closures == 0) return;
    ptr[0] = m.grid_barrier;
    bytes[0] = 64 * sizeof(uint32_t);
    ptr[1] = m.loop_state;
    bytes[1] = 2ull * kClosureSteps * sizeof(uint32_t);
    *count = 2;
}

// device.rs:963-1048
cudaError_t enqueue_mechanism(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s) {
    cudaError_t e;
    if ((e = bearing_cache(m, b, p, s)) != cudaSuccess) return e;
    for (uint32_t it = 0; it < std::max(1u, p.iterations); ++it)
        if ((e = bearing_projection_iteration(m, b, p, s)) != cudaSuccess) return e;
    k_advance_coordinates<<<nblocks(p.body_count), kMBlock, 0, s>>>(b, m, p);
    if ((e = forward_kinematics(m, p, s)) != cudaSuccess) return e;
    const uint32_t mode = g_closure_grid;
    const bool grid = p.closures > 0 && (mode == 2u || (mode == 0u && p.closures >= kGridClosures));
    if (pcg_residual_mode(p)) {
        for (uint32_t step = 0; step < kClosureSteps; ++step) {
            if (grid) {
                if ((e = launch_grid((const void*)k_closure_eval<true>, b, m, p, step, s)) != cudaSuccess) return e;
            } else {
                k_closure_eval<false><<<1, kClosureThreads, 0, s>>>(b, m, p, step);
            }
            if (p.learned_precond) {
                e = mlp::forward(m.precond_params, reinterpret_cast<const float*>(m.blk_feat), 0,
                                 &m.cstate->live_blocks, p.blocks, m.blk_out, 3, m.mlp_scratch, &b.diag->error_flags, s);
                if (e != cudaSuccess) return e;
            }
            if (grid) {
                if ((e = launch_grid((const void*)k_closure_pcg<true>, b, m, p, step, s)) != cudaSuccess) return e;
            } else {
                k_closure_pcg<false><<<1, kClosureThreads, 0, s>>>(b, m, p, step);
            }
        }
    } else if (p.closures > 0) {
        if (grid) {
            if ((e = launch_grid((const void*)k_closure_loop<true>, b, m, p, kNoStep, s)) != cudaSuccess) return e;
        } else {
            k_closure_loop<false><<<1, kClosureThreads, 0, s>>>(b, m, p);
        }
    }
    k_publish<<<nblocks(p.body_count), kMBlock, 0, s>>>(b, m, p);
    if ((e = reconstruct(m, b, s)) != cudaSuccess) return e;
    // the published poses hold for the rest of the tick: the projection passes
    // during and after the contact solve share one cache
    return bearing_cache(m, b, p, s);
}

// device.rs:1343-1416 with a dynamic mechanism root
cudaError_t enqueue_contact_solver_with_bearings(MechBuffers& m, const StepBuffers& b, const StepParams& sp,
                                                 const MechParams& p, const StepLaunch& l, int parity,
                                                 cudaStream_t s) {
    return launch_contact_solver_stepwise(b, sp, l, parity, p.serial_contacts != 0u, [&](bool serial) {
        if (serial) {
            k_project_bearings_serial<<<1, 32, 0, s>>>(b, m, p);
            return cudaGetLastError();
        }
        return bearing_projection_iteration(m, b, p, s);
    }, s);
}

// device.rs:1128-1155
cudaError_t enqueue_post_contact(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s) {
    cudaError_t e;
    if (!p.has_dynamic_root)
        for (uint32_t it = 0; it < std::max(1u, p.iterations); ++it)
            if ((e = bearing_projection_iteration(m, b, p, s)) != cudaSuccess) return e;
    k_capture_coordinates<<<nblocks(p.body_count), kMBlock, 0, s>>>(b, m, p);
    if (!p.has_dynamic_root) return reconstruct(m, b, s);
    return cudaGetLastError();
}

void enqueue_validate_state(MechBuffers& m, const StepBuffers& b, const MechParams& p, cudaStream_t s) {
    k_validate_state<<<nblocks(p.body_count), kMBlock, 0, s>>>(b, m, p);
}

void enqueue_validate_bearings(MechBuffers& m, const StepBuffers& b, const MechParams& p, bool mechanism_active,
                               cudaStream_t s) {
    if (p.bearing_count == 0) return;
    k_validate_bearings<<<nblocks(p.bearing_count), kMBlock, 0, s>>>(m.bearings, p.bearing_count, b.pos, b.rot,
                                                                      mechanism_active ? m.links_final : nullptr,
                                                                      b.diag);
}

void read_mechanism_readback(const MechBuffers& m, const MechParams& p, const GpuDiagnostics& d,
                             const ClosureState* cs, MkTickReadback* out) {
    (void)m;
    if (pcg_residual_mode(p) && cs) {
        out->closure_iterations = cs->pcg_iterations;
        out->closure_relative_residual = cs->max_relative_residual;
    } else {
        out->closure_iterations = d.reserved_c;
        out->closure_relative_residual = 0.0;
    }
}

uint64_t mechanism_mlp_scratch_bytes(const MechParams& p) {
    return p.learned_precond ? mlp::scratch_bytes(0) : 0;
}

}  // namespace mk
