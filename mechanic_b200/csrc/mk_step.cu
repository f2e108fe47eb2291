// mk_step.cu — the plain rigid-body tick on sm_100a.
//
// Stage map (reference kernel -> this file):
//   physics.wgsl integrate :92-132 + collision.wgsl update_world_masses
//     :144-162 + snapshot.wgsl publish_snapshot :6-14       -> k_integrate
//   lbvh.wgsl compute_morton :108-130                        -> k_collider_bounds
//   lbvh.wgsl sort_* :132-217                                -> mk_sort.cu (onesweep)
//   lbvh.wgsl build_topology :233-278                        -> k_karras
//   lbvh.wgsl prepare_leaves + build_bounds :280-319         -> k_refit
//   lbvh.wgsl traverse :361-398                              -> k_traverse + pair-key radix sort
//   collision.wgsl narrowphase :570-603                      -> k_narrowphase
//   collision.wgsl generate_ground_contacts :622-664         -> k_ground
//   collision.wgsl prepare_contacts :674-736                 -> k_prepare
//   collision.wgsl warm_start / solve_accumulate :774-906 and
//   solve_apply :1050-1069 (8 iterations)                    -> k_solve_all (cooperative, grid barriers)
//   collision.wgsl persist_contacts :1071-1088               -> the contact list itself (ping-pong)
//
// Variable-size stages (pairs, contacts, active contacts) run as persistent
// grids that take tiles in ticket order and append their output in
// canonical order through a decoupled look-back, so the whole tick is a
// fixed launch sequence (CUDA-graph friendly) with deterministic output.
#include <cstdio>
#include <functional>

#include "mk_device.cuh"
#include "mk_internal.h"

namespace mk {

constexpr uint32_t kBlock = 256;
constexpr uint32_t kFixedScale = 1048576;   // FIXED_VELOCITY_SCALE (collision.wgsl:63)

// ---------------------------------------------------------------- integrate
// physics.wgsl:92-132, then (no mechanism) world inverse inertia
// (collision.wgsl:134-162) and the snapshot ring copy (snapshot.wgsl:6-14):
// positions do not change again during a plain tick.
__device__ __forceinline__ f3 world_inverse_inertia_column(float4 r, const float4* m, f3 axis) {
    f3 local = quat_rotate(conjq(r), axis);
    f3 lr = xyz(m[1]) * local.x + xyz(m[2]) * local.y + xyz(m[3]) * local.z;
    return quat_rotate(r, lr);
}

__device__ __forceinline__ void write_world_mass(float4* wm, float4 r, const float4* m) {
    wm[0] = f4(world_inverse_inertia_column(r, m, mkf3(1, 0, 0)), m[0].x);
    wm[1] = f4(world_inverse_inertia_column(r, m, mkf3(0, 1, 0)), 0.0f);
    wm[2] = f4(world_inverse_inertia_column(r, m, mkf3(0, 0, 1)), 0.0f);
}

template <bool kFuse>
__global__ void __launch_bounds__(kBlock) k_integrate(StepBuffers b, StepParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.body_count) return;
    float4 pos = b.pos[i], q = b.rot[i], l = b.lin[i], a = b.ang[i];
    const float inv = b.inv_mass[i];
    if (inv > 0.0f) {
        l.y += p.gravity * p.dt;
        f3 lv = xyz(l) * p.lin_damp;
        l = f4(lv, l.w);
        f3 av = xyz(a) * p.ang_damp;
        a = f4(av, a.w);
        if (b.root_flags[i] != 0u) {
            f3 pv = xyz(pos) + xyz(l) * p.dt;
            pos = f4(pv, pos.w);
            float4 spin = f4(xyz(a), 0.0f);
            float4 d = quat_multiply(spin, q);
            const float h = 0.5f * p.dt;
            q = make_float4(q.x + d.x * h, q.y + d.y * h, q.z + d.z * h, q.w + d.w * h);
            float ns = dot4(q, q);
            if (ns > 1.0e-20f) {
                float s = rsqrt_ieee(ns);
                q = make_float4(q.x * s, q.y * s, q.z * s, q.w * s);
            } else {
                q = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                atomicOr(&b.diag->error_flags, MK_INVALID_NUMERIC_FLAG);
            }
        }
    }
    bool ok = finite4(pos) && finite4(q) && finite4(l) && finite4(a);
    if (!ok) {
        atomicOr(&b.diag->error_flags, MK_INVALID_NUMERIC_FLAG);
        pos = b.pos[i];
        q = b.rot[i];
    } else {
        b.pos[i] = pos;
        b.rot[i] = q;
        b.lin[i] = l;
        b.ang[i] = a;
    }
    if (kFuse) {
        const float4* m = b.mass + 4ull * i;
        float4 mr[4] = {__ldg(m), __ldg(m + 1), __ldg(m + 2), __ldg(m + 3)};
        write_world_mass(b.world_mass + 3ull * i, q, mr);
        const uint32_t slot = b.tick->snapshot_slot;
        b.snap_pos[(size_t)slot * p.body_count + i] = pos;
        b.snap_rot[(size_t)slot * p.body_count + i] = q;
    }
}

__global__ void __launch_bounds__(kBlock) k_world_masses(StepBuffers b, StepParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.body_count) return;
    const float4* m = b.mass + 4ull * i;
    float4 mr[4] = {__ldg(m), __ldg(m + 1), __ldg(m + 2), __ldg(m + 3)};
    write_world_mass(b.world_mass + 3ull * i, b.rot[i], mr);
}

__global__ void __launch_bounds__(kBlock) k_snapshot(StepBuffers b, StepParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.body_count) return;
    const uint32_t slot = b.tick->snapshot_slot;
    b.snap_pos[(size_t)slot * p.body_count + i] = b.pos[i];
    b.snap_rot[(size_t)slot * p.body_count + i] = b.rot[i];
}

// ------------------------------------------------------------ bounds/Morton
__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint64_t expand21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
// lbvh.wgsl:93-98: 10 bits per axis over 1 m cells in [-512, 512).
__device__ __forceinline__ uint32_t morton30(f3 c) {
    uint32_t qx = (uint32_t)clampf(floorf(c.x + 512.0f), 0.0f, 1023.0f);
    uint32_t qy = (uint32_t)clampf(floorf(c.y + 512.0f), 0.0f, 1023.0f);
    uint32_t qz = (uint32_t)clampf(floorf(c.z + 512.0f), 0.0f, 1023.0f);
    return expand10(qx) | (expand10(qy) << 1) | (expand10(qz) << 2);
}
// `qmax + 1` cells per axis (2^21 for 63-bit keys, 2^16 for 48-bit keys) over
// the tick's bounds of the collider centres (cubic cells: one scale from the
// largest extent), so the keys stay spread however far the scene moves.
__device__ __forceinline__ uint64_t morton_frame(f3 c, f3 lo, float scale, float qmax) {
    uint64_t qx = (uint64_t)clampf(floorf((c.x - lo.x) * scale), 0.0f, qmax);
    uint64_t qy = (uint64_t)clampf(floorf((c.y - lo.y) * scale), 0.0f, qmax);
    uint64_t qz = (uint64_t)clampf(floorf((c.z - lo.z) * scale), 0.0f, qmax);
    return expand21(qx) | (expand21(qy) << 1) | (expand21(qz) << 2);
}
__device__ __forceinline__ float frame_qmax(uint32_t mode) {
    return mode == MK_MORTON_30_ADAPTIVE ? 1023.0f
           : mode == MK_MORTON_39      ? 8191.0f
           : mode == MK_MORTON_48      ? 65535.0f
                                       : 2097151.0f;
}
// Floats as unsigned integers in the same order (-0 below +0), for exact
// order-free min / max with integer atomics.
__device__ __forceinline__ uint32_t float_order(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_unorder(uint32_t v) {
    return __uint_as_float((v & 0x80000000u) ? (v & 0x7fffffffu) : ~v);
}
// Scene bounds words (zeroed at the start of a tick): max of the ordered x, y, z, then
// max of their complements (the min).
__device__ __forceinline__ void key_frame(const uint32_t* bw, float qmax, f3& lo, float& scale) {
    lo = mkf3(float_unorder(~bw[3]), float_unorder(~bw[4]), float_unorder(~bw[5]));
    const f3 hi = mkf3(float_unorder(bw[0]), float_unorder(bw[1]), float_unorder(bw[2]));
    const float extent = mxf(mxf(hi.x - lo.x, hi.y - lo.y), hi.z - lo.z);
    scale = extent > 0.0f ? qmax / extent : 1.0f;
}

constexpr uint32_t kGroundTile = 1024;   // colliders per ground-contact tile (32 mask words)

// collision.wgsl:622-664 support point of collider i against the ground plane
// (defined with the ground contacts below); true when it touches.
__device__ __forceinline__ bool ground_point(const StepBuffers& b, uint32_t i, f3& sp, uint32_t& body,
                                             uint32_t& role);

// lbvh.wgsl:108-130 plus the world box row the narrowphase reads:
// box r0 = {center, half.x}, r1 = world rotation, r2 = {half.y, half.z, body, role}.
__global__ void __launch_bounds__(kBlock) k_collider_bounds(StepBuffers b, StepParams p, uint32_t morton_mode) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < p.collider_count;
    f3 center = mkf3(0, 0, 0);
    if (valid) {
        const float4* c = b.colliders + 4ull * i;
        const float4 lc = __ldg(c), lr = __ldg(c + 1), he = __ldg(c + 2);
        const uint4 meta = __ldg(reinterpret_cast<const uint4*>(c + 3));
        const uint32_t body = meta.x;
        const float4 bq = b.rot[body];
        center = xyz(b.pos[body]) + quat_rotate(bq, xyz(lc));
        const float4 r = quat_multiply(bq, lr);
        const f3 ax = quat_rotate(r, mkf3(1, 0, 0));
        const f3 ay = quat_rotate(r, mkf3(0, 1, 0));
        const f3 az = quat_rotate(r, mkf3(0, 0, 1));
        const f3 e = absf3(ax) * he.x + absf3(ay) * he.y + absf3(az) * he.z;
        b.aabbs[2ull * i] = f4(center - e, 0.0f);
        b.aabbs[2ull * i + 1] = f4(center + e, 0.0f);
        float4* box = b.boxes + 3ull * i;
        box[0] = f4(center, he.x);
        box[1] = r;
        box[2] = make_float4(he.y, he.z, __uint_as_float(body), __uint_as_float(meta.w));
        b.values[i] = i;
        if (morton_mode == MK_MORTON_REFERENCE_30)
            b.keys[i] = compose_key(morton_mode, p.scene_bits, p.scene_bits ? b.collider_scene[i] : 0u,
                                    morton30(center));
    }
    {   // ground test of each collider from its fresh box: a bit per collider and a
        // count per ground tile, so the ground contacts need neither a second
        // pass over every box nor an ordered-append look-back
        bool touch = false;
        if (valid) {
            f3 sp;
            uint32_t body, role;
            touch = ground_point(b, i, sp, body, role);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, touch);
        if (lane_id() == 0 && (uint64_t)i < p.collider_count) {
            b.ground_mask[i >> 5] = m;
            if (m) atomicAdd(b.ground_tile_count + i / kGroundTile, (uint32_t)__popc(m));
        }
    }
    if (morton_mode == MK_MORTON_REFERENCE_30) return;
    // the tick's bounds of the finite collider centres: warp then block reductions of
    // the ordered integers, one atomic per block and word, skipped when the word
    // already holds as much (exact and order-free; per-warp atomics on six words
    // serialised in L2 and cost 40 us at 400k colliders)
    const bool use = valid && isfinite(center.x) && isfinite(center.y) && isfinite(center.z);
    const float cc[3] = {center.x, center.y, center.z};
    uint32_t w[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const uint32_t o = use ? float_order(cc[a]) : 0u;
        w[a] = o;                         // max of the ordered value
        w[3 + a] = use ? ~o : 0u;         // max of its complement = min
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) w[k] = max(w[k], __shfl_xor_sync(0xffffffffu, w[k], d));
    }
    __shared__ uint32_t s_w[kBlock / 32][6];
    const uint32_t warp = threadIdx.x >> 5;
    if (lane_id() == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) s_w[warp][k] = w[k];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        uint32_t m = 0;
#pragma unroll
        for (uint32_t q = 0; q < kBlock / 32; ++q) m = max(m, s_w[q][threadIdx.x]);
        uint32_t* word = b.scene_bounds + threadIdx.x;
        if (m > *reinterpret_cast<volatile uint32_t*>(word)) atomicMax(word, m);
    }
}

// Keys over the tick's centre bounds (every mode but MK_MORTON_REFERENCE_30).
__global__ void __launch_bounds__(kBlock) k_morton_keys(StepBuffers b, StepParams p, uint32_t morton_mode) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.collider_count) return;
    const float qmax = frame_qmax(morton_mode);
    f3 lo;
    float scale;
    key_frame(b.scene_bounds, qmax, lo, scale);
    const uint64_t key = morton_frame(xyz(b.boxes[3ull * i]), lo, scale, qmax);
    b.keys[i] = compose_key(morton_mode, p.scene_bits, p.scene_bits ? b.collider_scene[i] : 0u, key);
}

// ------------------------------------------------------------- Karras tree
__device__ __forceinline__ int common_prefix(const uint64_t* __restrict__ k, const uint32_t* __restrict__ v,
                                             int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t d = k[i] ^ k[j];
    if (d != 0) return __clzll((long long)d);
    return 64 + __clz((int)(v[i] ^ v[j]));
}

// lbvh.wgsl:219-278 (Karras 2012) over (key, index) entries.
__global__ void __launch_bounds__(kBlock) k_karras(StepBuffers b, StepParams p) {
    const int n = (int)p.collider_count;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) b.parents[0] = 0u;
    if (n <= 1 || i >= n - 1) return;
    const uint64_t* k = b.skeys;
    const uint32_t* v = b.svals;
    const int dir = common_prefix(k, v, n, i, i + 1) > common_prefix(k, v, n, i, i - 1) ? 1 : -1;
    const int min_prefix = common_prefix(k, v, n, i, i - dir);
    int max_len = 2;
    while (common_prefix(k, v, n, i, i + max_len * dir) > min_prefix) max_len *= 2;
    int len = 0;
    for (int step = max_len / 2; step >= 1; step /= 2)
        if (common_prefix(k, v, n, i, i + (len + step) * dir) > min_prefix) len += step;
    const int other = i + len * dir;
    const int node_prefix = common_prefix(k, v, n, i, other);
    int split_off = 0;
    int step = (len + 1) / 2;
    while (step >= 1) {
        if (common_prefix(k, v, n, i, i + (split_off + step) * dir) > node_prefix) split_off += step;
        if (step == 1) break;
        step = (step + 1) / 2;
    }
    const int split = i + split_off * dir + min(dir, 0);
    const int first = min(i, other), last = max(i, other);
    const uint32_t leaf_base = (uint32_t)(n - 1);
    if (b.collider_scene) {   // batched scenes: the node over exactly one scene's leaves is that scene's root
        const uint32_t sc = b.collider_scene[v[first]];
        const uint32_t begin = sc ? b.scene_end[sc - 1] : 0u;
        if ((uint32_t)first == begin && (uint32_t)last + 1u == b.scene_end[sc]) b.scene_root[sc] = (uint32_t)i;
    }
    const uint32_t left = split == first ? leaf_base + (uint32_t)split : (uint32_t)split;
    const uint32_t right = split + 1 == last ? leaf_base + (uint32_t)(split + 1) : (uint32_t)(split + 1);
    b.children[i] = make_uint2(left, right);
    b.parents[left] = (uint32_t)i + 1u;
    b.parents[right] = (uint32_t)i + 1u;
    b.node_ranges[i] = make_uint2((uint32_t)first, (uint32_t)last);
}

// Traversal record codes: an internal node index, or kLeafCode | collider index
// for a leaf.
constexpr uint32_t kLeafCode = 0x80000000u;

// Parallel refit.  An internal node covers a contiguous range of sorted
// leaves (Karras), so its box is the union of the leaf boxes in that range;
// unions are min/max, exact in any order, so this equals the bottom-up climb
// of lbvh.wgsl:280-319 without its serial chain of tree depth.  Range unions
// come from prefix/suffix unions within 32-leaf chunks (warp scans), within
// 1024-leaf super-chunks (over chunk totals) and a sparse table over the
// super-chunk totals.
constexpr uint32_t kRefitBlock = 1024;   // one super-chunk of 32 chunks per block

struct Box2 {
    float4 mn, mx;
};
__device__ __forceinline__ Box2 box_empty() {
    return {make_float4(kFloatMax, kFloatMax, kFloatMax, 0.0f), make_float4(-kFloatMax, -kFloatMax, -kFloatMax, 0.0f)};
}
__device__ __forceinline__ Box2 box_union(Box2 a, Box2 c) {
    return {make_float4(mnf(a.mn.x, c.mn.x), mnf(a.mn.y, c.mn.y), mnf(a.mn.z, c.mn.z), 0.0f),
            make_float4(mxf(a.mx.x, c.mx.x), mxf(a.mx.y, c.mx.y), mxf(a.mx.z, c.mx.z), 0.0f)};
}
// Box shuffles move the six coordinates (the w lanes of a union are 0).
__device__ __forceinline__ Box2 shfl_box(Box2 v, int o, bool up) {
    auto sh = [&](float x) { return up ? __shfl_up_sync(0xffffffffu, x, o) : __shfl_down_sync(0xffffffffu, x, o); };
    return {make_float4(sh(v.mn.x), sh(v.mn.y), sh(v.mn.z), 0.0f), make_float4(sh(v.mx.x), sh(v.mx.y), sh(v.mx.z), 0.0f)};
}
__device__ __forceinline__ Box2 shfl_box_idx(Box2 v, uint32_t src) {
    auto sh = [&](float x) { return __shfl_sync(0xffffffffu, x, src); };
    return {make_float4(sh(v.mn.x), sh(v.mn.y), sh(v.mn.z), 0.0f), make_float4(sh(v.mx.x), sh(v.mx.y), sh(v.mx.z), 0.0f)};
}
// Sparse table over a warp's 32 boxes: T[k] at lane l is the union of lanes
// [l, l + 2^k) (cut at lane 31), so the union of lanes [a, z] is that of
// T[k] at a and at z + 1 - 2^k with k = min(floor(log2(z - a + 1)), 4).
__device__ __forceinline__ void warp_sparse_table(Box2 (&T)[5], Box2 v, uint32_t lane) {
    T[0] = v;
#pragma unroll
    for (int k = 1; k < 5; ++k) {
        const Box2 d = shfl_box(T[k - 1], 1 << (k - 1), false);
        T[k] = (int)lane + (1 << (k - 1)) < 32 ? box_union(T[k - 1], d) : T[k - 1];
    }
}
// Union of lanes [a, z] from the table (every lane takes part; `want` marks the
// lanes whose result is used).
__device__ __forceinline__ Box2 warp_range_union(const Box2 (&T)[5], bool want, uint32_t a, uint32_t z, uint32_t lane) {
    const uint32_t k = want ? min(31u - __clz(z - a + 1u), 4u) : 0u;   // 32 lanes: two 16-lane windows
    const uint32_t s0 = want ? a : lane, s1 = want ? z + 1u - (1u << k) : lane;
    Box2 r = box_empty();
#pragma unroll
    for (uint32_t kk = 0; kk < 5; ++kk) {
        const Box2 x0 = shfl_box_idx(T[kk], s0), x1 = shfl_box_idx(T[kk], s1);
        if (kk == k) r = box_union(x0, x1);
    }
    return r;
}
__device__ __forceinline__ Box2 ld_box(const float4* p) { return {__ldg(p), __ldg(p + 1)}; }   // written by earlier launches
__device__ __forceinline__ Box2 ld_box_cg(const float4* p) { return {__ldcg(p), __ldcg(p + 1)}; }
__device__ __forceinline__ void st_box(float4* p, Box2 v) { p[0] = v.mn; p[1] = v.mx; }

// Per internal node: its union box and a 4-wide traversal record (128 bytes,
// one cache line) holding its grandchildren in leaf order -- a leaf child is
// one entry, an internal child gives its two children -- so a traversal step
// descends two levels with one load.  Entry: {min.xyz, code} {max.xyz, last
// leaf}, code = child node index or kLeafCode | collider index; unused
// trailing entries are zero (last leaf 0).  An entry's first leaf is one past
// the last leaf of the entry before it (the first entry starts where the node
// does).
struct TravEntry {
    Box2 box;
    uint32_t code, last;
};
__device__ __forceinline__ void store_record(float4* rec, const TravEntry (&e)[4], uint32_t m) {
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        if (k < m) {
            rec[2 * k] = make_float4(e[k].box.mn.x, e[k].box.mn.y, e[k].box.mn.z, __uint_as_float(e[k].code));
            rec[2 * k + 1] = make_float4(e[k].box.mx.x, e[k].box.mx.y, e[k].box.mx.z, __uint_as_float(e[k].last));
        } else {
            rec[2 * k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            rec[2 * k + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// Traversal records of the in-chunk nodes, written by the warp that owns the
// chunk: every descendant of a node whose leaf range lies in one 32-leaf
// chunk is an internal node or leaf of that chunk (Karras node c sits at one
// end of its range), so children come from the lane c & 31 and boxes from
// the lane of the node or leaf -- no global reads besides the node's own
// children.  `v`/`j` are this lane's leaf box and collider index, `r` its
// node's box (valid where `inner`).  Every lane takes part in the shuffles.
__device__ __forceinline__ void write_chunk_records(const StepBuffers& b, bool inner, uint2 rg, Box2 r, Box2 v,
                                                    uint32_t j, uint32_t t, uint32_t leaf_base, uint32_t lane) {
    const uint2 ch = inner ? b.children[t] : make_uint2(0u, 0u);
    const Box2 nb = inner ? r : box_empty();
    auto lane_of_node = [&](uint32_t c) { return inner && c < leaf_base ? (c & 31u) : lane; };
    const uint32_t lx = lane_of_node(ch.x), ly = lane_of_node(ch.y);
    const uint2 cl = make_uint2(__shfl_sync(0xffffffffu, ch.x, lx), __shfl_sync(0xffffffffu, ch.y, lx));
    const uint2 cr = make_uint2(__shfl_sync(0xffffffffu, ch.x, ly), __shfl_sync(0xffffffffu, ch.y, ly));
    const uint32_t split = ch.x >= leaf_base ? ch.x - leaf_base : ch.x;
    // slots: left child's (one leaf, or its two children), then the right's
    uint32_t node[4], first[4], last[4];
    bool use[4];
    auto child = [&](uint32_t s, uint32_t c, uint2 cc, uint32_t f, uint32_t l) {
        if (c >= leaf_base) {   // a leaf child: one entry
            node[s] = c; first[s] = f; last[s] = f; use[s] = true;
            node[s + 1] = 0u; first[s + 1] = 0u; last[s + 1] = 0u; use[s + 1] = false;
        } else {
            const uint32_t sp = cc.x >= leaf_base ? cc.x - leaf_base : cc.x;
            node[s] = cc.x; first[s] = f; last[s] = sp; use[s] = true;
            node[s + 1] = cc.y; first[s + 1] = sp + 1u; last[s + 1] = l; use[s + 1] = true;
        }
    };
    child(0, ch.x, cl, rg.x, split);
    child(2, ch.y, cr, split + 1u, rg.y);
    TravEntry sl[4];
#pragma unroll
    for (uint32_t s = 0; s < 4; ++s) {
        const bool leaf = node[s] >= leaf_base;
        const uint32_t src = inner && use[s] ? (leaf ? first[s] & 31u : node[s] & 31u) : lane;
        const Box2 lb = shfl_box_idx(v, src), ib = shfl_box_idx(nb, src);
        const uint32_t jj = __shfl_sync(0xffffffffu, j, src);
        sl[s] = {leaf ? lb : ib, leaf ? (kLeafCode | jj) : node[s], last[s]};
    }
    // compact in leaf order: a leaf child leaves its second slot empty
    const bool li = use[1], ri = use[3];
    const TravEntry e[4] = {sl[0], li ? sl[1] : sl[2], li ? sl[2] : sl[3], sl[3]};
    if (inner) store_record(b.node_records + 8ull * t, e, (li ? 2u : 1u) + (ri ? 2u : 1u));
}

// Leaf boxes in sorted order, their prefix/suffix unions within 32-leaf chunks,
// the boxes of the internal nodes whose leaf range lies inside one chunk (from
// a warp sparse table; Karras node i's range has i at one end, so the warp of
// leaf i owns node i), the chunks' prefix/suffix unions and sparse table within
// the block's super-chunk, and the super-chunk's total (level 0 of the sparse
// table over super-chunks).
__global__ void __launch_bounds__(kRefitBlock) k_refit_leaves(StepBuffers b, StepParams p) {
    __shared__ Box2 s_chunk[32];
    const uint32_t n = p.collider_count;
    const uint32_t t = blockIdx.x * kRefitBlock + threadIdx.x;
    const uint32_t lane = lane_id(), w = warp_id();
    const uint32_t leaf_base = n - 1;
    Box2 v = box_empty();
    const uint32_t j = t < n ? b.svals[t] : 0u;
    if (t < n) {
        float4 mn = b.aabbs[2ull * j], mx = b.aabbs[2ull * j + 1];
        mn.w = __uint_as_float(t);
        b.node_aabbs[2ull * (leaf_base + t)] = mn;
        b.node_aabbs[2ull * (leaf_base + t) + 1] = mx;
        v = {make_float4(mn.x, mn.y, mn.z, 0.0f), make_float4(mx.x, mx.y, mx.z, 0.0f)};
    }
    Box2 pre = v, suf = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Box2 u = shfl_box(pre, o, true);
        if ((int)lane >= o) pre = box_union(pre, u);
        const Box2 d = shfl_box(suf, o, false);
        if ((int)lane + o < 32) suf = box_union(suf, d);
    }
    if (t < n) {
        float4* ls = b.leaf_scan + 4ull * t;
        ls[0] = pre.mn; ls[1] = pre.mx; ls[2] = suf.mn; ls[3] = suf.mx;
    }
    {
        Box2 T[5];
        warp_sparse_table(T, v, lane);
        uint2 rg = make_uint2(1u, 0u);
        bool inner = false;
        if (n > 1 && t < n - 1) {
            rg = b.node_ranges[t];
            inner = (rg.x >> 5) == (rg.y >> 5);
        }
        const Box2 r = warp_range_union(T, inner, rg.x & 31u, rg.y & 31u, lane);
        if (inner) {
            b.node_aabbs[2ull * t] = make_float4(r.mn.x, r.mn.y, r.mn.z, __uint_as_float(rg.y));
            b.node_aabbs[2ull * t + 1] = make_float4(r.mx.x, r.mx.y, r.mx.z, 0.0f);
        }
        write_chunk_records(b, inner, rg, r, v, j, t, leaf_base, lane);
        // the other internal nodes, listed for k_refit_nodes (one reservation per warp)
        const bool cross = n > 1 && t < n - 1 && !inner;
        const uint32_t cm = __ballot_sync(0xffffffffu, cross);
        if (cm) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&b.counts->cross_nodes, (uint32_t)__popc(cm));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (cross) b.cross_nodes[base + __popc(cm & ((1u << lane) - 1u))] = t;
        }
    }
    if (lane == 31) s_chunk[w] = pre;
    __syncthreads();
    if (w == 0) {
        const Box2 c = s_chunk[lane];
        Box2 cp = c, cs = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Box2 u = shfl_box(cp, o, true);
            if ((int)lane >= o) cp = box_union(cp, u);
            const Box2 d = shfl_box(cs, o, false);
            if ((int)lane + o < 32) cs = box_union(cs, d);
        }
        const uint32_t chunk = blockIdx.x * 32 + lane;
        if ((uint64_t)chunk * 32 < n) {
            float4* cr = b.chunk_scan + 6ull * chunk;   // total, prefix, suffix within the super-chunk
            cr[0] = c.mn; cr[1] = c.mx; cr[2] = cp.mn; cr[3] = cp.mx; cr[4] = cs.mn; cr[5] = cs.mx;
        }
        if (lane == 31) st_box(b.super_table + 2ull * blockIdx.x, cp);
        Box2 T[5];
        warp_sparse_table(T, c, lane);
        const uint32_t chunks = (n + 31) / 32;
        if (chunk < chunks) {
#pragma unroll
            for (int k = 1; k < 5; ++k) st_box(b.chunk_table + 2ull * (chunks * (k - 1) + chunk), T[k]);
        }
    }
}

// Sparse table over the super-chunk totals: level k holds unions of 2^k of them.
// Up to kSuperSmem super-chunks (2M colliders) the levels are built in shared
// memory and written out as they complete; beyond, level by level through L2.
constexpr uint32_t kSuperSmem = 2048;
__global__ void __launch_bounds__(1024) k_refit_super(StepBuffers b, StepParams p) {
    const uint32_t n = p.collider_count;
    const uint32_t ns = (n + kRefitBlock - 1) / kRefitBlock;
    if (ns <= kSuperSmem) {
        constexpr uint32_t kPer = kSuperSmem / 1024;
        __shared__ float s_t[6][kSuperSmem];   // min.xyz, max.xyz of the current level
        for (uint32_t q = threadIdx.x; q < ns; q += blockDim.x) {
            const Box2 v = ld_box_cg(b.super_table + 2ull * q);
            s_t[0][q] = v.mn.x; s_t[1][q] = v.mn.y; s_t[2][q] = v.mn.z;
            s_t[3][q] = v.mx.x; s_t[4][q] = v.mx.y; s_t[5][q] = v.mx.z;
        }
        __syncthreads();
        auto at = [&](uint32_t q) -> Box2 {
            return {make_float4(s_t[0][q], s_t[1][q], s_t[2][q], 0.0f), make_float4(s_t[3][q], s_t[4][q], s_t[5][q], 0.0f)};
        };
        for (uint32_t k = 1; (1u << k) <= ns; ++k) {
            const uint32_t half = 1u << (k - 1);
            float4* dst = b.super_table + 2ull * ns * k;
            Box2 u[kPer];
#pragma unroll
            for (uint32_t e = 0; e < kPer; ++e) {
                const uint32_t q = threadIdx.x + e * 1024u;
                if (q + (1u << k) <= ns) u[e] = box_union(at(q), at(q + half));
            }
            __syncthreads();   // every read of the level below is done
#pragma unroll
            for (uint32_t e = 0; e < kPer; ++e) {
                const uint32_t q = threadIdx.x + e * 1024u;
                if (q + (1u << k) <= ns) {
                    s_t[0][q] = u[e].mn.x; s_t[1][q] = u[e].mn.y; s_t[2][q] = u[e].mn.z;
                    s_t[3][q] = u[e].mx.x; s_t[4][q] = u[e].mx.y; s_t[5][q] = u[e].mx.z;
                    st_box(dst + 2ull * q, u[e]);
                }
            }
            __syncthreads();
        }
        return;
    }
    for (uint32_t k = 1; (1u << k) <= ns; ++k) {
        const float4* src = b.super_table + 2ull * ns * (k - 1);
        float4* dst = b.super_table + 2ull * ns * k;
        const uint32_t half = 1u << (k - 1);
        for (uint32_t s = threadIdx.x; s + (1u << k) <= ns; s += blockDim.x)
            st_box(dst + 2ull * s, box_union(ld_box_cg(src + 2ull * s), ld_box_cg(src + 2ull * (s + half))));
        __threadfence_block();
        __syncthreads();
    }
}

__device__ __forceinline__ Box2 leaf_box(const StepBuffers& b, uint32_t leaf_base, uint32_t t) {
    const float4* q = b.node_aabbs + 2ull * (leaf_base + t);
    const float4 mn = __ldg(q), mx = __ldg(q + 1);
    return {make_float4(mn.x, mn.y, mn.z, 0.0f), make_float4(mx.x, mx.y, mx.z, 0.0f)};
}

// Union of the chunk totals [c0, c1] inside one super-chunk: a prefix, a
// suffix, or two entries of the chunk sparse table.
__device__ __forceinline__ Box2 chunks_union(const StepBuffers& b, uint32_t n, uint32_t c0, uint32_t c1) {
    if ((c0 & 31u) == 0) return ld_box(b.chunk_scan + 6ull * c1 + 2);   // prefix of c1
    if ((c1 & 31u) == 31u) return ld_box(b.chunk_scan + 6ull * c0 + 4);   // suffix of c0
    const uint32_t k = 31u - __clz(c1 - c0 + 1u);
    if (k == 0) return ld_box(b.chunk_scan + 6ull * c0);   // one chunk's total
    const float4* lvl = b.chunk_table + 2ull * ((n + 31) / 32) * (k - 1);
    return box_union(ld_box(lvl + 2ull * c0), ld_box(lvl + 2ull * (c1 + 1u - (1u << k))));
}

// Union of the sorted leaves [f, l].
__device__ Box2 range_box(const StepBuffers& b, uint32_t n, uint32_t f, uint32_t l) {
    const uint32_t leaf_base = n - 1;
    const uint32_t cf = f >> 5, cl = l >> 5;
    if (cf == cl) {
        if ((f & 31u) == 0) return ld_box(b.leaf_scan + 4ull * l);        // prefix of l
        if ((l & 31u) == 31u || l == n - 1) return ld_box(b.leaf_scan + 4ull * f + 2);   // suffix of f
        Box2 u = box_empty();
        for (uint32_t t = f; t <= l; ++t) u = box_union(u, leaf_box(b, leaf_base, t));
        return u;
    }
    Box2 u = box_union(ld_box(b.leaf_scan + 4ull * f + 2), ld_box(b.leaf_scan + 4ull * l));
    if (cf + 1 > cl - 1) return u;
    const uint32_t a = cf + 1, z = cl - 1;
    const uint32_t sa = a >> 5, sz = z >> 5;
    if (sa == sz) return box_union(u, chunks_union(b, n, a, z));
    u = box_union(u, ld_box(b.chunk_scan + 6ull * a + 4));   // suffix of a within its super-chunk
    u = box_union(u, ld_box(b.chunk_scan + 6ull * z + 2));   // prefix of z within its super-chunk
    if (sa + 1 <= sz - 1) {
        const uint32_t ns = (n + kRefitBlock - 1) / kRefitBlock;
        const uint32_t lo = sa + 1, hi = sz - 1, len = hi - lo + 1;
        const uint32_t k = 31u - __clz(len);
        const float4* lvl = b.super_table + 2ull * ns * k;
        u = box_union(u, box_union(ld_box(lvl + 2ull * lo), ld_box(lvl + 2ull * (hi + 1 - (1u << k)))));
    }
    return u;
}

// The box and traversal record of internal node i, whose leaf range crosses a chunk.
__device__ __forceinline__ void refit_cross_node(const StepBuffers& b, uint32_t n, uint32_t i) {
    const uint32_t leaf_base = n - 1;
    const uint2 rg = b.node_ranges[i];
    const uint2 ch = b.children[i];
    const uint32_t split = ch.x >= leaf_base ? ch.x - leaf_base : ch.x;
    // children's children (Karras: an internal node's left child covers [first, split])
    const uint2 cl = ch.x < leaf_base ? b.children[ch.x] : make_uint2(0u, 0u);
    const uint2 cr = ch.y < leaf_base ? b.children[ch.y] : make_uint2(0u, 0u);
    auto code_of = [&](uint32_t c) { return c >= leaf_base ? (kLeafCode | b.svals[c - leaf_base]) : c; };
    auto split_of = [&](uint32_t left) { return left >= leaf_base ? left - leaf_base : left; };
    // a node's box: a leaf's own, an in-chunk node's from k_refit_leaves, else a range union
    auto box_of = [&](uint32_t c, uint32_t f, uint32_t l) -> Box2 {
        if (c >= leaf_base) return leaf_box(b, leaf_base, f);
        if ((f >> 5) == (l >> 5)) return ld_box(b.node_aabbs + 2ull * c);
        return range_box(b, n, f, l);
    };
    // slots: the left child's entries (one leaf, or its two children), then the right's
    const bool li = ch.x < leaf_base, ri = ch.y < leaf_base;
    TravEntry sl[4];
    sl[1] = sl[3] = {box_empty(), 0u, 0u};
    if (!li) {
        sl[0] = {leaf_box(b, leaf_base, rg.x), code_of(ch.x), rg.x};
    } else {
        const uint32_t s = split_of(cl.x);
        sl[0] = {box_of(cl.x, rg.x, s), code_of(cl.x), s};
        sl[1] = {box_of(cl.y, s + 1, split), code_of(cl.y), split};
    }
    if (!ri) {
        sl[2] = {leaf_box(b, leaf_base, rg.y), code_of(ch.y), rg.y};
    } else {
        const uint32_t s = split_of(cr.x);
        sl[2] = {box_of(cr.x, split + 1, s), code_of(cr.x), s};
        sl[3] = {box_of(cr.y, s + 1, rg.y), code_of(cr.y), rg.y};
    }
    // compacted in leaf order with static indices (no local-memory array)
    const TravEntry e[4] = {sl[0], li ? sl[1] : sl[2], li ? sl[2] : sl[3], sl[3]};
    const uint32_t m = (li ? 2u : 1u) + (ri ? 2u : 1u);
    store_record(b.node_records + 8ull * i, e, m);
    Box2 u = box_empty();
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k)
        if (k < m) u = box_union(u, e[k].box);
    b.node_aabbs[2ull * i] = make_float4(u.mn.x, u.mn.y, u.mn.z, __uint_as_float(rg.y));
    b.node_aabbs[2ull * i + 1] = make_float4(u.mx.x, u.mx.y, u.mx.z, 0.0f);
}

// Cross-chunk internal nodes: their union box and traversal record (in-chunk
// nodes got both from k_refit_leaves, which listed the others; a list keeps
// the warps dense where a grid over every node would leave each with a few
// active lanes).
__global__ void __launch_bounds__(kBlock) k_refit_nodes(StepBuffers b, StepParams p) {
    const uint32_t n = p.collider_count;
    if (n <= 1) return;
    const uint32_t count = b.counts->cross_nodes;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
        refit_cross_node(b, n, b.cross_nodes[q]);
}
// ---------------------------------------------------------------- traverse
__device__ __forceinline__ bool overlaps(float4 amin, float4 amax, float4 bmin, float4 bmax) {
    return amin.x <= bmax.x && amin.y <= bmax.y && amin.z <= bmax.z && bmin.x <= amax.x && bmin.y <= amax.y &&
           bmin.z <= amax.z;
}

// lbvh.wgsl:325-345 (binary search over sorted suppressed body pairs).
__device__ __forceinline__ bool pair_is_suppressed(const uint2* __restrict__ sup, uint32_t count, uint32_t a,
                                                   uint32_t c) {
    const uint32_t low = min(a, c), high = max(a, c);
    uint32_t left = 0, right = count;
    while (left < right) {
        const uint32_t mid = left + (right - left) / 2u;
        const uint2 cand = __ldg(sup + mid);
        if (cand.x < low || (cand.x == low && cand.y < high)) left = mid + 1u;
        else right = mid;
    }
    if (left >= count) return false;
    const uint2 hit = __ldg(sup + left);
    return hit.x == low && hit.y == high;
}

constexpr uint32_t kStack = 64;
constexpr uint32_t kNoNode = 0xffffffffu;
constexpr uint32_t kTravThreads = 128;
constexpr uint32_t kStage = 512;   // pair keys staged per warp in shared memory

// The pair set of lbvh.wgsl:361-398: every collider pair of different,
// unsuppressed bodies whose closed boxes overlap.  Threads take sorted leaves
// in order (neighbouring boxes in a warp walk the same nodes) and look only
// at leaves further right in Morton order, so whole left subtrees are cut off
// and each pair is found once.  A pair is emitted as the key
// (min index << shift) | max index into a per-warp shared-memory stage that
// is flushed with one global reservation; the keys are radix-sorted next,
// which yields the canonical (collider_a, collider_b) order.
template <bool kBatched>
__global__ void __launch_bounds__(kTravThreads) k_traverse(StepBuffers b, StepParams p) {
    __shared__ uint64_t s_stage[kTravThreads / 32][kStage];
    __shared__ uint32_t s_count[kTravThreads / 32];
    const uint32_t n = p.collider_count;
    const uint32_t w = warp_id(), lane = lane_id();
    if (lane == 0) s_count[w] = 0;
    __syncwarp();
    uint32_t* found = &b.counts->pairs_found;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = 0, body_i = 0, node = 0, sp = 0;
    uint32_t stack[kStack];
    float4 qmin = make_float4(0, 0, 0, 0), qmax = qmin;
    bool active = t < n && n > 1;
    if (active) {
        const uint32_t leaf_base = n - 1;
        i = b.svals[t];
        qmin = b.node_aabbs[2ull * (leaf_base + t)];
        qmax = b.node_aabbs[2ull * (leaf_base + t) + 1];
        body_i = __ldg(b.collider_body + i);
        // batched scenes: the walk starts at the scene's own subtree (Karras keeps
        // each scene's leaves under one node: the scene index sits above the
        // Morton bits), so every entry it meets lies inside the scene; a scene of
        // one collider has no pairs
        if (kBatched) {
            const uint32_t sc = b.collider_scene[i];
            const uint32_t begin = sc ? __ldg(b.scene_end + sc - 1) : 0u, end = __ldg(b.scene_end + sc);
            active = end - begin >= 2u;
            if (active) node = __ldg(b.scene_root + sc);
        }
    }
    // The warp steps in lockstep (one record per lane per step, at most four
    // pairs per lane), so the warp's shared-memory stage can be flushed with
    // one global reservation whenever fewer than 128 free entries remain: no
    // pair ever takes a global atomic of its own, however many a warp finds.
    while (__any_sync(0xffffffffu, active)) {
        if (active) {
            const float4* rec = b.node_records + 8ull * node;   // 4-wide: two levels per step
            float4 r[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) r[q] = __ldg(rec + q);
            // the first overlapping internal entry is visited next without a
            // trip through the stack (the pair keys are sorted afterwards, so
            // the visiting order does not matter)
            uint32_t next = kNoNode;
            bool overflow = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float4 cmin = r[2 * k], cmax = r[2 * k + 1];
                if (__float_as_uint(cmax.w) <= t) continue;     // nothing to the right of this leaf below
                if (!overlaps(qmin, qmax, cmin, cmax)) continue;
                const uint32_t code = __float_as_uint(cmin.w);
                if (code & kLeafCode) {
                    const uint32_t j = code & ~kLeafCode;
                    const uint32_t body_j = __ldg(b.collider_body + j);
                    if (body_i == body_j) continue;
                    if (p.suppression_count && pair_is_suppressed(b.suppressed, p.suppression_count, body_i, body_j))
                        continue;
                    const uint64_t key = ((uint64_t)min(i, j) << p.pair_shift) | max(i, j);
                    const uint32_t slot = atomicAdd(&s_count[w], 1u);   // < kStage: flushed below
                    s_stage[w][slot] = key;
                } else if (next == kNoNode) {
                    next = code;
                } else {
                    if (sp >= kStack) {   // lbvh.wgsl:389-392
                        atomicOr(&b.diag->error_flags, MK_PAIR_OVERFLOW_FLAG);
                        overflow = true;
                        break;
                    }
                    stack[sp++] = code;
                }
            }
            if (overflow) {
                active = false;
            } else if (next != kNoNode) {
                node = next;
            } else if (sp == 0) {
                active = false;
            } else {
                node = stack[--sp];
            }
        }
        __syncwarp();
        const uint32_t staged = s_count[w];
        if (staged > kStage - 4u * 32u) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(found, staged);
            base = __shfl_sync(0xffffffffu, base, 0);
            for (uint32_t k = lane; k < staged; k += 32)
                if (base + k < p.pair_capacity) b.pair_stage[base + k] = s_stage[w][k];
            __syncwarp();
            if (lane == 0) s_count[w] = 0;
            __syncwarp();
        }
    }
    __syncwarp();
    const uint32_t staged = s_count[w];
    uint32_t base = 0;
    if (lane == 0 && staged) base = atomicAdd(found, staged);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t k = lane; k < staged; k += 32)
        if (base + k < p.pair_capacity) b.pair_stage[base + k] = s_stage[w][k];
}


// ------------------------------------------------------------- narrowphase
struct Box {
    f3 c;
    float4 q;
    f3 ax[3];
    float h[3];
};

__device__ __forceinline__ Box make_box(const float4* boxes, uint32_t i) {
    const float4* p = boxes + 3ull * i;
    const float4 r0 = __ldg(p), r1 = __ldg(p + 1), r2 = __ldg(p + 2);
    Box o;
    o.c = xyz(r0);
    o.q = r1;
    o.h[0] = r0.w;
    o.h[1] = r2.x;
    o.h[2] = r2.y;
    o.ax[0] = quat_rotate(r1, mkf3(1, 0, 0));
    o.ax[1] = quat_rotate(r1, mkf3(0, 1, 0));
    o.ax[2] = quat_rotate(r1, mkf3(0, 0, 1));
    return o;
}

struct Sat { f3 n; float pen; uint32_t near; uint32_t axis; uint32_t early; };

__device__ __forceinline__ float projection_radius(const Box& o, f3 axis) {
    return fabsf(dot(o.ax[0], axis)) * o.h[0] + fabsf(dot(o.ax[1], axis)) * o.h[1] + fabsf(dot(o.ax[2], axis)) * o.h[2];
}

// collision.wgsl:399-420
__device__ __forceinline__ Sat test_axis(f3 delta, const Box& a, const Box& b, f3 raw, uint32_t idx) {
    const float l2 = dot(raw, raw);
    if (l2 < 1.0e-10f) return {mkf3(1, 0, 0), kFloatMax, 0u, idx, 0u};
    f3 axis = raw * rsqrt_ieee(l2);
    const float sd = dot(delta, axis);
    const float pen = projection_radius(a, axis) + projection_radius(b, axis) - fabsf(sd);
    if (sd < 0.0f) axis = -axis;
    return {axis, pen, 0u, idx, 0u};
}

// collision.wgsl:422-486: axes A0 B0 A1 B1 A2 B2 then Ai x Bj, first negative
// penetration returns immediately.
__device__ Sat obb_sat(const Box& a, const Box& b) {
    const f3 delta = b.c - a.c;
    Sat best = {mkf3(1, 0, 0), kFloatMax, 0u, 0u, 0u};
    uint32_t near = 0;
#pragma unroll
    for (uint32_t i = 0; i < 3; ++i) {
        Sat ra = test_axis(delta, a, b, a.ax[i], 2 * i);
        if (ra.pen < 0.0f) { ra.early = 1; return ra; }
        if (ra.pen <= 1.0e-4f) near += 1;
        if (ra.pen < best.pen) best = ra;
        Sat rb = test_axis(delta, a, b, b.ax[i], 2 * i + 1);
        if (rb.pen < 0.0f) { rb.early = 1; return rb; }
        if (rb.pen <= 1.0e-4f) near += 1;
        if (rb.pen < best.pen) best = rb;
    }
#pragma unroll
    for (uint32_t i = 0; i < 3; ++i)
#pragma unroll
        for (uint32_t j = 0; j < 3; ++j) {
            Sat r = test_axis(delta, a, b, cross(a.ax[i], b.ax[j]), 6 + 3 * i + j);
            if (r.pen < 0.0f) { r.early = 1; return r; }
            if (r.pen < best.pen) best = r;
        }
    best.near = near;
    return best;
}

// collision.wgsl:175-191 (box support) and :240-287 (averaged contact point).
__device__ __forceinline__ f3 support_point(const Box& o, f3 dir) {
    f3 p = o.c;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float proj = dot(o.ax[a], dir);
        if (fabsf(proj) > 1.0e-5f) p = p + o.ax[a] * o.h[a] * sgnf(proj);
    }
    return p;
}
__device__ __forceinline__ f3 vertex(const Box& o, uint32_t v) {
    f3 p = o.c;
#pragma unroll
    for (uint32_t a = 0; a < 3; ++a) {
        const float d = (v & (1u << a)) ? 1.0f : -1.0f;
        p = p + o.ax[a] * o.h[a] * d;
    }
    return p;
}
__device__ __forceinline__ bool contains(const Box& o, f3 pt) {
    const f3 l = quat_rotate(conjq(o.q), pt - o.c);
    return fabsf(l.x) <= o.h[0] + 1.0e-5f && fabsf(l.y) <= o.h[1] + 1.0e-5f && fabsf(l.z) <= o.h[2] + 1.0e-5f;
}
__device__ f3 contact_point(const Box& a, const Box& b, f3 n) {
    f3 sum = mkf3(0, 0, 0);
    float count = 0.0f;
#pragma unroll 1
    for (uint32_t v = 0; v < 8; ++v) {
        const f3 pa = vertex(a, v);
        if (contains(b, pa)) { sum = sum + pa; count += 1.0f; }
        const f3 pb = vertex(b, v);
        if (contains(a, pb)) { sum = sum + pb; count += 1.0f; }
    }
    if (count > 0.0f) return sum / count;
    const f3 pa = support_point(a, n), pb = support_point(b, -n);
    return (pa + pb) * 0.5f;
}

// Clipped manifold (MK_MANIFOLD_CLIPPED): the contact rule of the reference's
// CPU narrowphase (collision.rs:68-103) on the GPU boxes: A's vertices inside B,
// then B's vertices inside A (the containment test of contact_point), later
// points within 1e-5 m of an earlier one dropped, sorted by (x, y, z), the
// first four kept; no contained vertex gives the support midpoint.  Returns
// the number of points (1..4).
__device__ uint32_t manifold_points(const Box& a, const Box& b, f3 n, f3* out) {
    f3 cand[16];
    uint32_t c = 0;
#pragma unroll 1
    for (uint32_t side = 0; side < 2; ++side) {
        const Box& src = side == 0 ? a : b;
        const Box& dst = side == 0 ? b : a;
#pragma unroll 1
        for (uint32_t v = 0; v < 8; ++v) {
            const f3 pt = vertex(src, v);
            if (!contains(dst, pt)) continue;
            bool dup = false;
            for (uint32_t q = 0; q < c; ++q) {
                const f3 d = cand[q] - pt;
                if (!(dot(d, d) > 1.0e-10f)) { dup = true; break; }
            }
            if (!dup) cand[c++] = pt;
        }
    }
    if (c == 0) {
        out[0] = (support_point(a, n) + support_point(b, -n)) * 0.5f;
        return 1;
    }
    // insertion sort by (x, y, z)
    for (uint32_t i = 1; i < c; ++i) {
        const f3 key = cand[i];
        uint32_t j = i;
        while (j > 0) {
            const f3 prv = cand[j - 1];
            const bool greater = prv.x != key.x ? prv.x > key.x : (prv.y != key.y ? prv.y > key.y : prv.z > key.z);
            if (!greater) break;
            cand[j] = prv;
            --j;
        }
        cand[j] = key;
    }
    const uint32_t m = c < 4u ? c : 4u;
    for (uint32_t i = 0; i < m; ++i) out[i] = cand[i];
    return m;
}

__device__ __forceinline__ void store_contact(GpuContact* dst, uint32_t ba, uint32_t bb, uint32_t ca, uint32_t cb,
                                              float4 np, float4 aa, float4 ab) {
    float4* d = reinterpret_cast<float4*>(dst);
    d[0] = make_float4(__uint_as_float(ba), __uint_as_float(bb), __uint_as_float(ca), __uint_as_float(cb));
    d[1] = np;
    d[2] = aa;
    d[3] = ab;
}

// Persistent ordered append over tiles of kBlock items.  The functor decides
// per item whether it emits; emitted items are written in item order.
struct AppendSite {
    uint64_t* states;
    uint32_t* ticket;
};

__device__ __forceinline__ uint32_t take_tile(uint32_t* ticket, uint32_t* s_tile) {
    if (threadIdx.x == 0) *s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    uint32_t t = *s_tile;
    __syncthreads();
    return t;
}

// Heavy ticks with one contact per pair (the averaged point): tiles of
// kNarrowRows rows of kBlock pairs.  Each row's contacts are staged in shared
// memory (normal and depth, point and feature word, bodies and colliders:
// 48 bytes) and the tile takes one ordered-append offset for all its rows, so
// the look-back and the tile's barriers are paid once per 512 pairs.  The
// rows are written in pair order, as with one row per tile.
constexpr uint32_t kNarrowRows = 2;
constexpr uint32_t kNarrowWarps = kBlock / 32;
// Its own kernel, launched after k_narrowphase with the same grid: each leaves
// at once where the other one takes the tick (one register allocation each;
// as one kernel the single-row path spilled more and light ticks slowed).
__device__ __forceinline__ bool narrowphase_takes_rows(const StepParams& p, uint32_t n) {
    return !p.clipped_manifold && n >= 4u * kNarrowRows * kBlock * gridDim.x;
}
__global__ void __launch_bounds__(kBlock, 3) k_narrowphase_rows(StepBuffers b, StepParams p, AppendSite site,
                                                             GpuContact* out, uint64_t* out_keys, uint32_t* out_feat) {
    const uint32_t n = min(b.counts->pairs_found, p.pair_capacity);
    if (!narrowphase_takes_rows(p, n)) return;
    __shared__ float4 s_np[kNarrowRows * kBlock];
    __shared__ float4 s_pt[kNarrowRows * kBlock];
    __shared__ uint4 s_ids[kNarrowRows * kBlock];
    __shared__ uint32_t s_rows[kNarrowRows * kNarrowWarps];
    __shared__ uint32_t s_total;
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_prefix;
    constexpr uint32_t kTile = kNarrowRows * kBlock;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t lane = lane_id(), w = warp_id();
    for (;;) {
        const uint32_t tile = take_tile(site.ticket, &s_tile);
        if (tile >= tiles) break;
        uint32_t emit_rows = 0;
#pragma unroll 1
        for (uint32_t j = 0; j < kNarrowRows; ++j) {
            const uint32_t idx = tile * kTile + j * kBlock + threadIdx.x;
            bool emit = false;
            if (idx < n) {
                const uint64_t key = b.pair_keys[idx];
                const uint2 pr = make_uint2((uint32_t)(key >> p.pair_shift),
                                            (uint32_t)(key & ((1ull << p.pair_shift) - 1)));
                const Box A = make_box(b.boxes, pr.x), Bx = make_box(b.boxes, pr.y);
                const uint32_t ba = __float_as_uint(__ldg(b.boxes + 3ull * pr.x + 2).z);
                const uint32_t bb = __float_as_uint(__ldg(b.boxes + 3ull * pr.y + 2).z);
                const bool skip = b.components && __ldg(b.components + ba) == __ldg(b.components + bb);
                if (!skip) {
                    const Sat st = obb_sat(A, Bx);
                    if (!(st.pen < -1.0e-5f)) {
                        const f3 pt = contact_point(A, Bx, st.n);
                        const uint32_t feat = st.axis | (st.near << 8) | (st.early << 16);
                        const uint32_t slot = j * kBlock + threadIdx.x;
                        s_np[slot] = f4(st.n, mxf(st.pen, 0.0f));
                        s_pt[slot] = f4(pt, __uint_as_float(feat));
                        s_ids[slot] = make_uint4(ba, bb, pr.x, pr.y);
                        emit = true;
                    }
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, emit);
            if (emit) emit_rows |= 1u << j;
            if (lane == 0) s_rows[j * kNarrowWarps + w] = __popc(m);
        }
        __syncthreads();
        // offsets of the (row, warp) groups in pair order, then the tile's prefix
        if (w == 0) {
            const uint32_t c = lane < kNarrowRows * kNarrowWarps ? s_rows[lane] : 0u;
            const uint32_t inc = warp_inclusive_scan(c);
            if (lane < kNarrowRows * kNarrowWarps) s_rows[lane] = inc - c;
            const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
            const uint64_t pre = tile_lookback(site.states, tile, total, &b.diag->error_flags);
            if (lane == 0) {
                s_prefix = pre;
                s_total = total;
            }
        }
        __syncthreads();
        const uint64_t pre = s_prefix;
        const uint32_t below = (1u << lane) - 1u;
#pragma unroll 1
        for (uint32_t j = 0; j < kNarrowRows; ++j) {
            const bool emit = (emit_rows >> j) & 1u;
            const uint32_t m = __ballot_sync(0xffffffffu, emit);
            if (!emit) continue;
            const uint64_t o = pre + s_rows[j * kNarrowWarps + w] + __popc(m & below);
            if (o >= p.pair_capacity) continue;
            const uint32_t slot = j * kBlock + threadIdx.x;
            const float4 np = s_np[slot], pt4 = s_pt[slot];
            const uint4 ids = s_ids[slot];
            const uint32_t feat = __float_as_uint(pt4.w);
            const f3 pt = xyz(pt4);
            const f3 xa = xyz(b.pos[ids.x]), xb = xyz(b.pos[ids.y]);
            store_contact(out + o, ids.x, ids.y, ids.z, ids.w, np, f4(pt - xa, 0.0f),
                          f4(pt - xb, (float)((feat >> 8) & 0xffu)));
            out_keys[o] = ((uint64_t)ids.z << 32) | ids.w;
            out_feat[o] = feat;
        }
        if (tile == tiles - 1 && threadIdx.x == 0) {
            const uint64_t all = pre + s_total;
            b.counts->narrow = (uint32_t)umin64(all, p.pair_capacity);
            b.counts->requested_contacts = (uint32_t)umin64(all, 0xffffffffull);
        }
        __syncthreads();
    }
}

// collision.wgsl:570-620 (narrowphase with the optional self-collision filter).
__global__ void __launch_bounds__(kBlock, 3) k_narrowphase(StepBuffers b, StepParams p, AppendSite site,
                                                        GpuContact* out, uint64_t* out_keys, uint32_t* out_feat) {
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_prefix;
    // the tick's pair count (diag[1] keeps the requested count, lbvh.wgsl:353-358)
    const uint32_t found = b.counts->pairs_found;
    const uint32_t n = min(found, p.pair_capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.diag->pair_count = found;
        b.counts->pairs = n;
        if (found > p.pair_capacity) atomicOr(&b.diag->error_flags, MK_PAIR_OVERFLOW_FLAG);
    }
    const uint32_t tiles = (n + kBlock - 1) / kBlock;
    // the grid is sized for the capacity: CTAs past the tile count leave
    // before taking a ticket (block 0 stays for the empty-list counts)
    if (blockIdx.x != 0 && blockIdx.x >= tiles) return;
    // several rows per tile (k_narrowphase_rows) only where every CTA still gets four tiles of them
    if (narrowphase_takes_rows(p, n)) return;
    for (;;) {
        const uint32_t tile = take_tile(site.ticket, &s_tile);
        if (tile >= tiles) break;
        const uint32_t idx = tile * kBlock + threadIdx.x;
        uint32_t emit = 0;
        uint2 pr = make_uint2(0, 0);
        Sat s;
        f3 pts[4];
        uint32_t ba = 0, bb = 0;
        if (idx < n) {
            const uint64_t key = b.pair_keys[idx];
            pr = make_uint2((uint32_t)(key >> p.pair_shift), (uint32_t)(key & ((1ull << p.pair_shift) - 1)));
            const Box A = make_box(b.boxes, pr.x), Bx = make_box(b.boxes, pr.y);
            ba = __float_as_uint(__ldg(b.boxes + 3ull * pr.x + 2).z);
            bb = __float_as_uint(__ldg(b.boxes + 3ull * pr.y + 2).z);
            bool skip = b.components && __ldg(b.components + ba) == __ldg(b.components + bb);
            if (!skip) {
                s = obb_sat(A, Bx);
                if (!(s.pen < -1.0e-5f)) {
                    if (p.clipped_manifold) {
                        emit = manifold_points(A, Bx, s.n, pts);
                    } else {
                        pts[0] = contact_point(A, Bx, s.n);
                        emit = 1;
                    }
                }
            }
        }
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(emit, s_scan, &total);
        if (warp_id() == 0) {
            uint64_t pre = tile_lookback(site.states, tile, total, &b.diag->error_flags);
            if (lane_id() == 0) s_prefix = pre;
        }
        __syncthreads();
        const uint64_t pre = s_prefix;
        if (emit) {
            const f3 xa = xyz(b.pos[ba]), xb = xyz(b.pos[bb]);
            for (uint32_t q = 0; q < emit; ++q) {
                const uint64_t o = pre + ex + q;
                if (o >= p.pair_capacity) break;
                store_contact(out + o, ba, bb, pr.x, pr.y, f4(s.n, mxf(s.pen, 0.0f)), f4(pts[q] - xa, 0.0f),
                              f4(pts[q] - xb, (float)s.near));
                out_keys[o] = ((uint64_t)pr.x << 32) | pr.y;
                out_feat[o] = s.axis | (s.near << 8) | (s.early << 16) | (q << 25);
            }
        }
        if (tile == tiles - 1 && threadIdx.x == 0) {
            const uint64_t all = pre + total;
            b.counts->narrow = (uint32_t)umin64(all, p.pair_capacity);
            b.counts->requested_contacts = (uint32_t)umin64(all, 0xffffffffull);
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && tiles == 0) {
        b.counts->narrow = 0;
        b.counts->requested_contacts = 0;
    }
}

// collision.wgsl:175-238 and :622-664: analytic contact with the y = 0 plane.
// One collider's analytic ground contact: support point (or analytic rim
// point of a full cylinder segment) and whether it emits.
__device__ __forceinline__ bool ground_point(const StepBuffers& b, uint32_t i, f3& sp, uint32_t& body,
                                             uint32_t& role) {
    const Box o = make_box(b.boxes, i);
    const float4 r2 = __ldg(b.boxes + 3ull * i + 2);
    body = __float_as_uint(r2.z);
    role = __float_as_uint(r2.w);
    const f3 down = mkf3(0, -1, 0);
    sp = support_point(o, down);
    if (role != 0u) {
        const float center_radius = __ldg(b.colliders + 4ull * i).w;
        const float outer_radius = __ldg(b.colliders + 4ull * i + 2).w;
        const f3 caxis = o.ax[1];
        const float ap = dot(caxis, down);
        const f3 radial = down - caxis * ap;
        const float rl = length(radial);
        const uint32_t cc = rl < 0.05f ? 4u : 1u;
        if (role > cc) return false;
        f3 q = o.c - o.ax[0] * center_radius;
        if (rl < 0.05f) {
            q = q + caxis * sgnf(ap) * o.h[1];
            const f3 ta = normalize(mkf3(1, 0, 0) - caxis * caxis.x);
            const f3 tb = normalize(cross(caxis, ta));
            if (role == 1u) q = q + ta * outer_radius;
            else if (role == 2u) q = q - ta * outer_radius;
            else if (role == 3u) q = q + tb * outer_radius;
            else q = q - tb * outer_radius;
        } else {
            q = q + radial * (outer_radius / rl);
            if (fabsf(ap) >= 0.05f) q = q + caxis * sgnf(ap) * o.h[1];
        }
        sp = q;
    }
    return !(sp.y > 1.0e-5f);
}

// Ground contacts in collider order after the narrowphase's.  k_collider_bounds
// left a bit per collider and a count per tile of kGroundTile colliders, so a
// tile's output offset is the sum of the earlier tiles' counts (no look-back
// chain) and only the touching colliders' boxes are read again.  Each thread
// takes kGroundItems consecutive colliders of its tile.
constexpr uint32_t kGroundItems = kGroundTile / kBlock;
__global__ void __launch_bounds__(kBlock) k_ground(StepBuffers b, StepParams p, GpuContact* out, uint64_t* out_keys,
                                                   uint32_t* out_feat) {
    __shared__ uint32_t s_scan[33];
    const uint32_t n = p.collider_count;
    const uint32_t tiles = (n + kGroundTile - 1) / kGroundTile;
    const uint32_t narrow = b.counts->narrow;
    const uint32_t requested_narrow = b.counts->requested_contacts;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint32_t part = 0;
        for (uint32_t q = threadIdx.x; q < tile; q += blockDim.x) part += __ldg(b.ground_tile_count + q);
        uint32_t pre;
        block_exclusive_scan(part, s_scan, &pre);   // pre = touching colliders of the tiles before this one
        const uint32_t first = tile * kGroundTile + threadIdx.x * kGroundItems;   // 4-aligned: one mask word
        const uint32_t mask = first < n ? (__ldg(b.ground_mask + (first >> 5)) >> (first & 31u)) & 0xfu : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan((uint32_t)__popc(mask), s_scan, &total);
        uint32_t q = 0;
        for (uint32_t k = 0; k < kGroundItems; ++k) {
            if (!((mask >> k) & 1u)) continue;
            const uint32_t i = first + k;
            f3 sp;
            uint32_t body, role;
            ground_point(b, i, sp, body, role);
            const uint64_t o = (uint64_t)narrow + pre + ex + q++;
            if (o < p.pair_capacity) {
                store_contact(out + o, body, kInvalid, i, kInvalid, make_float4(0.0f, -1.0f, 0.0f, mxf(-sp.y, 0.0f)),
                              f4(sp - xyz(b.pos[body]), 0.0f), make_float4(0.0f, 0.0f, 0.0f, role != 0u ? -1.0f : 0.0f));
                out_keys[o] = ((uint64_t)i << 32) | kInvalid;
                out_feat[o] = 0xffffu;
            }
        }
        if (tile == tiles - 1 && threadIdx.x == 0) {
            const uint64_t all = (uint64_t)requested_narrow + pre + total;
            const uint64_t stored = (uint64_t)narrow + pre + total;
            b.counts->contacts = (uint32_t)umin64(stored, p.pair_capacity);
            b.diag->contact_count = (uint32_t)umin64(all, 0xffffffffull);
            if (all > p.pair_capacity) atomicOr(&b.diag->error_flags, MK_PAIR_OVERFLOW_FLAG);
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && tiles == 0) {
        b.counts->contacts = narrow;
        b.diag->contact_count = requested_narrow;
    }
}

// ------------------------------------------------------------ contact solve
__device__ __forceinline__ f3 contact_velocity(const StepBuffers& b, uint32_t body, f3 arm) {
    return xyz(b.lin[body]) + cross(xyz(b.ang[body]), arm);
}

// Manifold lookup: the previous tick's contact list is sorted by
// (collider_a, collider_b) within its narrowphase part and its ground part.
__device__ __forceinline__ int64_t find_previous(const uint64_t* __restrict__ keys, uint32_t lo, uint32_t end,
                                                 uint64_t key) {
    uint32_t hi = end;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const uint64_t k = __ldg(keys + mid);
        if (k < key) lo = mid + 1u;
        else hi = mid;
    }
    return (lo < end && __ldg(keys + lo) == key) ? (int64_t)lo : -1;
}

// collision.wgsl:674-736 with the persistent manifold of the previous tick
// read from its contact list (acquired rows carry feature bit 24).
// A tile is `rows` rows of kBlock contacts (contact k of row j is
// (tile * rows + j) * kBlock + threadIdx.x), with rows = 1..kPrepareItems
// chosen from the count so that every CTA of the grid still gets at least
// four tiles: on the heaviest ticks the ordered append's look-back frontier,
// which advances 32 tiles per L2 round trip, then covers up to 8 x the
// contacts per round trip (9.5M contacts: 7 rows, 5,285 tiles instead of
// 36,991), while smaller counts keep one row per tile and every contact's
// lookup in flight at once.
constexpr uint32_t kPrepareItems = 8;
constexpr uint32_t kPrepareWarps = kBlock / 32;
__global__ void __launch_bounds__(kBlock) k_prepare(StepBuffers b, StepParams p, AppendSite site, GpuContact* cur,
                                                    uint64_t* cur_keys, uint32_t* cur_feat, const GpuContact* prev,
                                                    const uint64_t* prev_keys, const uint32_t* prev_feat) {
    __shared__ uint32_t s_rows[kPrepareItems * kPrepareWarps];   // active count of each (row, warp), then its offset
    __shared__ uint32_t s_total;
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_prefix;
    const uint32_t n = b.counts->contacts;
    const uint32_t rows = min(kPrepareItems, max(1u, n / (4u * kBlock * gridDim.x)));
    const uint32_t tile_contacts = rows * kBlock;
    const uint32_t tiles = (n + tile_contacts - 1) / tile_contacts;
    const uint32_t tick = b.tick->tick_index;
    const bool prev_ok = b.counts->prev_valid != 0u && b.counts->prev_tick == tick - 1u;
    const uint32_t prev_narrow = b.counts->prev_narrow, prev_all = b.counts->prev_contacts;
    // run index: [parity][0 narrow, 1 ground][collider] = {tick, first row of the collider's rows}
    const uint64_t C = p.collider_count;
    uint2* index_cur = b.contact_index + 2ull * C * (tick & 1u);
    const uint2* index_prev = b.contact_index + 2ull * C * ((tick - 1u) & 1u);
    const bool indexed = prev_ok && b.counts->prev_indexed != 0u;
    const uint32_t narrow_now = b.counts->narrow;
    if (blockIdx.x != 0 && blockIdx.x >= tiles) return;   // as in k_narrowphase
    const uint32_t lane = lane_id(), w = warp_id();
    for (;;) {
        const uint32_t tile = take_tile(site.ticket, &s_tile);
        if (tile >= tiles) break;
        uint32_t act_rows = 0;   // bit j: this thread's contact of row j is active
#pragma unroll 1
        for (uint32_t j = 0; j < rows; ++j) {
            const uint32_t k = tile * tile_contacts + j * kBlock + threadIdx.x;
            bool act = false;
            if (k < n) {
                {   // index this tick's list for the next tick's lookups
                    const uint64_t key = cur_keys[k];
                    const uint32_t ca = (uint32_t)(key >> 32);
                    if (k >= narrow_now) index_cur[C + ca] = make_uint2(tick, k);            // one ground row per collider
                    else if (k == 0 || (uint32_t)(cur_keys[k - 1] >> 32) != ca) index_cur[ca] = make_uint2(tick, k);
                }
                float4* row = reinterpret_cast<float4*>(cur + k);
                const float4 r0 = row[0], np = row[1], aa = row[2], ab = row[3];
                const uint32_t a = __float_as_uint(r0.x), bb = __float_as_uint(r0.y);
                const f3 arm_a = xyz(aa), arm_b = xyz(ab);
                float inv_b = 0.0f;
                f3 vb = mkf3(0, 0, 0);
                if (bb != kInvalid) {
                    inv_b = b.world_mass[3ull * bb].w;
                    vb = contact_velocity(b, bb, arm_b);
                }
                if (!(b.world_mass[3ull * a].w + inv_b <= 0.0f)) {
                    const f3 rel = vb - contact_velocity(b, a, arm_a);
                    const f3 nrm = xyz(np);
                    const float vn = dot(rel, nrm);
                    if (np.w <= 1.0e-6f && vn >= 0.0f) {
                        row[0] = make_float4(r0.x, r0.y, __uint_as_float(kInvalid), __uint_as_float(0u));
                    } else {
                        float cached = 0.0f;
                        if (prev_ok) {
                            // the previous rows of this collider pair (one, or up to four with a
                            // clipped manifold): the first acquired row whose normal and arm match
                            const uint64_t key = cur_keys[k];
                            const bool ground = (uint32_t)key == kInvalid;
                            const uint32_t end = ground ? prev_all : prev_narrow;
                            int64_t m = -1;
                            if (indexed) {   // the collider's run, then a short scan to the key
                                const uint32_t ca = (uint32_t)(key >> 32);
                                const uint2 e = __ldg(index_prev + (ground ? C : 0ull) + ca);
                                if (e.x == tick - 1u) {
                                    uint32_t r = e.y;
                                    while (r < end && __ldg(prev_keys + r) < key && (uint32_t)(__ldg(prev_keys + r) >> 32) == ca)
                                        ++r;
                                    if (r < end && __ldg(prev_keys + r) == key) m = r;
                                }
                            } else {
                                m = ground ? find_previous(prev_keys, prev_narrow, prev_all, key)
                                           : find_previous(prev_keys, 0u, prev_narrow, key);
                            }
                            for (int64_t r = m; r >= 0 && r < (int64_t)end && __ldg(prev_keys + r) == key; ++r) {
                                if (!(__ldg(prev_feat + r) & (1u << 24))) continue;
                                const float4* pr = reinterpret_cast<const float4*>(prev + r);
                                const float4 pn = __ldg(pr + 1), pa = __ldg(pr + 2);
                                const bool match = dot(xyz(pn), nrm) >= 0.98f && length(xyz(pa) - arm_a) <= 0.02f;
                                if (match) {
                                    cached = pa.w;
                                    break;
                                }
                            }
                        }
                        row[0] = make_float4(r0.x, r0.y, __uint_as_float(k), __uint_as_float(1u));
                        row[2] = f4(arm_a, cached);
                        cur_feat[k] |= 1u << 24;
                        act = np.w > 1.0e-5f || vn < -1.0e-5f || cached > 1.0e-6f;
                    }
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, act);
            if (act) act_rows |= 1u << j;
            if (lane == 0) s_rows[j * kPrepareWarps + w] = __popc(m);
        }
        __syncthreads();
        // offsets of the (row, warp) groups in contact order, then the tile's prefix
        if (w == 0) {
            uint32_t carry = 0;
            for (uint32_t e0 = 0; e0 < rows * kPrepareWarps; e0 += 32) {
                const uint32_t e = e0 + lane;
                const uint32_t c = e < rows * kPrepareWarps ? s_rows[e] : 0u;
                const uint32_t inc = warp_inclusive_scan(c);
                if (e < rows * kPrepareWarps) s_rows[e] = carry + inc - c;
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            const uint64_t pre = tile_lookback(site.states, tile, carry, &b.diag->error_flags);
            if (lane == 0) {
                s_prefix = pre;
                s_total = carry;
            }
        }
        __syncthreads();
        const uint64_t pre = s_prefix;
        const uint32_t below = (1u << lane) - 1u;
#pragma unroll 1
        for (uint32_t j = 0; j < rows; ++j) {
            const bool act = (act_rows >> j) & 1u;
            const uint32_t m = __ballot_sync(0xffffffffu, act);
            if (act)
                b.active[pre + s_rows[j * kPrepareWarps + w] + __popc(m & below)] =
                    tile * tile_contacts + j * kBlock + threadIdx.x;
        }
        if (tile == tiles - 1 && threadIdx.x == 0) {
            b.counts->active = (uint32_t)(pre + s_total);
            b.diag->active_contact_count = (uint32_t)(pre + s_total);
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && tiles == 0) {
        b.counts->active = 0;
        b.diag->active_contact_count = 0;
    }
}

__device__ __forceinline__ f3 inverse_inertia(const float4* wm, f3 v) {
    return xyz(wm[0]) * v.x + xyz(wm[1]) * v.y + xyz(wm[2]) * v.z;
}

// collision.wgsl:116-132
__device__ __forceinline__ float impulse_denominator(const float4* wa, const float4* wb, f3 arm_a, f3 arm_b, f3 d) {
    float r = wa[0].w;
    const f3 ang_a = cross(inverse_inertia(wa, cross(arm_a, d)), arm_a);
    r += dot(ang_a, d);
    if (wb) {
        r += wb[0].w;
        const f3 ang_b = cross(inverse_inertia(wb, cross(arm_b, d)), arm_b);
        r += dot(ang_b, d);
    }
    return r;
}

// Segmented sum over runs of equal `key` in consecutive lanes; the last lane
// of each run returns the run total (others return garbage) in *v.
__device__ __forceinline__ bool run_tail_sum(uint32_t key, int32_t* v, int n) {
    const uint32_t lane = lane_id();
    const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    const uint32_t next = __shfl_down_sync(0xffffffffu, key, 1);
    const bool head = lane == 0 || prev != key;
    const bool tail = lane == 31 || next != key;
    const uint32_t heads = __ballot_sync(0xffffffffu, head);
    // distance to the run head
    const uint32_t below = heads & ((2u << lane) - 1u);
    const uint32_t head_lane = 31u - __clz(below);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            if (c >= n) break;
            const int32_t u = __shfl_up_sync(0xffffffffu, v[c], o);
            if (lane >= head_lane + (uint32_t)o) v[c] = (int32_t)((uint32_t)v[c] + (uint32_t)u);
        }
    }
    return tail;
}

// collision.wgsl:774-906 for the active contacts [first, A) in strides of
// `stride`.  kWarm: warm_start (iteration 0), else solve_accumulate.  The
// velocities of iteration k live in their own buffer pair (vl, va), written
// by the previous phase and never written again in this launch, so they are
// read through the L1/texture path; contact rows and deltas change between
// phases of the launch and are read through L2 (ld.cg).
__device__ __forceinline__ f3 contact_velocity_it(const float4* vl, const float4* va, uint32_t body, f3 arm) {
    return xyz(__ldg(vl + body)) + cross(xyz(__ldg(va + body)), arm);
}

// Fused pass (light ticks): a pass computes the velocities of its contacts'
// bodies itself, as the apply of the previous pass would (V_k = V_{k-1} +
// D_{k-1} / 2^20, the same float operations), stores them as V_k for the next
// pass, and accumulates into the next of three rotating delta buffers, so a
// pass needs one grid barrier and no apply over all bodies.
struct FusedPass {
    uint32_t it;                 // pass index
    const float4 *pl, *pa;       // V_{it-1} (it > 0), or V_0 (it == 0)
    const int32_t* dprev;        // D_{it-1}
    float4 *cl, *ca;             // V_it (it > 0)
    uint32_t gen;                // generation stamped on touched bodies (pass 0)
};

__device__ __forceinline__ void fused_body(const StepBuffers& b, const FusedPass& f, uint32_t x, f3& lin, f3& ang) {
    if (f.it == 0) {
        lin = xyz(__ldg(f.pl + x));
        ang = xyz(__ldg(f.pa + x));
        b.body_stamp[x] = f.gen;
        return;
    }
    const float s = (float)kFixedScale;
    const int2* d2 = reinterpret_cast<const int2*>(f.dprev + 6ull * x);
    const int2 x0 = __ldcg(d2), x1 = __ldcg(d2 + 1), x2 = __ldcg(d2 + 2);
    const f3 ld = mkf3((float)x0.x, (float)x0.y, (float)x1.x) / s;
    const f3 ad = mkf3((float)x1.y, (float)x2.x, (float)x2.y) / s;
    const float4 nl = f4(xyz(__ldg(f.pl + x)) + ld, 0.0f);
    const float4 na = f4(xyz(__ldg(f.pa + x)) + ad, 0.0f);
    f.cl[x] = nl;   // every contact of the body stores the same value
    f.ca[x] = na;
    lin = xyz(nl);
    ang = xyz(na);
}

// One relaxed-Jacobi projection of a contact (collision.wgsl:774-906) at the
// relative velocity `rel` (vB - vA at the arms).  `acc` holds the row's stored
// impulse on entry and the value the row keeps on return; returns whether an
// impulse is applied (then da / db hold its fixed-point body deltas).
template <bool kWarm>
__device__ __forceinline__ bool contact_project(const StepParams& p, const float4* wa, const float4* wb, f3 arm_a,
                                                f3 arm_b, f3 nrm, float depth, bool cyl, float den, f3 rel,
                                                float& acc_io, int32_t* da, int32_t* db) {
    const float scale = (float)kFixedScale;
    const float vn = dot(rel, nrm);
    if (depth <= 1.0e-5f && vn >= -1.0e-5f && acc_io <= 1.0e-6f) {
        acc_io = 0.0f;
        return false;
    }
    const float recovery = cyl ? 1.0f : 0.2f;
    const float bias = mnf(mxf(depth - 0.001f, 0.0f) * recovery / p.dt, 1.0f);
    float acc, delta;
    if (kWarm) {
        const float warmed = acc_io * (cyl ? 1.0f : 0.5f);
        acc = mxf(warmed + 0.125f * (-vn + bias) / den, 0.0f);
        delta = acc;
    } else {
        const float prev = mxf(acc_io, 0.0f);
        acc = mxf(prev + 0.125f * (-vn + bias) / den, 0.0f);
        delta = acc - prev;
    }
    acc_io = acc;
    f3 imp = nrm * delta;
    const f3 tv = rel - nrm * vn;
    const float ts = length(tv);
    if (ts > 1.0e-6f) {
        const f3 tg = tv / ts;
        const float tden = impulse_denominator(wa, wb, arm_a, arm_b, tg);
        const float fr = mnf(ts / tden, (kWarm ? acc : fabsf(delta)) * 0.05f);
        imp = imp - tg * fr;
    }
    const f3 la = -imp * wa[0].w;
    const f3 ga = inverse_inertia(wa, cross(arm_a, -imp));
    da[0] = fixed_i32(la.x * scale); da[1] = fixed_i32(la.y * scale); da[2] = fixed_i32(la.z * scale);
    da[3] = fixed_i32(ga.x * scale); da[4] = fixed_i32(ga.y * scale); da[5] = fixed_i32(ga.z * scale);
    if (wb) {
        const f3 lb = imp * wb[0].w;
        const f3 gb = inverse_inertia(wb, cross(arm_b, imp));
        db[0] = fixed_i32(lb.x * scale); db[1] = fixed_i32(lb.y * scale); db[2] = fixed_i32(lb.z * scale);
        db[3] = fixed_i32(gb.x * scale); db[4] = fixed_i32(gb.y * scale); db[5] = fixed_i32(gb.z * scale);
    }
    return true;
}

// Adds a contact's body deltas: body A's through warp sums over runs of equal
// bodies (contacts arrive grouped by collider A; integer sums are order-free),
// body B's directly.
__device__ __forceinline__ void add_contact_deltas(int32_t* deltas, bool live, uint32_t a, uint32_t bb, int32_t* da,
                                                   const int32_t* db) {
    const uint32_t key_a = live ? a : kInvalid;
    const bool tail = run_tail_sum(key_a, da, 6);
    if (tail && key_a != kInvalid) {
        int32_t* d = deltas + 6ull * key_a;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            if (da[c]) atomicAdd(d + c, da[c]);
    }
    if (live && bb != kInvalid) {
        int32_t* d = deltas + 6ull * bb;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            if (db[c]) atomicAdd(d + c, db[c]);
    }
}

// This block's contiguous, warp-aligned slice [x, y) of the A active contacts:
// every SM gets about A / blocks of them (a pass is issue bound on the SMs
// that hold contacts, so whole 1024-contact blocks on a few SMs left the
// others idle).  Contacts keep their order inside a warp.
__device__ __forceinline__ uint2 contact_slice(uint32_t A, uint32_t blocks) {
    const uint32_t per = ((A + blocks - 1u) / blocks + 31u) & ~31u;
    const uint32_t begin = (uint32_t)min((uint64_t)A, (uint64_t)blockIdx.x * per);
    return make_uint2(begin, min(A, begin + per));
}

// The contacts [sl.x, sl.y) of this block, blockDim.x at a time.
template <bool kWarm, bool kFused = false>
__device__ __forceinline__ void solve_span(const StepBuffers& b, const StepParams& p, GpuContact* cur, uint2 sl,
                                           const float4* vl, const float4* va, const FusedPass* fp = nullptr,
                                           int32_t* dacc = nullptr) {
    int32_t* deltas = kFused ? dacc : b.deltas;
    for (uint32_t base = sl.x; base < sl.y; base += blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        bool live = false;
        uint32_t a = kInvalid, bb = kInvalid;
        int32_t da[6] = {0, 0, 0, 0, 0, 0}, db[6] = {0, 0, 0, 0, 0, 0};
        if (t < sl.y) {
            const uint32_t k = __ldcg(b.active + t);
            float4* row = reinterpret_cast<float4*>(cur + k);
            const float4 r0 = __ldcg(row), np = __ldcg(row + 1), aa = __ldcg(row + 2), ab = __ldcg(row + 3);
            a = __float_as_uint(r0.x);
            bb = __float_as_uint(r0.y);
            const f3 arm_a = xyz(aa), arm_b = xyz(ab);
            const float4* wa = b.world_mass + 3ull * a;
            const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
            f3 la = mkf3(0, 0, 0), ga = mkf3(0, 0, 0), lb = mkf3(0, 0, 0), gb = mkf3(0, 0, 0);
            if (kFused) {
                fused_body(b, *fp, a, la, ga);
                if (bb != kInvalid) fused_body(b, *fp, bb, lb, gb);
            }
            f3 vb = mkf3(0, 0, 0);
            if (bb != kInvalid) vb = kFused ? lb + cross(gb, arm_b) : contact_velocity_it(vl, va, bb, arm_b);
            const f3 nrm = xyz(np);
            const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
            if (!(den <= 0.0f)) {
                const f3 rel = vb - (kFused ? la + cross(ga, arm_a) : contact_velocity_it(vl, va, a, arm_a));
                float acc = aa.w;
                live = contact_project<kWarm>(p, wa, wb, arm_a, arm_b, nrm, np.w, ab.w < 0.0f, den, rel, acc, da, db);
                row[2] = f4(arm_a, acc);
            }
        }
        add_contact_deltas(deltas, live, a, bb, da, db);
    }
}

// collision.wgsl:1050-1069: v += delta / 2^20 (from the iteration's buffer
// into the next one), then clear the delta.
__device__ __forceinline__ void apply_span(const StepBuffers& b, const StepParams& p, uint32_t first,
                                           uint32_t stride, const float4* sl, const float4* sa, float4* dl,
                                           float4* da) {
    const float s = (float)kFixedScale;
    for (uint32_t i = first; i < p.body_count; i += stride) {
        int2* d2 = reinterpret_cast<int2*>(b.deltas + 6ull * i);   // 24-byte rows are 8-byte aligned
        const int2 x0 = __ldcg(d2), x1 = __ldcg(d2 + 1), x2 = __ldcg(d2 + 2);
        if ((x0.x | x0.y | x1.x | x1.y | x2.x | x2.y) != 0) {
            d2[0] = make_int2(0, 0);
            d2[1] = make_int2(0, 0);
            d2[2] = make_int2(0, 0);
        }
        const f3 ld = mkf3((float)x0.x, (float)x0.y, (float)x1.x) / s;
        const f3 ad = mkf3((float)x1.y, (float)x2.x, (float)x2.y) / s;
        dl[i] = f4(xyz(__ldg(sl + i)) + ld, 0.0f);
        da[i] = f4(xyz(__ldg(sa + i)) + ad, 0.0f);
    }
}

// Fused passes with one contact per thread held in registers for the whole
// solve (active contacts <= threads of the grid): the contact row, its
// normal-row denominator and its running impulse are loaded once, so a pass
// reads only the two bodies' velocity state.  Each pass also clears its
// bodies' rows of the delta buffer the next pass accumulates into (the active
// contacts touch the same bodies in every pass; rows of other bodies are never
// read).  The row keeps the last pass's impulse, as after per-pass stores.
__device__ __forceinline__ void solve_fused_resident(const StepBuffers& b, const StepParams& p, GpuContact* cur,
                                                  uint32_t A, uint32_t iterations, int32_t* const* D,
                                                  uint32_t gen, uint32_t* barrier, uint32_t parts) {
    const uint2 sl = contact_slice(A, parts);   // at most blockDim.x contacts: A <= parts * blockDim.x
    const uint32_t t = sl.x + threadIdx.x;
    const bool has = t < sl.y;
    uint32_t a = kInvalid, bb = kInvalid;
    f3 arm_a = mkf3(0, 0, 0), arm_b = mkf3(0, 0, 0), nrm = mkf3(0, 0, 0);
    float depth = 0.0f, acc = 0.0f, den = 0.0f;
    bool cyl = false;
    float4* row = nullptr;
    if (has) {
        const uint32_t k = __ldcg(b.active + t);
        row = reinterpret_cast<float4*>(cur + k);
        const float4 r0 = __ldcg(row), np = __ldcg(row + 1), aa = __ldcg(row + 2), ab = __ldcg(row + 3);
        a = __float_as_uint(r0.x);
        bb = __float_as_uint(r0.y);
        arm_a = xyz(aa);
        arm_b = xyz(ab);
        nrm = xyz(np);
        depth = np.w;
        acc = aa.w;
        cyl = ab.w < 0.0f;
        den = impulse_denominator(b.world_mass + 3ull * a, bb != kInvalid ? b.world_mass + 3ull * bb : nullptr,
                                  arm_a, arm_b, nrm);
    }
    const size_t B = p.body_count;
    for (uint32_t it = 0; it < iterations; ++it) {
        FusedPass fp;
        fp.it = it;
        fp.pl = it <= 1 ? b.lin : b.vel_iter + (2 * (it - 2)) * B;
        fp.pa = it <= 1 ? b.ang : b.vel_iter + (2 * (it - 2) + 1) * B;
        fp.dprev = it == 0 ? nullptr : D[(it - 1) % 3];
        fp.cl = it == 0 ? nullptr : b.vel_iter + (2 * (it - 1)) * B;
        fp.ca = it == 0 ? nullptr : b.vel_iter + (2 * (it - 1) + 1) * B;
        fp.gen = gen;
        bool live = false;
        int32_t da[6] = {0, 0, 0, 0, 0, 0}, db[6] = {0, 0, 0, 0, 0, 0};
        if (has) {
            f3 la, ga, lb = mkf3(0, 0, 0), gb = mkf3(0, 0, 0);
            fused_body(b, fp, a, la, ga);
            if (bb != kInvalid) fused_body(b, fp, bb, lb, gb);
            int2* za = reinterpret_cast<int2*>(D[(it + 1) % 3] + 6ull * a);   // 24-byte rows: 8-byte aligned
            za[0] = make_int2(0, 0); za[1] = make_int2(0, 0); za[2] = make_int2(0, 0);
            if (bb != kInvalid) {
                int2* zb = reinterpret_cast<int2*>(D[(it + 1) % 3] + 6ull * bb);
                zb[0] = make_int2(0, 0); zb[1] = make_int2(0, 0); zb[2] = make_int2(0, 0);
            }
            if (!(den <= 0.0f)) {
                const float4* wa = b.world_mass + 3ull * a;
                const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
                const f3 vb = bb != kInvalid ? lb + cross(gb, arm_b) : mkf3(0, 0, 0);
                const f3 rel = vb - (la + cross(ga, arm_a));
                live = it == 0 ? contact_project<true>(p, wa, wb, arm_a, arm_b, nrm, depth, cyl, den, rel, acc, da, db)
                               : contact_project<false>(p, wa, wb, arm_a, arm_b, nrm, depth, cyl, den, rel, acc, da,
                                                        db);
            }
        }
        add_contact_deltas(D[it % 3], live, a, bb, da, db);
        grid_barrier(barrier, &b.diag->error_flags, parts);
    }
    if (has && !(den <= 0.0f)) row[2] = f4(arm_a, acc);
}

// ------------------------------------------- gather form of the contact solve
// On heavy ticks (more active contacts than twice the bodies, e.g. an
// overlapping start with dozens of contacts per body) the atomics of the
// scatter form serialise on the bodies' 24-byte delta rows.  This form writes
// each contact's twelve fixed-point deltas to its own slot instead, and each
// body then sums the slots of its contacts through an incidence list built
// once per tick (counts, a grid scan, a fill).  The integer sums wrap as the
// atomics do and are order-free, so the velocities are bit-identical to the
// scatter form (and to the reference's atomic Jacobi, collision.wgsl:752-1069).

// Exclusive scan of inc_count[0, B) into inc_off over the grid: each
// participating block scans a contiguous segment after adding up the totals
// of the segments before it (published in inc_blocks).
__device__ __forceinline__ void gather_scan(const StepBuffers& b, uint32_t B, uint32_t parts, uint32_t* barrier,
                                            uint32_t* flags, uint32_t* s_scan) {
    const uint32_t seg = (B + parts - 1) / parts;
    const uint32_t lo = min(B, blockIdx.x * seg), hi = min(B, lo + seg);
    uint32_t sum = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) sum += b.inc_count[i];
    uint32_t total;
    block_exclusive_scan(sum, s_scan, &total);
    if (threadIdx.x == 0) b.inc_blocks[blockIdx.x] = total;
    grid_barrier(barrier, flags, parts);
    uint32_t base = 0;
    for (uint32_t j = threadIdx.x; j < blockIdx.x; j += blockDim.x) base += __ldcg(b.inc_blocks + j);
    block_exclusive_scan(base, s_scan, &base);
    for (uint32_t c0 = lo; c0 < hi; c0 += blockDim.x) {
        const uint32_t i = c0 + threadIdx.x;
        const uint32_t v = i < hi ? __ldcg(b.inc_count + i) : 0u;
        uint32_t chunk;
        const uint32_t ex = block_exclusive_scan(v, s_scan, &chunk);
        if (i < hi) b.inc_off[i] = base + ex;
        base += chunk;
    }
    if (blockIdx.x == parts - 1 && threadIdx.x == 0) b.inc_off[B] = base;
}

// Bodies of active contact t (its row is read through the active list).
__device__ __forceinline__ uint2 active_bodies(const StepBuffers& b, const GpuContact* cur, uint32_t t) {
    const uint32_t k = __ldcg(b.active + t);
    const float4 r0 = __ldcg(reinterpret_cast<const float4*>(cur + k));
    return make_uint2(__float_as_uint(r0.x), __float_as_uint(r0.y));
}

__device__ void solve_gather(const StepBuffers& b, const StepParams& p, GpuContact* cur, uint32_t A,
                             uint32_t iterations, uint32_t* barrier, uint32_t parts) {
    __shared__ uint32_t s_scan[33];
    uint32_t* flags = &b.diag->error_flags;
    const uint32_t B = p.body_count;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, stride = parts * blockDim.x;
    // ---- incidence lists: counts, offsets, fill (2 t + side, grouped by body)
    for (uint32_t i = gtid; i < B; i += stride) b.inc_count[i] = 0u;
    grid_barrier(barrier, flags, parts);
    for (uint32_t t = gtid; t < A; t += stride) {
        const uint2 ab = active_bodies(b, cur, t);
        atomicAdd(b.inc_count + ab.x, 1u);
        if (ab.y != kInvalid) atomicAdd(b.inc_count + ab.y, 1u);
    }
    grid_barrier(barrier, flags, parts);
    gather_scan(b, B, parts, barrier, flags, s_scan);
    grid_barrier(barrier, flags, parts);
    for (uint32_t t = gtid; t < A; t += stride) {
        const uint2 ab = active_bodies(b, cur, t);
        b.inc_list[__ldcg(b.inc_off + ab.x) + atomicSub(b.inc_count + ab.x, 1u) - 1u] = 2u * t;
        if (ab.y != kInvalid)
            b.inc_list[__ldcg(b.inc_off + ab.y) + atomicSub(b.inc_count + ab.y, 1u) - 1u] = 2u * t + 1u;
    }
    grid_barrier(barrier, flags, parts);
    const size_t Bs = B;
    const float s = (float)kFixedScale;
    const uint32_t lane = lane_id();
    const uint32_t gwarp = gtid >> 5, nwarps = stride >> 5;
    const uint2 sl = contact_slice(A, parts);
    for (uint32_t it = 0; it < iterations; ++it) {
        // iteration `it` reads buffer it (0 = the integrated velocities) and
        // writes buffer it + 1 (the last one back into lin/ang)
        const float4* vl = it == 0 ? b.lin : b.vel_iter + (2 * (it - 1)) * Bs;
        const float4* va = it == 0 ? b.ang : b.vel_iter + (2 * (it - 1) + 1) * Bs;
        float4* dl = it + 1 == iterations ? b.lin : b.vel_iter + (2 * it) * Bs;
        float4* da_out = it + 1 == iterations ? b.ang : b.vel_iter + (2 * it + 1) * Bs;
        // ---- each contact's projection into its own delta slot
        for (uint32_t t = sl.x + threadIdx.x; t < sl.y; t += blockDim.x) {
            const uint32_t k = __ldcg(b.active + t);
            float4* row = reinterpret_cast<float4*>(cur + k);
            const float4 r0 = __ldcg(row), np = __ldcg(row + 1), aa = __ldcg(row + 2), ab = __ldcg(row + 3);
            const uint32_t a = __float_as_uint(r0.x), bb = __float_as_uint(r0.y);
            const f3 arm_a = xyz(aa), arm_b = xyz(ab);
            const float4* wa = b.world_mass + 3ull * a;
            const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
            int32_t da[6] = {0, 0, 0, 0, 0, 0}, db[6] = {0, 0, 0, 0, 0, 0};
            const f3 vb = bb != kInvalid ? contact_velocity_it(vl, va, bb, arm_b) : mkf3(0, 0, 0);
            const f3 nrm = xyz(np);
            const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
            if (!(den <= 0.0f)) {
                const f3 rel = vb - contact_velocity_it(vl, va, a, arm_a);
                float acc = aa.w;
                const bool live = it == 0
                    ? contact_project<true>(p, wa, wb, arm_a, arm_b, nrm, np.w, ab.w < 0.0f, den, rel, acc, da, db)
                    : contact_project<false>(p, wa, wb, arm_a, arm_b, nrm, np.w, ab.w < 0.0f, den, rel, acc, da, db);
                if (!live) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) da[c] = db[c] = 0;
                }
                row[2] = f4(arm_a, acc);
            }
            int4* d = reinterpret_cast<int4*>(b.contact_deltas + 12ull * t);
            d[0] = make_int4(da[0], da[1], da[2], da[3]);
            d[1] = make_int4(da[4], da[5], db[0], db[1]);
            d[2] = make_int4(db[2], db[3], db[4], db[5]);
        }
        grid_barrier(barrier, flags, parts);
        // ---- each body (one warp) sums its contacts' slots: v += delta / 2^20
        for (uint32_t x = gwarp; x < B; x += nwarps) {
            const uint32_t e0 = __ldcg(b.inc_off + x), e1 = __ldcg(b.inc_off + x + 1);
            int32_t sum[6] = {0, 0, 0, 0, 0, 0};
            for (uint32_t e = e0 + lane; e < e1; e += 32) {
                const uint32_t ent = __ldcg(b.inc_list + e);
                const int2* q = reinterpret_cast<const int2*>(b.contact_deltas + 12ull * (ent >> 1) + 6u * (ent & 1u));
                const int2 x0 = __ldcg(q), x1 = __ldcg(q + 1), x2 = __ldcg(q + 2);
                sum[0] = (int32_t)((uint32_t)sum[0] + (uint32_t)x0.x);
                sum[1] = (int32_t)((uint32_t)sum[1] + (uint32_t)x0.y);
                sum[2] = (int32_t)((uint32_t)sum[2] + (uint32_t)x1.x);
                sum[3] = (int32_t)((uint32_t)sum[3] + (uint32_t)x1.y);
                sum[4] = (int32_t)((uint32_t)sum[4] + (uint32_t)x2.x);
                sum[5] = (int32_t)((uint32_t)sum[5] + (uint32_t)x2.y);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    sum[c] = (int32_t)((uint32_t)sum[c] + (uint32_t)__shfl_down_sync(0xffffffffu, sum[c], o));
            if (lane == 0) {
                const f3 ld = mkf3((float)sum[0], (float)sum[1], (float)sum[2]) / s;
                const f3 ad = mkf3((float)sum[3], (float)sum[4], (float)sum[5]) / s;
                dl[x] = f4(xyz(__ldg(vl + x)) + ld, 0.0f);
                da_out[x] = f4(xyz(__ldg(va + x)) + ad, 0.0f);
            }
        }
        grid_barrier(barrier, flags, parts);
    }
}

// Split form: contacts arrive grouped by body a (sorted by collider a), so
// body a's deltas take warp-aggregated atomics over runs (one per run and
// component, as in the scatter form), while body b's -- one atomic per
// contact and component in the scatter form, spread over many bodies and
// serialised per body -- go to the contact's own 24-byte slot and each body
// sums its slots through an incidence list in the apply.  The running normal
// impulses live in a dense array during the solve (the rows are read-only
// until the last pass writes them back).  Same integer sums, same bits.
__device__ void solve_split(const StepBuffers& b, const StepParams& p, GpuContact* cur, uint32_t A,
                            uint32_t iterations, uint32_t* barrier, uint32_t parts) {
    __shared__ uint32_t s_scan[33];
    uint32_t* flags = &b.diag->error_flags;
    const uint32_t B = p.body_count;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, stride = parts * blockDim.x;
    // ---- incidence lists of body b: counts, offsets, fill (active positions t)
    for (uint32_t i = gtid; i < B; i += stride) b.inc_count[i] = 0u;
    grid_barrier(barrier, flags, parts);
    for (uint32_t t = gtid; t < A; t += stride) {
        const uint2 ab = active_bodies(b, cur, t);
        if (ab.y != kInvalid) atomicAdd(b.inc_count + ab.y, 1u);
    }
    grid_barrier(barrier, flags, parts);
    gather_scan(b, B, parts, barrier, flags, s_scan);
    grid_barrier(barrier, flags, parts);
    for (uint32_t t = gtid; t < A; t += stride) {
        const uint2 ab = active_bodies(b, cur, t);
        if (ab.y != kInvalid)
            b.inc_list[__ldcg(b.inc_off + ab.y) + atomicSub(b.inc_count + ab.y, 1u) - 1u] = t;
    }
    grid_barrier(barrier, flags, parts);
    const size_t Bs = B;
    const float s = (float)kFixedScale;
    const uint32_t lane = lane_id();
    const uint32_t gwarp = gtid >> 5, nwarps = stride >> 5;
    const uint2 sl = contact_slice(A, parts);
    int2* slots = reinterpret_cast<int2*>(b.contact_deltas);   // 3 x int2 per active contact
    for (uint32_t it = 0; it < iterations; ++it) {
        const float4* vl = it == 0 ? b.lin : b.vel_iter + (2 * (it - 1)) * Bs;
        const float4* va = it == 0 ? b.ang : b.vel_iter + (2 * (it - 1) + 1) * Bs;
        float4* dl = it + 1 == iterations ? b.lin : b.vel_iter + (2 * it) * Bs;
        float4* da_out = it + 1 == iterations ? b.ang : b.vel_iter + (2 * it + 1) * Bs;
        // ---- projections: body a by run sums and atomics, body b into the slot
        for (uint32_t base = sl.x; base < sl.y; base += blockDim.x) {
            const uint32_t t = base + threadIdx.x;
            bool live = false;
            uint32_t a = kInvalid;
            int32_t da[6] = {0, 0, 0, 0, 0, 0}, db[6] = {0, 0, 0, 0, 0, 0};
            // the row this thread reads next, fetched into L2 while this one is projected
            const uint32_t kn = t + blockDim.x < sl.y ? __ldcg(b.active + t + blockDim.x) : kInvalid;
            if (t < sl.y) {
                const uint32_t k = __ldcg(b.active + t);
                const float4* row = reinterpret_cast<const float4*>(cur + k);
                const float4 r0 = __ldg(row), np = __ldg(row + 1), aa = __ldg(row + 2), ab = __ldg(row + 3);
                a = __float_as_uint(r0.x);
                const uint32_t bb = __float_as_uint(r0.y);
                const f3 arm_a = xyz(aa), arm_b = xyz(ab);
                const float4* wa = b.world_mass + 3ull * a;
                const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
                const f3 vb = bb != kInvalid ? contact_velocity_it(vl, va, bb, arm_b) : mkf3(0, 0, 0);
                const f3 nrm = xyz(np);
                const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
                float acc = it == 0 ? aa.w : __ldcg(b.lam_heavy + t);
                if (!(den <= 0.0f)) {
                    const f3 rel = vb - contact_velocity_it(vl, va, a, arm_a);
                    live = it == 0
                        ? contact_project<true>(p, wa, wb, arm_a, arm_b, nrm, np.w, ab.w < 0.0f, den, rel, acc, da, db)
                        : contact_project<false>(p, wa, wb, arm_a, arm_b, nrm, np.w, ab.w < 0.0f, den, rel, acc, da, db);
                    if (!live) {
#pragma unroll
                        for (int c = 0; c < 6; ++c) da[c] = db[c] = 0;
                    }
                }
                b.lam_heavy[t] = acc;
                if (bb != kInvalid) {
                    int2* q = slots + 3ull * t;
                    q[0] = make_int2(db[0], db[1]);
                    q[1] = make_int2(db[2], db[3]);
                    q[2] = make_int2(db[4], db[5]);
                }
                if (it + 1 == iterations && !(den <= 0.0f))
                    reinterpret_cast<float*>(cur + k)[11] = acc;   // the row's impulse (arm_a_impulse.w)
            }
            if (kn != kInvalid) asm volatile("prefetch.global.L2 [%0];" ::"l"(cur + kn));
            add_contact_deltas(b.deltas, live, a, kInvalid, da, db);
        }
        grid_barrier(barrier, flags, parts);
        // ---- apply: body a's atomic sums plus the slots of the contacts where it is b
        for (uint32_t x = gwarp; x < B; x += nwarps) {
            const uint32_t e0 = __ldcg(b.inc_off + x), e1 = __ldcg(b.inc_off + x + 1);
            int32_t sum[6] = {0, 0, 0, 0, 0, 0};
            for (uint32_t e = e0 + lane; e < e1; e += 32) {
                const int2* q = slots + 3ull * __ldcg(b.inc_list + e);
                const int2 x0 = __ldcg(q), x1 = __ldcg(q + 1), x2 = __ldcg(q + 2);
                sum[0] = (int32_t)((uint32_t)sum[0] + (uint32_t)x0.x);
                sum[1] = (int32_t)((uint32_t)sum[1] + (uint32_t)x0.y);
                sum[2] = (int32_t)((uint32_t)sum[2] + (uint32_t)x1.x);
                sum[3] = (int32_t)((uint32_t)sum[3] + (uint32_t)x1.y);
                sum[4] = (int32_t)((uint32_t)sum[4] + (uint32_t)x2.x);
                sum[5] = (int32_t)((uint32_t)sum[5] + (uint32_t)x2.y);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    sum[c] = (int32_t)((uint32_t)sum[c] + (uint32_t)__shfl_down_sync(0xffffffffu, sum[c], o));
            if (lane == 0) {
                int2* d2 = reinterpret_cast<int2*>(b.deltas + 6ull * x);   // 24-byte rows are 8-byte aligned
                const int2 x0 = __ldcg(d2), x1 = __ldcg(d2 + 1), x2 = __ldcg(d2 + 2);
                if ((x0.x | x0.y | x1.x | x1.y | x2.x | x2.y) != 0) {
                    d2[0] = make_int2(0, 0);
                    d2[1] = make_int2(0, 0);
                    d2[2] = make_int2(0, 0);
                }
                const int32_t t0 = (int32_t)((uint32_t)sum[0] + (uint32_t)x0.x);
                const int32_t t1 = (int32_t)((uint32_t)sum[1] + (uint32_t)x0.y);
                const int32_t t2 = (int32_t)((uint32_t)sum[2] + (uint32_t)x1.x);
                const int32_t t3 = (int32_t)((uint32_t)sum[3] + (uint32_t)x1.y);
                const int32_t t4 = (int32_t)((uint32_t)sum[4] + (uint32_t)x2.x);
                const int32_t t5 = (int32_t)((uint32_t)sum[5] + (uint32_t)x2.y);
                const f3 ld = mkf3((float)t0, (float)t1, (float)t2) / s;
                const f3 ad = mkf3((float)t3, (float)t4, (float)t5) / s;
                dl[x] = f4(xyz(__ldg(vl + x)) + ld, 0.0f);
                da_out[x] = f4(xyz(__ldg(va + x)) + ad, 0.0f);
            }
        }
        grid_barrier(barrier, flags, parts);
    }
}

// All solver iterations in one cooperative launch: warm start, then
// (iterations - 1) projections, each followed by the velocity apply
// (device.rs:1343-1416 dispatch order), separated by grid barriers.
constexpr uint32_t kSolveThreads = 1024;   // one block per SM: 148 barrier participants

// Blocks that take part in a cooperative solve: with `items` > 0, enough for
// the active contacts and the bodies at that many items per thread (at least
// 8), the others leaving at once so that light ticks pay for smaller grid
// barriers; with 0, every block.
__device__ __forceinline__ uint32_t solve_participants(uint32_t A, uint32_t B, uint32_t items) {
    if (items == 0) return gridDim.x;   // default: every SM
    const uint32_t per_block = kSolveThreads * items;
    const uint32_t want = max((A + per_block - 1) / per_block, (B + 4u * per_block - 1) / (4u * per_block));
    return min(gridDim.x, max(want, 8u));
}

__global__ void __launch_bounds__(kSolveThreads) k_solve_all(StepBuffers b, StepParams p, GpuContact* cur,
                                                      uint32_t iterations, uint32_t* barrier, uint32_t items) {
    const uint32_t A = b.counts->active;
    if (A == 0u) return;   // collision.wgsl:744-747: no solve and no apply dispatch
    const uint32_t parts = solve_participants(A, p.body_count, items);
    if (blockIdx.x >= parts) return;
    const uint32_t first = blockIdx.x * blockDim.x;
    const uint32_t stride = parts * blockDim.x;
    const size_t B = p.body_count;
    if (A <= 2u * p.body_count && b.deltas_extra && b.body_stamp) {
        // fused passes: one grid barrier per pass, one apply at the end
        const uint64_t dstride = (6ull * B + 3) & ~3ull;   // keeps every delta buffer 16-byte aligned
        int32_t* D[3] = {b.deltas, b.deltas_extra, b.deltas_extra + dstride};
        const uint32_t gen = b.tick->generation;
        const uint32_t gtid = first + threadIdx.x;
        if (A <= stride) {
            solve_fused_resident(b, p, cur, A, iterations, D, gen, barrier, parts);
        } else {
        for (uint32_t it = 0; it < iterations; ++it) {
            FusedPass fp;
            fp.it = it;
            fp.pl = it <= 1 ? b.lin : b.vel_iter + (2 * (it - 2)) * B;
            fp.pa = it <= 1 ? b.ang : b.vel_iter + (2 * (it - 2) + 1) * B;
            fp.dprev = it == 0 ? nullptr : D[(it - 1) % 3];
            fp.cl = it == 0 ? nullptr : b.vel_iter + (2 * (it - 1)) * B;
            fp.ca = it == 0 ? nullptr : b.vel_iter + (2 * (it - 1) + 1) * B;
            fp.gen = gen;
            if (it == 0) solve_span<true, true>(b, p, cur, contact_slice(A, parts), nullptr, nullptr, &fp, D[0]);
            else solve_span<false, true>(b, p, cur, contact_slice(A, parts), nullptr, nullptr, &fp, D[it % 3]);
            int4* dz = reinterpret_cast<int4*>(D[(it + 1) % 3]);   // dead since the last barrier; used next pass
            for (uint64_t i = gtid; i < (6ull * B) / 4; i += stride) dz[i] = make_int4(0, 0, 0, 0);
            if (gtid == 0 && (6ull * B) % 4) {
                for (uint64_t i = (6ull * B) & ~3ull; i < 6ull * B; ++i) D[(it + 1) % 3][i] = 0;
            }
            grid_barrier(barrier, &b.diag->error_flags, parts);
        }
        }
        // the apply of the last pass, for every body (bodies no contact touched
        // get the reference's apply of zero deltas)
        const float s = (float)kFixedScale;
        const float4* vl = iterations <= 1 ? b.lin : b.vel_iter + (2 * (iterations - 2)) * B;
        const float4* va = iterations <= 1 ? b.ang : b.vel_iter + (2 * (iterations - 2) + 1) * B;
        const int32_t* dl = D[(iterations - 1) % 3];
        for (uint32_t i = gtid; i < B; i += stride) {
            const bool touched = __ldcg(b.body_stamp + i) == gen;
            int2 x0 = make_int2(0, 0), x1 = x0, x2 = x0;
            if (touched) {
                const int2* d2 = reinterpret_cast<const int2*>(dl + 6ull * i);
                x0 = __ldcg(d2); x1 = __ldcg(d2 + 1); x2 = __ldcg(d2 + 2);
            }
            const f3 ld = mkf3((float)x0.x, (float)x0.y, (float)x1.x) / s;
            const f3 ad = mkf3((float)x1.y, (float)x2.x, (float)x2.y) / s;
            const float4 sl = touched ? __ldg(vl + i) : __ldg(b.lin + i);
            const float4 sa = touched ? __ldg(va + i) : __ldg(b.ang + i);
            b.lin[i] = f4(xyz(sl) + ld, 0.0f);
            b.ang[i] = f4(xyz(sa) + ad, 0.0f);
        }
        return;
    }
    if (b.heavy_form == MK_HEAVY_GATHER) {   // no per-contact atomics
        solve_gather(b, p, cur, A, iterations, barrier, parts);
        return;
    }
    if (b.heavy_form == MK_HEAVY_SPLIT) {   // body a's deltas by atomics, body b's gathered
        solve_split(b, p, cur, A, iterations, barrier, parts);
        return;
    }
    for (uint32_t it = 0; it < iterations; ++it) {
        // iteration `it` reads buffer it (0 = the integrated velocities) and
        // its apply writes buffer it + 1 (the last one back into lin/ang)
        const float4* sl = it == 0 ? b.lin : b.vel_iter + (2 * (it - 1)) * B;
        const float4* sa = it == 0 ? b.ang : b.vel_iter + (2 * (it - 1) + 1) * B;
        float4* dl = it + 1 == iterations ? b.lin : b.vel_iter + (2 * it) * B;
        float4* da = it + 1 == iterations ? b.ang : b.vel_iter + (2 * it + 1) * B;
        if (it == 0) solve_span<true>(b, p, cur, contact_slice(A, parts), sl, sa);
        else solve_span<false>(b, p, cur, contact_slice(A, parts), sl, sa);
        grid_barrier(barrier, &b.diag->error_flags, parts);
        apply_span(b, p, first + threadIdx.x, stride, sl, sa, dl, da);
        grid_barrier(barrier, &b.diag->error_flags, parts);
    }
}

// ------------------------------------------------- contact solve to a residual
// The reference runs a fixed number of relaxed-Jacobi passes.  This form
// runs the same passes until the normal-row residual has fallen by
// `contact_tol` relative to the cold residual (the residual of zero impulses
// at the integrated velocities), or `contact_max_iterations` passes.  The
// residual of a contact at the state entering a pass is the unrelaxed
// projected step  r = max(prev + (-vn + bias)/D, 0) - prev  (the relaxed pass
// moves the impulse by 0.125 r when no clamp is active).  Norms are FP64
// sums in one fixed order (1024-element stride-halving trees over chunks of
// the active list, then over the chunk sums), so every block reaches the same
// stopping decision and repeated runs are bitwise identical.  Velocity
// deltas use 64-bit fixed point (x 2^32): 2^20 quantises velocity to ~1e-6
// m/s, about the size of the residual a 1e-5 relative tolerance asks for.
//
// With a learned warm start two candidates run side by side for the first
// two passes (cached start in the contact rows, learned start in lam_alt);
// the one with the smaller residual after its first pass continues, so the
// cached start is the fallback whenever the learned one raises the initial
// residual.
constexpr uint32_t kResChunk = 1024;
constexpr float kFixed64Scale = 4294967296.0f;        // 2^32
constexpr float kFixed64Inverse = 2.3283064365386963e-10f;   // 2^-32

__device__ __forceinline__ int64_t fixed_i64(float x) { return __float2ll_rn(x); }   // half-even, saturating

__device__ __forceinline__ bool run_tail_sum64(uint32_t key, int64_t* v) {
    const uint32_t lane = lane_id();
    const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    const uint32_t next = __shfl_down_sync(0xffffffffu, key, 1);
    const bool head = lane == 0 || prev != key;
    const bool tail = lane == 31 || next != key;
    const uint32_t heads = __ballot_sync(0xffffffffu, head);
    const uint32_t below = heads & ((2u << lane) - 1u);
    const uint32_t head_lane = 31u - __clz(below);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const long long u = __shfl_up_sync(0xffffffffu, (long long)v[c], o);
            if (lane >= head_lane + (uint32_t)o) v[c] = (int64_t)((uint64_t)v[c] + (uint64_t)u);
        }
    }
    return tail;
}

// Sum of x[0..n) (n <= 1024, zero padded) by the stride-halving tree; all
// 1024 threads of the block take part.
__device__ __forceinline__ double tree1024(double mine, double* s) {
    const uint32_t t = threadIdx.x;
    __syncthreads();
    s[t] = mine;
#pragma unroll 1
    for (uint32_t stride = kResChunk / 2; stride >= 1; stride >>= 1) {
        __syncthreads();
        if (t < stride) s[t] += s[t + stride];
    }
    __syncthreads();
    const double r = s[0];
    __syncthreads();
    return r;
}

// canonical_sum of the n chunk sums (n <= 1024 * 1024), computed by one block.
__device__ double canonical_sum(const double* chunks, uint32_t n, double* s_tree, double* s_top) {
    const uint32_t t = threadIdx.x;
    if (n <= kResChunk) return tree1024(t < n ? __ldcg(chunks + t) : 0.0, s_tree);
    const uint32_t groups = (n + kResChunk - 1) / kResChunk;
    for (uint32_t g = 0; g < groups; ++g) {
        const uint64_t i = (uint64_t)g * kResChunk + t;
        const double r = tree1024(i < n ? __ldcg(chunks + i) : 0.0, s_tree);
        if (t == 0) s_top[g] = r;
    }
    __syncthreads();
    return tree1024(t < groups ? s_top[t] : 0.0, s_tree);
}

struct ResCandidate {
    const float4* sl;   // velocities entering the pass
    const float4* sa;
    float4* dl;         // velocities after it
    float4* da;
};

__device__ __forceinline__ f3 contact_velocity_cg(const float4* vl, const float4* va, uint32_t body, f3 arm) {
    return xyz(__ldcg(vl + body)) + cross(xyz(__ldcg(va + body)), arm);
}

// One pass for candidate `c` (0: impulses in the contact rows, 1: in lam_alt).
__device__ __forceinline__ void solve_span_res(const StepBuffers& b, const StepParams& p, GpuContact* cur, uint32_t A,
                                               bool warm, uint32_t c, const ResCandidate& v, bool write_res) {
    int64_t* deltas = b.deltas64 + 6ull * p.body_count * c;
    double* res2 = b.res2 + (uint64_t)p.pair_capacity * c;
    const uint2 sl = contact_slice(A, gridDim.x);
    for (uint32_t base = sl.x; base < sl.y; base += blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        bool live = false;
        uint32_t a = kInvalid, bb = kInvalid;
        float r = 0.0f;
        int64_t da[6] = {0, 0, 0, 0, 0, 0}, db[6] = {0, 0, 0, 0, 0, 0};
        if (t < sl.y) {
            const uint32_t k = __ldcg(b.active + t);
            float4* row = reinterpret_cast<float4*>(cur + k);
            const float4 r0 = __ldcg(row), np = __ldcg(row + 1), aa = __ldcg(row + 2), ab = __ldcg(row + 3);
            a = __float_as_uint(r0.x);
            bb = __float_as_uint(r0.y);
            const f3 arm_a = xyz(aa), arm_b = xyz(ab);
            const float4* wa = b.world_mass + 3ull * a;
            const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
            f3 vb = mkf3(0, 0, 0);
            if (bb != kInvalid) vb = contact_velocity_cg(v.sl, v.sa, bb, arm_b);
            const f3 nrm = xyz(np);
            const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
            float lam = c == 0 ? aa.w : (warm ? __ldcg(b.warm_pred + t) : __ldcg(b.lam_alt + t));
            if (!(den <= 0.0f)) {
                const f3 rel = vb - contact_velocity_cg(v.sl, v.sa, a, arm_a);
                const float vn = dot(rel, nrm);
                if (np.w <= 1.0e-5f && vn >= -1.0e-5f && lam <= 1.0e-6f) {
                    lam = 0.0f;
                } else {
                    const bool cyl = ab.w < 0.0f;
                    const float recovery = cyl ? 1.0f : 0.2f;
                    const float bias = mnf(mxf(np.w - 0.001f, 0.0f) * recovery / p.dt, 1.0f);
                    float acc, delta;
                    if (warm) {
                        const float start = c == 0 ? aa.w * (cyl ? 1.0f : 0.5f) : lam;
                        acc = mxf(start + 0.125f * (-vn + bias) / den, 0.0f);
                        delta = acc;
                        r = mxf((-vn + bias) / den, 0.0f);
                    } else {
                        const float prev = mxf(lam, 0.0f);
                        acc = mxf(prev + 0.125f * (-vn + bias) / den, 0.0f);
                        delta = acc - prev;
                        r = mxf(prev + (-vn + bias) / den, 0.0f) - prev;
                    }
                    lam = acc;
                    f3 imp = nrm * delta;
                    const f3 tv = rel - nrm * vn;
                    const float ts = length(tv);
                    if (ts > 1.0e-6f) {
                        const f3 tg = tv / ts;
                        const float tden = impulse_denominator(wa, wb, arm_a, arm_b, tg);
                        const float fr = mnf(ts / tden, (warm ? acc : fabsf(delta)) * 0.05f);
                        imp = imp - tg * fr;
                    }
                    const f3 la = -imp * wa[0].w;
                    const f3 ga = inverse_inertia(wa, cross(arm_a, -imp));
                    da[0] = fixed_i64(la.x * kFixed64Scale); da[1] = fixed_i64(la.y * kFixed64Scale);
                    da[2] = fixed_i64(la.z * kFixed64Scale); da[3] = fixed_i64(ga.x * kFixed64Scale);
                    da[4] = fixed_i64(ga.y * kFixed64Scale); da[5] = fixed_i64(ga.z * kFixed64Scale);
                    live = true;
                    if (wb) {
                        const f3 lb = imp * wb[0].w;
                        const f3 gb = inverse_inertia(wb, cross(arm_b, imp));
                        db[0] = fixed_i64(lb.x * kFixed64Scale); db[1] = fixed_i64(lb.y * kFixed64Scale);
                        db[2] = fixed_i64(lb.z * kFixed64Scale); db[3] = fixed_i64(gb.x * kFixed64Scale);
                        db[4] = fixed_i64(gb.y * kFixed64Scale); db[5] = fixed_i64(gb.z * kFixed64Scale);
                    }
                }
            }
            if (c == 0) row[2] = f4(arm_a, lam);
            else b.lam_alt[t] = lam;
            if (write_res) res2[t] = (double)r * (double)r;
        }
        const uint32_t key_a = live ? a : kInvalid;
        const bool tail = run_tail_sum64(key_a, da);
        if (tail && key_a != kInvalid) {
            unsigned long long* d = reinterpret_cast<unsigned long long*>(deltas + 6ull * key_a);
#pragma unroll
            for (int q = 0; q < 6; ++q)
                if (da[q]) atomicAdd(d + q, (unsigned long long)da[q]);
        }
        if (live && bb != kInvalid) {
            unsigned long long* d = reinterpret_cast<unsigned long long*>(deltas + 6ull * bb);
#pragma unroll
            for (int q = 0; q < 6; ++q)
                if (db[q]) atomicAdd(d + q, (unsigned long long)db[q]);
        }
    }
}

__device__ __forceinline__ void apply_span_res(const StepBuffers& b, const StepParams& p, uint32_t c,
                                               const ResCandidate& v) {
    const uint32_t stride = gridDim.x * blockDim.x;
    longlong2* dl = reinterpret_cast<longlong2*>(b.deltas64 + 6ull * p.body_count * c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.body_count; i += stride) {
        longlong2* d = dl + 3ull * i;
        const longlong2 x0 = __ldcg(d), x1 = __ldcg(d + 1), x2 = __ldcg(d + 2);
        if ((x0.x | x0.y | x1.x | x1.y | x2.x | x2.y) != 0) {
            d[0] = make_longlong2(0, 0);
            d[1] = make_longlong2(0, 0);
            d[2] = make_longlong2(0, 0);
        }
        const f3 ld = mkf3(__ll2float_rn(x0.x), __ll2float_rn(x0.y), __ll2float_rn(x1.x)) * kFixed64Inverse;
        const f3 ad = mkf3(__ll2float_rn(x1.y), __ll2float_rn(x2.x), __ll2float_rn(x2.y)) * kFixed64Inverse;
        v.dl[i] = f4(xyz(__ldcg(v.sl + i)) + ld, 0.0f);
        v.da[i] = f4(xyz(__ldcg(v.sa + i)) + ad, 0.0f);
    }
}

__device__ __forceinline__ void chunk_sums(const StepBuffers& b, const StepParams& p, uint32_t A, uint32_t ncand,
                                           uint32_t c_first, double* s_tree) {
    const uint32_t chunks = (A + kResChunk - 1) / kResChunk;
    for (uint32_t job = blockIdx.x; job < chunks * ncand; job += gridDim.x) {
        const uint32_t c = c_first + job / chunks, ch = job % chunks;
        const uint64_t i = (uint64_t)ch * kResChunk + threadIdx.x;
        const double* res2 = b.res2 + (uint64_t)p.pair_capacity * c;
        const double sum = tree1024(i < A ? __ldcg(res2 + i) : 0.0, s_tree);
        if (threadIdx.x == 0) b.res_chunks[(uint64_t)b.res_chunk_cap * c + ch] = sum;
    }
}

__global__ void __launch_bounds__(kSolveThreads) k_solve_residual(StepBuffers b, StepParams p, GpuContact* cur,
                                                           uint32_t learned, uint32_t* barrier) {
    __shared__ double s_tree[kResChunk];
    __shared__ double s_top[kResChunk];
    const uint32_t A = b.counts->active;
    if (A == 0u) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *b.solve_stats = SolveStats{0u, 0u, 1u, 0u, 0.0, 0.0};
        return;
    }
    const size_t B = p.body_count;
    const double tol2 = (double)p.contact_tol * (double)p.contact_tol;
    // candidate c ping-pongs between velocity pairs 2c and 2c + 1
    const float4* src_l[2] = {b.lin, b.lin};
    const float4* src_a[2] = {b.ang, b.ang};
    uint32_t next_pair[2] = {0u, 2u};
    bool dual = learned != 0u;
    uint32_t chosen = 0;
    double s0 = 0.0, sk = 0.0;
    uint32_t it = 0, converged = 0;
    const uint32_t max_it = p.contact_max_iterations;
    while (it < max_it) {
        const uint32_t c_first = dual ? 0u : chosen, c_last = dual ? 1u : chosen;
        ResCandidate v[2];
        for (uint32_t c = c_first; c <= c_last; ++c) {
            const uint32_t q = next_pair[c];
            v[c] = {src_l[c], src_a[c], b.vel_res + (2ull * q) * B, b.vel_res + (2ull * q + 1) * B};
            // the cold residual (pass 0) is the same for both candidates
            solve_span_res(b, p, cur, A, it == 0, c, v[c], !(it == 0 && c == 1));
        }
        grid_barrier(barrier, &b.diag->error_flags, gridDim.x);
        for (uint32_t c = c_first; c <= c_last; ++c) apply_span_res(b, p, c, v[c]);
        const uint32_t nres = (it == 0) ? 1u : (c_last - c_first + 1);
        chunk_sums(b, p, A, nres, c_first, s_tree);
        grid_barrier(barrier, &b.diag->error_flags, gridDim.x);
        const uint32_t chunks = (A + kResChunk - 1) / kResChunk;
        double S[2] = {0.0, 0.0};
        for (uint32_t c = c_first; c < c_first + nres; ++c)
            S[c] = canonical_sum(b.res_chunks + (uint64_t)b.res_chunk_cap * c, chunks, s_tree, s_top);
        for (uint32_t c = c_first; c <= c_last; ++c) {
            src_l[c] = v[c].dl;
            src_a[c] = v[c].da;
            next_pair[c] ^= 1u;
        }
        ++it;
        if (it == 1) {
            s0 = S[c_first];
            sk = s0;
            continue;
        }
        if (dual) {
            chosen = S[1] <= S[0] ? 1u : 0u;
            dual = false;
        }
        sk = S[chosen];
        if (sk <= tol2 * s0) {
            converged = 1;
            break;
        }
    }
    // final velocities (and the learned candidate's impulses) into place
    const uint32_t gs = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gs) {
        b.lin[i] = __ldcg(src_l[chosen] + i);
        b.ang[i] = __ldcg(src_a[chosen] + i);
    }
    if (chosen == 1u) {
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A; t += gs) {
            float4* row = reinterpret_cast<float4*>(cur + __ldcg(b.active + t));
            const float4 aa = __ldcg(row + 2);
            row[2] = make_float4(aa.x, aa.y, aa.z, __ldcg(b.lam_alt + t));
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *b.solve_stats = SolveStats{it, chosen, converged, 0u, s0, sk};
}

// ------------------------------------------------------ learned warm start
// Per-contact inputs of the warm-start network, taken at the state the
// contact solve starts from (integrated velocities, this tick's contact
// rows), in velocity units so that mass drops out:
//   0 vn   1 tangential speed   2 depth / dt   3-5 normal
//   6 inverse-mass share of body A   7 cached impulse x D   8 bias
//   9 cylinder-ground   10 ground   11 max(-vn + bias, 0)   12 log D
//   13 cached impulse present   14 D   15 (constant 1, set by the network)
// with D the impulse denominator along the normal (inverse effective mass).
// The network predicts the converged impulse x D; impulse = max(y, 0) / D.
__global__ void __launch_bounds__(kBlock) k_warm_features(StepBuffers b, StepParams p, const GpuContact* cur,
                                                          float4* features) {
    const uint32_t A = b.counts->active;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A; t += gridDim.x * blockDim.x) {
        const uint32_t k = b.active[t];
        const float4* row = reinterpret_cast<const float4*>(cur + k);
        const float4 r0 = row[0], np = row[1], aa = row[2], ab = row[3];
        const uint32_t a = __float_as_uint(r0.x), bb = __float_as_uint(r0.y);
        const f3 arm_a = xyz(aa), arm_b = xyz(ab);
        const float4* wa = b.world_mass + 3ull * a;
        const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
        const f3 nrm = xyz(np);
        const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
        float4 f[4] = {make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0),
                       make_float4(0, 0, 0, 0)};
        if (den > 0.0f) {
            f3 vb = mkf3(0, 0, 0);
            if (bb != kInvalid) vb = xyz(b.lin[bb]) + cross(xyz(b.ang[bb]), arm_b);
            const f3 rel = vb - (xyz(b.lin[a]) + cross(xyz(b.ang[a]), arm_a));
            const float vn = dot(rel, nrm);
            const float ts = length(rel - nrm * vn);
            const bool cyl = ab.w < 0.0f;
            const float bias = mnf(mxf(np.w - 0.001f, 0.0f) * (cyl ? 1.0f : 0.2f) / p.dt, 1.0f);
            const float inv_a = wa[0].w, inv_b = wb ? wb[0].w : 0.0f;
            f[0] = make_float4(vn, ts, np.w / p.dt, nrm.x);
            f[1] = make_float4(nrm.y, nrm.z, inv_a / (inv_a + inv_b), aa.w * den);
            f[2] = make_float4(bias, cyl ? 1.0f : 0.0f, bb == kInvalid ? 1.0f : 0.0f, mxf(-vn + bias, 0.0f));
            f[3] = make_float4(logf(den), aa.w > 0.0f ? 1.0f : 0.0f, den, 1.0f);
        }
        float4* out = features + 4ull * t;
        out[0] = f[0]; out[1] = f[1]; out[2] = f[2]; out[3] = f[3];
    }
}

// network output (one column) -> warm-start impulse
__global__ void __launch_bounds__(kBlock) k_warm_impulses(StepBuffers b, const float4* features, const float* y,
                                                          float* warm) {
    const uint32_t A = b.counts->active;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A; t += gridDim.x * blockDim.x) {
        const float den = features[4ull * t + 3].z;
        const float v = y[t];
        warm[t] = (den > 0.0f && v > 0.0f) ? v / den : 0.0f;   // NaN outputs give 0
    }
}

// training targets of the last tick: converged impulse x D per active contact
__global__ void __launch_bounds__(kBlock) k_warm_targets(StepBuffers b, const GpuContact* cur, const float4* features,
                                                         uint32_t A, float* targets) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A; t += gridDim.x * blockDim.x) {
        const float lam = reinterpret_cast<const float4*>(cur + b.active[t])[2].w;
        targets[t] = lam * features[4ull * t + 3].z;
    }
}

cudaError_t launch_warm_features(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                 cudaStream_t s) {
    k_warm_features<<<(uint32_t)l.sm_count * 8, kBlock, 0, s>>>(b, p, b.contacts[parity], b.warm_features);
    return cudaGetLastError();
}

cudaError_t launch_warm_impulses(const StepBuffers& b, const StepLaunch& l, const float* y, cudaStream_t s) {
    k_warm_impulses<<<(uint32_t)l.sm_count * 8, kBlock, 0, s>>>(b, b.warm_features, y, b.warm_pred);
    return cudaGetLastError();
}

cudaError_t launch_warm_targets(const StepBuffers& b, int parity, uint32_t A, float* targets, cudaStream_t s) {
    if (A == 0) return cudaSuccess;
    k_warm_targets<<<(A + kBlock - 1) / kBlock, kBlock, 0, s>>>(b, b.contacts[parity], b.warm_features, A, targets);
    return cudaGetLastError();
}

// Per-iteration kernels for ticks that interleave bearing projection with
// the contact iterations (device.rs:1363-1416): velocities are updated in
// place, so each phase is its own launch.
template <bool kWarm>
__global__ void __launch_bounds__(kBlock) k_solve_iter(StepBuffers b, StepParams p, GpuContact* cur) {
    const uint32_t A = b.counts->active;
    solve_span<kWarm>(b, p, cur, contact_slice(A, gridDim.x), b.lin, b.ang);
}

__global__ void __launch_bounds__(kBlock) k_apply_iter(StepBuffers b, StepParams p) {
    if (b.counts->active == 0u) return;   // collision.wgsl:744 (no apply dispatch without active contacts)
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const float s = (float)kFixedScale;
    for (uint32_t i = first; i < p.body_count; i += stride) {
        int2* d2 = reinterpret_cast<int2*>(b.deltas + 6ull * i);
        const int2 x0 = d2[0], x1 = d2[1], x2 = d2[2];
        if ((x0.x | x0.y | x1.x | x1.y | x2.x | x2.y) == 0) {   // untouched body: write only if bits change
            if (zero_apply_is_identity(b.lin[i]) && zero_apply_is_identity(b.ang[i])) continue;
        } else {
            d2[0] = make_int2(0, 0);
            d2[1] = make_int2(0, 0);
            d2[2] = make_int2(0, 0);
        }
        const f3 ld = mkf3((float)x0.x, (float)x0.y, (float)x1.x) / s;
        const f3 ad = mkf3((float)x1.y, (float)x2.x, (float)x2.y) / s;
        b.lin[i] = f4(xyz(b.lin[i]) + ld, 0.0f);
        b.ang[i] = f4(xyz(b.ang[i]) + ad, 0.0f);
    }
}

// collision.wgsl:908-977: one contact, velocities updated immediately.
__device__ void solve_contact_immediate(const StepBuffers& b, const StepParams& p, GpuContact* cur, uint32_t k) {
    float4* row = reinterpret_cast<float4*>(cur + k);
    const float4 r0 = row[0], np = row[1], aa = row[2], ab = row[3];
    const uint32_t a = __float_as_uint(r0.x), bb = __float_as_uint(r0.y);
    const f3 arm_a = xyz(aa), arm_b = xyz(ab);
    const float4* wa = b.world_mass + 3ull * a;
    const float4* wb = bb != kInvalid ? b.world_mass + 3ull * bb : nullptr;
    f3 vb = mkf3(0, 0, 0);
    if (bb != kInvalid) vb = contact_velocity(b, bb, arm_b);
    const f3 nrm = xyz(np);
    const float den = impulse_denominator(wa, wb, arm_a, arm_b, nrm);
    if (den <= 0.0f) return;
    const f3 rel = vb - contact_velocity(b, a, arm_a);
    const float vn = dot(rel, nrm);
    if (np.w <= 1.0e-5f && vn >= -1.0e-5f && aa.w <= 1.0e-6f) {
        row[2] = f4(arm_a, 0.0f);
        return;
    }
    const bool cyl = ab.w < 0.0f;
    const float bias = mnf(mxf(np.w - 0.001f, 0.0f) * (cyl ? 1.0f : 0.2f) / p.dt, 1.0f);
    const float prev = mxf(aa.w, 0.0f);
    const float acc = mxf(prev + (-vn + bias) / den, 0.0f);
    const float delta = acc - prev;
    row[2] = f4(arm_a, acc);
    f3 imp = nrm * delta;
    const f3 tv = rel - nrm * vn;
    const float ts = length(tv);
    if (ts > 1.0e-6f) {
        const f3 tg = tv / ts;
        const float tden = impulse_denominator(wa, wb, arm_a, arm_b, tg);
        const float fr = mnf(ts / tden, fabsf(delta) * 0.05f);
        imp = imp - tg * fr;
    }
    b.lin[a] = f4(xyz(b.lin[a]) - imp * wa[0].w, 0.0f);
    b.ang[a] = f4(xyz(b.ang[a]) + inverse_inertia(wa, cross(arm_a, -imp)), 0.0f);
    if (wb) {
        b.lin[bb] = f4(xyz(b.lin[bb]) + imp * wb[0].w, 0.0f);
        b.ang[bb] = f4(xyz(b.ang[bb]) + inverse_inertia(wb, cross(arm_b, imp)), 0.0f);
    }
}

// collision.wgsl:979-1048: forward then backward Gauss-Seidel sweeps, one
// thread; at most 64 active contacts are visited in (body a, body b,
// manifold slot) order, more in active-list order.
__global__ void k_solve_serial(StepBuffers b, StepParams p, GpuContact* cur) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t A = b.counts->active;
    if (A > 64u) {
        for (uint32_t k = 0; k < A; ++k) solve_contact_immediate(b, p, cur, b.active[k]);
        for (uint32_t k = A; k > 0; --k) solve_contact_immediate(b, p, cur, b.active[k - 1]);
        return;
    }
    uint32_t order[64];
    for (uint32_t k = 0; k < A; ++k) order[k] = b.active[k];
    for (uint32_t x = 1; x < A; ++x) {   // sort by (body a, body b, manifold slot)
        const uint32_t v = order[x];
        const uint4 kv = *reinterpret_cast<const uint4*>(cur[v].metadata);
        int y = (int)x - 1;
        while (y >= 0) {
            const uint4 ky = *reinterpret_cast<const uint4*>(cur[order[y]].metadata);
            const bool greater = ky.x > kv.x || (ky.x == kv.x && (ky.y > kv.y || (ky.y == kv.y && ky.z > kv.z)));
            if (!greater) break;
            order[y + 1] = order[y];
            --y;
        }
        order[y + 1] = v;
    }
    for (uint32_t k = 0; k < A; ++k) solve_contact_immediate(b, p, cur, order[k]);
    for (uint32_t k = A; k > 0; --k) solve_contact_immediate(b, p, cur, order[k - 1]);
}

// Bookkeeping at the end of a tick: this tick's contact list becomes the
// manifold cache of the next one.
__global__ void k_finish_tick(StepBuffers b) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    DevCounts* c = b.counts;
    c->prev_narrow = c->narrow;
    c->prev_contacts = c->contacts;
    c->prev_tick = b.tick->tick_index;
    c->prev_valid = 1u;
    c->prev_indexed = 1u;   // this tick's prepare indexed its list
}

// physics.wgsl:73-90
__global__ void k_apply_impulse(StepBuffers b, uint32_t body, float3 point, float3 impulse) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float4* m = b.mass + 4ull * body;
    const float inv = m[0].x;
    if (inv <= 0.0f) return;
    const f3 J = mkf3(impulse.x, impulse.y, impulse.z);
    const f3 arm = mkf3(point.x, point.y, point.z) - xyz(b.pos[body]);
    b.lin[body] = f4(xyz(b.lin[body]) + J * inv, 0.0f);
    const float4 r = b.rot[body];
    const f3 v = cross(arm, J);
    const f3 local = quat_rotate(conjq(r), v);
    const f3 lr = xyz(m[1]) * local.x + xyz(m[2]) * local.y + xyz(m[3]) * local.z;
    b.ang[body] = f4(xyz(b.ang[body]) + quat_rotate(r, lr), 0.0f);
}

// Standalone batched SAT (mk_op_obb_sat): boxes as 4 float4 rows
// {center, hx}, {axis_x, hy}, {axis_y, hz}, {axis_z, -}.
__global__ void __launch_bounds__(kBlock) k_obb_sat_op(const float4* __restrict__ ba, const float4* __restrict__ bb,
                                                       uint32_t count, float4* __restrict__ np, uint32_t* __restrict__ feat) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    auto load = [](const float4* p) {
        Box o;
        const float4 r0 = __ldg(p), r1 = __ldg(p + 1), r2 = __ldg(p + 2), r3 = __ldg(p + 3);
        o.c = xyz(r0);
        o.h[0] = r0.w; o.h[1] = r1.w; o.h[2] = r2.w;
        o.ax[0] = xyz(r1); o.ax[1] = xyz(r2); o.ax[2] = xyz(r3);
        o.q = make_float4(0, 0, 0, 1);
        return o;
    };
    const Box A = load(ba + 4ull * i), B = load(bb + 4ull * i);
    const Sat s = obb_sat(A, B);
    np[i] = f4(s.n, s.pen);
    feat[i] = s.axis | (s.near << 8) | (s.early << 16);
}

// ------------------------------------------------------------------ launch
static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

cudaError_t launch_integrate(const StepBuffers& b, const StepParams& p, const StepLaunch& l, cudaStream_t s) {
    if (p.body_count == 0) return cudaSuccess;
    if (l.fuse_world_mass) k_integrate<true><<<blocks_for(p.body_count, kBlock), kBlock, 0, s>>>(b, p);
    else k_integrate<false><<<blocks_for(p.body_count, kBlock), kBlock, 0, s>>>(b, p);
    return cudaGetLastError();
}

cudaError_t launch_world_masses(const StepBuffers& b, const StepParams& p, cudaStream_t s) {
    if (p.body_count == 0) return cudaSuccess;
    k_world_masses<<<blocks_for(p.body_count, kBlock), kBlock, 0, s>>>(b, p);
    return cudaGetLastError();
}

cudaError_t launch_snapshot(const StepBuffers& b, const StepParams& p, cudaStream_t s) {
    if (p.body_count == 0) return cudaSuccess;
    k_snapshot<<<blocks_for(p.body_count, kBlock), kBlock, 0, s>>>(b, p);
    return cudaGetLastError();
}

cudaError_t launch_broadphase(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                              cudaStream_t s) {
    (void)parity;
    const uint32_t C = p.collider_count;
    if (C == 0) return cudaSuccess;
    k_collider_bounds<<<blocks_for(C, kBlock), kBlock, 0, s>>>(b, p, l.morton_mode);
    if (l.morton_mode != MK_MORTON_REFERENCE_30)
        k_morton_keys<<<blocks_for(C, kBlock), kBlock, 0, s>>>(b, p, l.morton_mode);
    const uint32_t key_bits = sort_key_bits(l.morton_mode, p.scene_bits);
    cudaError_t e = launch_sort(b.keys, b.values, b.skeys, b.svals, C, nullptr, key_bits, b.sort_scratch,
                                b.sort_scratch_bytes, &b.diag->error_flags, s, l.sm_count, l.sort_items, l.sort_ctas,
                                true);   // bins and tickets cleared by the tick's reset
    if (e != cudaSuccess) return e;
    k_karras<<<blocks_for(C, kBlock), kBlock, 0, s>>>(b, p);
    k_refit_leaves<<<blocks_for(C, kRefitBlock), kRefitBlock, 0, s>>>(b, p);
    k_refit_super<<<1, 1024, 0, s>>>(b, p);
    // persistent over the listed nodes (their count is known on the device only)
    k_refit_nodes<<<std::min<uint32_t>(blocks_for(C, kBlock), (uint32_t)l.sm_count * 2u), kBlock, 0, s>>>(b, p);
    if (b.collider_scene) k_traverse<true><<<blocks_for(C, kTravThreads), kTravThreads, 0, s>>>(b, p);
    else k_traverse<false><<<blocks_for(C, kTravThreads), kTravThreads, 0, s>>>(b, p);
    e = launch_sort(b.pair_stage, nullptr, b.pair_keys, nullptr, p.pair_capacity, &b.counts->pairs_found,
                    2 * p.pair_shift, b.pair_sort_scratch, b.pair_sort_scratch_bytes, &b.diag->error_flags, s,
                    l.sm_count, pair_sort_items(), 0, true);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_narrowphase(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                               cudaStream_t s) {
    const uint32_t grid = (uint32_t)l.sm_count * (l.append_ctas ? l.append_ctas : 8u);
    AppendSite narrow{b.lookback + 1 * b.lookback_words, b.tickets + 1};
    k_narrowphase<<<grid, kBlock, 0, s>>>(b, p, narrow, b.contacts[parity], b.contact_keys[parity], b.features[parity]);
    k_narrowphase_rows<<<grid, kBlock, 0, s>>>(b, p, narrow, b.contacts[parity], b.contact_keys[parity],
                                               b.features[parity]);
    k_ground<<<std::max<uint32_t>(1u, blocks_for(p.collider_count, kGroundTile)), kBlock, 0, s>>>(
        b, p, b.contacts[parity], b.contact_keys[parity], b.features[parity]);
    return cudaGetLastError();
}

// Form of the heavy-tick solve (MK_TUNE_HEAVY_SOLVE; 0 = the default, the
// fastest measured); every form gives the same bits.  Read when a tick is captured.
static uint32_t g_heavy_solve_form = 0;
void set_heavy_solve_form(uint32_t form) { g_heavy_solve_form = form <= MK_HEAVY_SPLIT ? form : 0u; }
uint32_t heavy_solve_form() { return g_heavy_solve_form; }
constexpr uint32_t kDefaultHeavyForm = MK_HEAVY_SPLIT;   // measured fastest: tick 1 of the 100,000-body config 4.44 ms (scatter 5.12, gather 6.02)

cudaError_t launch_contact_solver(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                  cudaStream_t s, const std::function<cudaError_t()>& before_solve) {
    const uint32_t grid = (uint32_t)l.sm_count * (l.append_ctas ? l.append_ctas : 8u);
    AppendSite prep{b.lookback + 3 * b.lookback_words, b.tickets + 3};
    const int prev = parity ^ 1;
    k_prepare<<<grid, kBlock, 0, s>>>(b, p, prep, b.contacts[parity], b.contact_keys[parity], b.features[parity],
                                       b.contacts[prev], b.contact_keys[prev], b.features[prev]);
    if (before_solve) {
        cudaError_t eb = before_solve();
        if (eb != cudaSuccess) return eb;
    }
    // one co-resident grid for every iteration (cooperative launch)
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_all, kSolveThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const uint32_t blocks = (uint32_t)l.sm_count;
    const uint32_t iters = std::max<uint32_t>(1u, l.iterations);
    GpuContact* cur = b.contacts[parity];
    uint32_t* barrier = b.grid_barrier;
    StepBuffers bb = b;
    bb.heavy_form = g_heavy_solve_form ? g_heavy_solve_form : kDefaultHeavyForm;
    StepParams pp = p;
    uint32_t learned = l.learned_warm ? 1u : 0u;
    const bool residual = p.contact_tol > 0.0f;
    if (residual) {
        if (!b.deltas64 || !b.vel_res) return cudaErrorInvalidValue;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_residual, kSolveThreads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
    }
    uint32_t solve_items = l.solve_items;   // 0: all blocks take part
    void* args[] = {&bb, &pp, &cur, (void*)&iters, &barrier, &solve_items};
    void* args_res[] = {&bb, &pp, &cur, (void*)&learned, &barrier};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kSolveThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = residual ? cudaLaunchKernelExC(&cfg, (const void*)k_solve_residual, args_res)
                 : cudaLaunchKernelExC(&cfg, (const void*)k_solve_all, args);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_contact_solver_stepwise(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                           bool serial, const std::function<cudaError_t(bool)>& after_apply,
                                           cudaStream_t s) {
    const uint32_t grid = (uint32_t)l.sm_count * (l.append_ctas ? l.append_ctas : 8u);
    AppendSite prep{b.lookback + 3 * b.lookback_words, b.tickets + 3};
    const int prev = parity ^ 1;
    GpuContact* cur = b.contacts[parity];
    k_prepare<<<grid, kBlock, 0, s>>>(b, p, prep, cur, b.contact_keys[parity], b.features[parity], b.contacts[prev],
                                       b.contact_keys[prev], b.features[prev]);
    const uint32_t body_blocks = std::max<uint32_t>(1u, std::min<uint32_t>(blocks_for(p.body_count, kBlock), grid));
    k_solve_iter<true><<<grid, kBlock, 0, s>>>(b, p, cur);
    k_apply_iter<<<body_blocks, kBlock, 0, s>>>(b, p);
    cudaError_t e = after_apply(serial);
    if (e != cudaSuccess) return e;
    const uint32_t iters = serial ? std::max<uint32_t>(1u, l.iterations) * 12u : std::max<uint32_t>(1u, l.iterations);
    for (uint32_t it = 1; it < iters; ++it) {
        if (serial) {
            k_solve_serial<<<1, 32, 0, s>>>(b, p, cur);
        } else {
            k_solve_iter<false><<<grid, kBlock, 0, s>>>(b, p, cur);
            k_apply_iter<<<body_blocks, kBlock, 0, s>>>(b, p);
        }
        if ((e = after_apply(serial)) != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_finish_tick(const StepBuffers& b, const StepParams& p, int parity, cudaStream_t s) {
    (void)p;
    (void)parity;
    k_finish_tick<<<1, 32, 0, s>>>(b);
    return cudaGetLastError();
}

// Every region a tick needs at zero, cleared by one kernel (16-byte stores)
// instead of one memset node per region.
__global__ void __launch_bounds__(kBlock) k_tick_reset(ZeroList z) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t r = 0; r < z.count; ++r)
        for (uint64_t i = first; i < z.n16[r]; i += stride) z.ptr[r][i] = make_uint4(0u, 0u, 0u, 0u);
}

cudaError_t launch_tick_reset(const ZeroList& z, int sm_count, cudaStream_t s) {
    uint64_t most = 0;
    for (uint32_t r = 0; r < z.count; ++r) most = most > z.n16[r] ? most : z.n16[r];
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((most + kBlock - 1) / kBlock,
                                                                               (uint64_t)sm_count * 4));
    k_tick_reset<<<grid, kBlock, 0, s>>>(z);
    return cudaGetLastError();
}

cudaError_t launch_apply_impulse(const StepBuffers& b, uint32_t body, float3 point, float3 impulse, cudaStream_t s) {
    k_apply_impulse<<<1, 32, 0, s>>>(b, body, point, impulse);
    return cudaGetLastError();
}

cudaError_t launch_obb_sat(const float* boxes_a, const float* boxes_b, uint32_t count, float* np, uint32_t* features,
                           cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_obb_sat_op<<<blocks_for(count, kBlock), kBlock, 0, s>>>(reinterpret_cast<const float4*>(boxes_a),
                                                               reinterpret_cast<const float4*>(boxes_b), count,
                                                               reinterpret_cast<float4*>(np), features);
    return cudaGetLastError();
}

}  // namespace mk
