// mk_internal.h — host/device shared declarations of libmechanic_b200.
#pragma once

#include <algorithm>
#include <cstdint>
#include <functional>
#include <cuda_runtime.h>

#include "../../include/mechanic_b200.h"

namespace mk {

inline uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

// True when the byte ranges [a, a + a_bytes) and [b, b + b_bytes) share a byte.
inline bool ranges_overlap(const void* a, uint64_t a_bytes, const void* b, uint64_t b_bytes) {
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + b_bytes && y < x + a_bytes;
}

// A sort whose input and output overlap gives wrong results: with an odd
// pass count the first pass reads keys_in while it writes keys_out.
inline bool sort_buffers_overlap(const void* keys_in, const void* values_in, const void* keys_out,
                                 const void* values_out, uint32_t n) {
    const uint64_t kb = 8ull * n, vb = 4ull * n;
    return ranges_overlap(keys_in, kb, keys_out, kb) || ranges_overlap(keys_in, kb, values_out, vb) ||
           ranges_overlap(values_in, vb, keys_out, kb) || ranges_overlap(values_in, vb, values_out, vb) ||
           ranges_overlap(keys_out, kb, values_out, vb);
}

// Records the text mk_last_error() returns on this thread.
void set_last_error(const char* msg);

// Per-tick values the host writes before each graph launch (64 bytes).
struct DevTick {
    uint32_t tick_index;
    uint32_t snapshot_slot;
    uint32_t generation;       // dispatch counter of the handle (never repeats, unlike tick_index)
    uint32_t pad[13];
};

// Counts produced on the device during a tick.  `prev_*` describe the
// contact list of the previous tick, which doubles as the manifold cache.
struct DevCounts {
    // reset at the start of every tick (first kResetWords words)
    uint32_t pairs;            // candidate pairs stored (clamped to capacity)
    uint32_t narrow;           // narrowphase contacts stored
    uint32_t contacts;         // narrowphase + ground contacts stored
    uint32_t active;           // active contacts
    uint32_t pairs_found;      // candidate pairs found by the traversal
    uint32_t requested_contacts;
    uint32_t cross_nodes;      // entries of StepBuffers::cross_nodes
    uint32_t reset_pad;
    // carried across ticks
    uint32_t prev_narrow;      // previous tick: narrowphase contacts
    uint32_t prev_contacts;    // previous tick: all contacts
    uint32_t prev_tick;        // previous tick index
    uint32_t prev_valid;       // 1 when the previous list may be matched
    uint32_t prev_indexed;     // 1 when the previous tick's prepare wrote its run index
    uint32_t pad[3];
};
constexpr uint32_t kCountResetBytes = 8 * sizeof(uint32_t);

// Solver-side constants of a handle.
// Bits of the spatial Morton key per mode (MK_MORTON_*), and of the sort key
// once a batch's scene index sits above it.
__host__ __device__ inline uint32_t spatial_key_bits(uint32_t mode) {
    return mode == MK_MORTON_REFERENCE_30 || mode == MK_MORTON_30_ADAPTIVE ? 30u
           : mode == MK_MORTON_39                                        ? 39u
           : mode == MK_MORTON_48                                        ? 48u
                                                                         : 63u;
}
__host__ __device__ inline uint32_t sort_key_bits(uint32_t mode, uint32_t scene_bits) {
    const uint32_t w = spatial_key_bits(mode) + scene_bits;
    return w < 63u ? w : 63u;
}
// Batched scenes: the scene index above the spatial key; when both do not fit
// in 63 bits the spatial key loses its lowest bits.
__host__ __device__ inline uint64_t compose_key(uint32_t mode, uint32_t scene_bits, uint64_t scene, uint64_t key) {
    if (!scene_bits) return key;
    const uint32_t w = spatial_key_bits(mode);
    if (w + scene_bits <= 63u) return (scene << w) | key;
    return (scene << (63u - scene_bits)) | (key >> (w + scene_bits - 63u));
}

struct StepParams {
    float dt, gravity, lin_damp, ang_damp;
    uint32_t body_count, collider_count, pair_capacity, suppression_count;
    uint32_t pair_shift;       // bits of a collider index inside a pair key
    uint32_t scene_bits;       // batched scenes: bits of the scene index above each collider's Morton key
    uint32_t clipped_manifold; // MK_MANIFOLD_CLIPPED: up to four points per colliding pair
    float contact_tol;         // > 0: iterate the contact solve to ||r|| <= tol * ||r_cold||
    uint32_t contact_max_iterations;
};

// Outcome of a contact solve run to a residual (written by the solver).
struct SolveStats {
    uint32_t iterations;       // solve + apply passes executed, the warm pass included
    uint32_t chosen;           // 0: cached (reference) warm start, 1: learned warm start
    uint32_t converged;
    uint32_t pad;
    double s0, sk;             // squared norms of the cold and of the last residual
};

// Launches implemented in mk_sort.cu.
uint32_t sort_passes(uint32_t key_bits);
void set_sort_items(uint32_t items);
uint32_t sort_items_for(uint32_t n, int sm_count);   // keys per thread of the onesweep tile by size
bool valid_sort_items(uint32_t items);              // 2, 4, 6, 8, 11 or 16 keys per thread
cudaError_t sort_prepare();   // per-device kernel attributes; call outside stream capture
// Default CTAs per SM of each onesweep shape, and the fixed shape of the pair-key
// sort (its count is only known on the device).
inline uint32_t default_sort_ctas(uint32_t items) {
    return items == 32 ? 1u : items >= 11 ? 2u : items == 8 ? 3u : 6u;
}
uint32_t pair_sort_items();                  // keys per thread of the pair-key sort's tile (MK_TUNE_PAIR_SORT_ITEMS)
void set_pair_sort_items(uint32_t items);    // 0 = the default
uint64_t sort_scratch_bytes(uint32_t n, uint32_t key_bits, bool values = true);
cudaError_t launch_sort(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out, uint32_t* vals_out,
                        uint32_t n, const uint32_t* n_dev, uint32_t key_bits, void* scratch,
                        uint64_t scratch_bytes, uint32_t* error_flags, cudaStream_t stream, int sm_count,
                        uint32_t items = 0, uint32_t ctas_per_sm = 0, bool precleared = false);
void sort_clear_region(void* scratch, uint32_t n, uint32_t key_bits, bool values, void** ptr, uint64_t* bytes);

// Device buffers of one handle's step (all device pointers).
struct StepBuffers {
    float4 *pos, *rot, *lin, *ang;
    float4* vel_iter;            // (iterations - 1) x {lin, ang} x body_count: per-iteration velocities
    const float* inv_mass;
    const float4* mass;          // GpuMass rows (4 x float4)
    float4* world_mass;          // 3 x float4 per body
    const uint32_t* root_flags;
    const uint32_t* components;  // null unless mechanism self-collisions are disabled
    int32_t* deltas;             // 6 per body
    int32_t* deltas_extra;       // 2 buffers of 6 per body (each padded to 16 bytes): with `deltas`, the
                                 // rotating deltas of the fused solve
    uint32_t* body_stamp;        // generation of the last tick whose contacts touched the body
    float4 *snap_pos, *snap_rot; // ring base, slot-major
    const float4* colliders;     // GpuCollider rows (4 x float4)
    float4* boxes;               // 3 x float4 per collider (world box)
    const uint32_t* collider_body;   // per collider: its body (the collider rows' metadata.x, set at creation)
    float4* aabbs;               // 2 x float4 per collider
    uint64_t* keys;              // per collider
    uint32_t* values;            // identity
    uint64_t* skeys;             // sorted
    uint32_t* svals;
    uint2* children;             // C-1
    uint32_t* parents;           // 2C-1
    uint32_t* cross_nodes;       // C-1: this tick's internal nodes whose leaf range crosses a 32-leaf chunk
    uint2* node_ranges;          // C-1: first and last sorted leaf below each internal node
    float4* leaf_scan;           // 4 per leaf: prefix and suffix unions within its 32-leaf chunk
    float4* chunk_scan;          // 6 per chunk: total, prefix and suffix unions within its 1024-leaf super-chunk
    float4* super_table;         // 2 x super-chunks x levels: sparse table of super-chunk totals
    float4* chunk_table;         // 2 x chunks x 4: sparse table levels 1-4 of chunk totals within a super-chunk
    uint2* contact_index;        // [parity][narrow, ground][collider]: {tick, first row} of the collider's run
    uint32_t* ground_mask;       // a bit per collider: touches the ground plane this tick
    uint32_t* ground_tile_count; // touching colliders per 1,024-collider tile (zeroed per tick)
    float4* node_aabbs;          // 2 x float4 per node (union boxes)
    float4* node_records;        // 8 x float4 per internal node (4-wide record of its grandchildren)
    const uint2* suppressed;
    uint64_t* pair_stage;        // pair keys as found (pair_capacity)
    uint64_t* pair_keys;         // pair keys sorted: canonical pair list
    void* pair_sort_scratch;
    uint64_t pair_sort_scratch_bytes;
    GpuContact* contacts[2];     // ping-pong, pair_capacity rows each
    uint64_t* contact_keys[2];
    uint32_t* features[2];
    uint32_t* active;            // pair_capacity
    // gather form of the contact solve (heavy ticks: more active contacts than 2 x bodies)
    int32_t* contact_deltas;     // 12 per active contact: fixed-point deltas of body a, then of body b
    uint32_t* inc_count;         // per body: contacts touching it (then a countdown while listing them)
    uint32_t* inc_off;           // body_count + 1: each body's first entry in inc_list
    uint32_t* inc_list;          // 2 x pair_capacity: 2 t + side of every active contact t, grouped by body
    uint32_t* inc_blocks;        // per block of the cooperative solve: its bodies' entry total
    float* lam_heavy;            // split form: running normal impulse per active contact
    uint32_t heavy_form;         // heavy ticks: MK_HEAVY_SCATTER, MK_HEAVY_GATHER or MK_HEAVY_SPLIT
    uint64_t* lookback;          // look-back words for ordered compaction
    uint64_t lookback_words;     // per site
    uint32_t* tickets;           // 8 tile tickets
    uint32_t* grid_barrier;      // arrival word of the cooperative solvers' grid barrier (zero at rest)
    GpuDiagnostics* diag;
    DevTick* tick;
    DevCounts* counts;
    void* sort_scratch;
    uint64_t sort_scratch_bytes;
    // batched scenes (null for a single scene)
    uint32_t* scene_bounds;      // 8 words, zeroed each tick: ordered max and complemented min of the centres
    uint32_t* collider_scene;    // scene of each collider
    uint32_t* scene_end;         // per scene: end of its sorted leaf positions
    uint32_t* scene_root;        // per scene: the internal node over exactly its leaves (scenes of >= 2 colliders)
    // contact solve to a residual (null unless enabled at creation)
    int64_t* deltas64;           // 2 candidates x 6 per body, fixed point x 2^32
    double* res2;                // 2 candidates x pair_capacity squared residuals
    double* res_chunks;          // 2 candidates x res_chunk_cap chunk sums
    uint32_t res_chunk_cap;
    float* lam_alt;              // learned candidate's normal impulse per active contact
    float* warm_pred;            // learned warm-start impulse per active contact (network output)
    float4* warm_features;       // 4 x float4 network inputs per active contact
    float4* vel_res;             // 4 x {lin, ang} x body_count ping-pong velocities
    SolveStats* solve_stats;
};

struct StepLaunch {
    int sm_count;
    uint32_t morton_mode;     // MK_MORTON_*
    uint32_t iterations;
    bool fuse_world_mass;     // no mechanism: integrate also writes world masses + snapshot
    bool collisions;
    bool learned_warm;        // run the learned warm start next to the cached one
    // launch shapes (0 = default); picked by mk_autotune or mk_set_handle_tuning
    uint32_t sort_items;      // keys per thread of the collider sort's onesweep tile (0: size-based)
    uint32_t sort_ctas;       // onesweep CTAs per SM
    uint32_t append_ctas;     // CTAs per SM of the ordered-append kernels (narrowphase, ground, prepare)
    uint32_t solve_items;     // 0: every block joins the cooperative solve; n: blocks for n contacts per thread
};

// Device regions to clear at the start of a tick (16-byte aligned, sizes in 16-byte units).
struct ZeroList {
    static constexpr uint32_t kMax = 16;   // a tick adds at most 12 regions
    uint4* ptr[kMax];
    uint64_t n16[kMax];
    uint32_t count;
    uint32_t dropped;                      // regions that did not fit (the tick refuses to run)
    void add(void* p, uint64_t bytes) {
        if (!p || bytes == 0) return;
        if (count >= kMax) {
            ++dropped;
            return;
        }
        ptr[count] = reinterpret_cast<uint4*>(p);
        n16[count] = (bytes + 15) / 16;   // the arena pads every buffer to 256 bytes
        ++count;
    }
};

// mk_step.cu
cudaError_t launch_tick_reset(const ZeroList& z, int sm_count, cudaStream_t s);
cudaError_t launch_integrate(const StepBuffers& b, const StepParams& p, const StepLaunch& l, cudaStream_t s);
cudaError_t launch_world_masses(const StepBuffers& b, const StepParams& p, cudaStream_t s);
cudaError_t launch_snapshot(const StepBuffers& b, const StepParams& p, cudaStream_t s);
cudaError_t launch_broadphase(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                              cudaStream_t s);
cudaError_t launch_narrowphase(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                               cudaStream_t s);
cudaError_t launch_warm_features(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                 cudaStream_t s);
cudaError_t launch_warm_impulses(const StepBuffers& b, const StepLaunch& l, const float* y, cudaStream_t s);
cudaError_t launch_warm_targets(const StepBuffers& b, int parity, uint32_t A, float* targets, cudaStream_t s);
cudaError_t launch_contact_solver(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                  cudaStream_t s, const std::function<cudaError_t()>& before_solve = nullptr);
cudaError_t launch_finish_tick(const StepBuffers& b, const StepParams& p, int parity, cudaStream_t s);
// Contact solve forms of heavy ticks (MK_TUNE_HEAVY_SOLVE).
constexpr uint32_t MK_HEAVY_SCATTER = 1, MK_HEAVY_GATHER = 2, MK_HEAVY_SPLIT = 3;
void set_heavy_solve_form(uint32_t form);   // 0 = the default form
uint32_t heavy_solve_form();
// Contact iterations as separate launches with a hook after each velocity
// apply (bearing projection of mechanisms with a dynamic root).
cudaError_t launch_contact_solver_stepwise(const StepBuffers& b, const StepParams& p, const StepLaunch& l, int parity,
                                           bool serial, const std::function<cudaError_t(bool)>& after_apply,
                                           cudaStream_t s);
cudaError_t launch_apply_impulse(const StepBuffers& b, uint32_t body, float3 point, float3 impulse,
                                 cudaStream_t s);
cudaError_t launch_obb_sat(const float* boxes_a, const float* boxes_b, uint32_t count, float* np,
                           uint32_t* features, cudaStream_t s);

}  // namespace mk
