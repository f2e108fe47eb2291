// mk_api.cu — C ABI of libmechanic_b200: the GpuPhysics replacement
// (crates/mechanic-gpu/src/device.rs:369-1663) over CUDA streams and graphs.
//
// One handle = one scene on one device: a single device arena holds every
// buffer, one stream orders all work, and each tick is one CUDA graph launch
// (two graphs, one per contact-buffer parity, because the previous tick's
// contact list is the manifold cache of the next).
#include <cmath>
#include <cstdarg>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mk_device.cuh"
#include "mk_internal.h"
#include "mk_mechanism.h"
#include "mk_mlp.h"

namespace {

thread_local std::string g_last_error;

constexpr uint32_t kTickRing = 64;       // tick-config slots in flight

static bool valid_morton_mode(uint32_t m) {
    return m == MK_MORTON_63 || m == MK_MORTON_REFERENCE_30 || m == MK_MORTON_48 || m == MK_MORTON_39 ||
           m == MK_MORTON_30_ADAPTIVE;
}
constexpr uint32_t kStageEvents = 8;

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void set_error(MkError* err, int code, const char* fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    if (err) {
        std::memset(err, 0, sizeof(*err));
        err->code = code;
        std::snprintf(err->message, sizeof(err->message), "%s", buf);
    }
}

}  // namespace

void mk::set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

struct MkHandle {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    MkConfig config{};
    mk::StepParams params{};
    mk::StepLaunch launch{};
    mk::StepBuffers buf{};
    mk::MechBuffers mech{};
    mk::MechParams mech_params{};
    uint32_t B = 0, C = 0, J = 0, S = 0, Q = 0, max_depth = 0, closure_count = 0;
    uint32_t pair_capacity = 0;
    bool mechanism_active = false;
    bool collisions = false;
    // memory
    void* arena = nullptr;
    size_t arena_bytes = 0;
    float4* staging = nullptr;          // 2 x float4 per body (interleaved transforms)
    float4* snap_staging = nullptr;     // the same for snapshot reads on copy_stream
    // Snapshot reads run on their own stream: a read of slot s waits for the
    // tick that last wrote s (slot_written), and the next tick that writes s
    // waits for the read (slot_read), so reading tick k's slot overlaps the
    // ticks dispatched after it.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t slot_written[3] = {};
    cudaEvent_t slot_read[3] = {};
    bool slot_read_pending[3] = {};
    // the same for interpolations, which run on the caller's stream
    cudaEvent_t slot_interp[3] = {};
    bool slot_interp_pending[3] = {};
    // published snapshot pair (runtime.rs:60-75, publish_tick :222-237): the
    // two most recently dispatched ticks' slots
    uint64_t pub_generation = 0;
    uint64_t pub_prev_tick = 0, pub_cur_tick = 0;
    uint8_t pub_prev_slot = 0, pub_cur_slot = 0;
    // host
    mk::DevTick* h_tick = nullptr;      // tick rows as dispatched (a ring: at most kTickRing ticks in flight)
    GpuDiagnostics* h_diag = nullptr;   // pinned, written at the end of every tick
    mk::SolveStats* h_stats = nullptr;  // pinned, contact solve outcome (residual mode)
    mk::ClosureState* h_cstate = nullptr;   // pinned, closure solve outcome (MK_CLOSURE_PCG_RESIDUAL)
    GpuDiagnostics* d_diag = nullptr;   // the three pinned rows above as device addresses
    mk::SolveStats* d_stats = nullptr;
    mk::ClosureState* d_cstate = nullptr;
    bool residual = false;              // contact solve runs to a residual
    float* warm_params = nullptr;       // warm-start network parameters (device, mlp::kParams)
    void* mlp_scratch = nullptr;        // bf16 weights + partials of the network kernels
    uint64_t mlp_scratch_bytes = 0;
    cudaEvent_t tick_done[kTickRing] = {};
    uint64_t tick_sub[kTickRing] = {};
    cudaEvent_t stage[kStageEvents] = {};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int parity = 0;                     // parity of the next tick's contact buffer
    uint64_t submissions = 0;
    uint64_t last_submission = 0;
    bool any_tick = false;
    uint32_t kernels_per_tick = 0;
    std::vector<uint32_t> mech_level_offsets;   // host side of MechBuffers::level_offsets
    std::vector<uint32_t> scene_body_offsets;      // batched scenes: body / collider offset per scene (+ totals)
    std::vector<uint32_t> scene_collider_offsets;
    uint32_t scene_count = 0;
};

namespace {

bool check(cudaError_t e, MkError* err, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(err, MK_ERR_DEVICE_FAILURE, "%s: %s", what, cudaGetErrorString(e));
    return false;
}

// Bump allocator over one device arena.
struct Carver {
    char* base = nullptr;
    uint64_t off = 0;
    template <class T>
    T* take(uint64_t count) {
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += mk::align256(count * sizeof(T) + (count == 0 ? 16 : 0));
        return p;
    }
};

uint32_t pick(uint32_t v, uint32_t fallback) { return v ? v : fallback; }

// Lays out every buffer of the handle; with base == nullptr it only sizes.
uint64_t carve(MkHandle* h, char* base) {
    Carver c{base, 0};
    const uint32_t B = std::max(h->B, 1u), C = std::max(h->C, 1u);
    const uint64_t P = h->pair_capacity;
    mk::StepBuffers& b = h->buf;
    b.pos = c.take<float4>(B);
    b.rot = c.take<float4>(B);
    b.lin = c.take<float4>(B);
    b.ang = c.take<float4>(B);
    b.vel_iter = c.take<float4>(2ull * B * std::max(1u, h->launch.iterations - 1));
    b.inv_mass = c.take<float>(B);
    b.mass = c.take<float4>(4ull * B);
    b.world_mass = c.take<float4>(3ull * B);
    b.root_flags = c.take<uint32_t>(B);
    b.components = nullptr;
    b.deltas = c.take<int32_t>(6ull * B);
    b.deltas_extra = c.take<int32_t>(2 * ((6ull * B + 3) & ~3ull));
    b.body_stamp = c.take<uint32_t>(B);
    b.snap_pos = c.take<float4>(3ull * B);
    b.snap_rot = c.take<float4>(3ull * B);
    b.colliders = c.take<float4>(4ull * C);
    b.boxes = c.take<float4>(3ull * C);
    b.collider_body = c.take<uint32_t>(C);
    b.aabbs = c.take<float4>(2ull * C);
    b.keys = c.take<uint64_t>(C);
    b.values = c.take<uint32_t>(C);
    b.skeys = c.take<uint64_t>(C);
    b.svals = c.take<uint32_t>(C);
    b.children = c.take<uint2>(C);
    b.parents = c.take<uint32_t>(2ull * C);
    b.cross_nodes = c.take<uint32_t>(C);
    b.scene_bounds = c.take<uint32_t>(8);
    b.node_ranges = c.take<uint2>(C);
    b.leaf_scan = c.take<float4>(4ull * C);
    b.chunk_scan = c.take<float4>(6ull * ((C + 31) / 32));
    b.chunk_table = c.take<float4>(8ull * ((C + 31) / 32));
    b.contact_index = c.take<uint2>(4ull * C);
    b.ground_mask = c.take<uint32_t>((C + 31) / 32);
    b.ground_tile_count = c.take<uint32_t>((C + 1023) / 1024);
    {
        const uint64_t ns = (C + 1023) / 1024;
        uint64_t levels = 1;
        while ((1ull << levels) <= ns) ++levels;
        b.super_table = c.take<float4>(2 * ns * levels);
    }
    b.node_aabbs = c.take<float4>(4ull * C);
    b.node_records = c.take<float4>(8ull * C);   // 128-byte 4-wide record per internal node
    b.suppressed = c.take<uint2>(std::max(h->S, 1u));
    b.pair_stage = c.take<uint64_t>(P);
    b.pair_keys = c.take<uint64_t>(P);
    b.pair_sort_scratch_bytes = mk::sort_scratch_bytes((uint32_t)P, 2 * h->params.pair_shift, false);
    b.pair_sort_scratch = c.take<char>(b.pair_sort_scratch_bytes);
    for (int k = 0; k < 2; ++k) {
        b.contacts[k] = c.take<GpuContact>(P);
        b.contact_keys[k] = c.take<uint64_t>(P);
        b.features[k] = c.take<uint32_t>(P);
    }
    b.active = c.take<uint32_t>(P);
    b.contact_deltas = c.take<int32_t>(12 * P);
    b.inc_count = c.take<uint32_t>(B);
    b.inc_off = c.take<uint32_t>(B + 1ull);
    b.inc_list = c.take<uint32_t>(2 * P);
    b.inc_blocks = c.take<uint32_t>(1024);
    b.lam_heavy = c.take<float>(P);
    b.lookback_words = std::max<uint64_t>(P / 256 + 2, C / 256 + 2);
    b.lookback = c.take<uint64_t>(4 * b.lookback_words);
    b.tickets = c.take<uint32_t>(16);
    b.grid_barrier = c.take<uint32_t>(64);
    b.diag = c.take<GpuDiagnostics>(1);
    b.tick = c.take<mk::DevTick>(1);
    b.counts = c.take<mk::DevCounts>(1);
    if (h->scene_count > 1) {
        b.collider_scene = c.take<uint32_t>(C);
        b.scene_end = c.take<uint32_t>(h->scene_count);
        b.scene_root = c.take<uint32_t>(h->scene_count);
    }
    b.sort_scratch_bytes = mk::sort_scratch_bytes(C, 63);
    b.sort_scratch = c.take<char>(b.sort_scratch_bytes);
    h->staging = c.take<float4>(2ull * B);
    h->snap_staging = c.take<float4>(2ull * B);
    if (h->residual) {
        b.deltas64 = c.take<int64_t>(12ull * B);
        b.res2 = c.take<double>(2 * P);
        b.res_chunk_cap = (uint32_t)(P / 1024 + 1);
        b.res_chunks = c.take<double>(2ull * b.res_chunk_cap);
        b.lam_alt = c.take<float>(P);
        b.warm_pred = c.take<float>(P);
        b.warm_features = c.take<float4>(4 * P);
        h->warm_params = c.take<float>(mk::mlp::kParams + 16);
        h->mlp_scratch_bytes = mk::mlp::scratch_bytes(0);
        h->mlp_scratch = c.take<char>(h->mlp_scratch_bytes);
        b.vel_res = c.take<float4>(8ull * B);
        b.solve_stats = c.take<mk::SolveStats>(1);
    }
    // mechanism buffers
    if (h->mechanism_active || h->J > 0) {
        mk::carve_mechanism(h->mech, h->mech_params, h->B, h->J, h->Q,
                            [&](uint64_t bytes) { return c.take<char>(bytes); });
    }
    if (h->config.mechanism_self_collisions == 0) b.components = c.take<uint32_t>(B);
    return c.off;
}

// The tick's config row, passed by value.  A host-to-device copy there is a
// copy-engine operation between two ticks: it queues behind a snapshot read
// in flight on the copy engines and holds the next tick back by the read's
// length.
__global__ void k_set_tick(mk::DevTick* dst, mk::DevTick v) {
    if (threadIdx.x == 0) *dst = v;
}

// End-of-tick host rows (diagnostics, solve outcomes), stored by the device
// into pinned host memory mapped into its address space: no copy-engine
// operation inside the tick either.
struct HostRows {
    const uint32_t* src[3];
    uint32_t* dst[3];
    uint32_t words[3];
    uint32_t count;
};
__global__ void k_publish_host_rows(HostRows r) {
    for (uint32_t c = 0; c < r.count; ++c)
        for (uint32_t i = threadIdx.x; i < r.words[c]; i += blockDim.x) r.dst[c][i] = __ldcg(r.src[c] + i);
    __threadfence_system();
}
static_assert(sizeof(GpuDiagnostics) % 4 == 0 && sizeof(mk::SolveStats) % 4 == 0 &&
              sizeof(mk::ClosureState) % 4 == 0, "host rows are copied as 32-bit words");

// The full tick on `stream` (captured into a graph or launched directly).
cudaError_t enqueue_tick(MkHandle* h, int parity, bool capturing) {
    cudaStream_t s = h->stream;
    mk::StepBuffers& b = h->buf;
    // Stage boundaries: external event-record nodes inside a graph, plain
    // records when launched directly.
    auto mark = [&](int i) -> cudaError_t {
        return capturing ? cudaEventRecordWithFlags(h->stage[i], s, cudaEventRecordExternal)
                         : cudaEventRecord(h->stage[i], s);
    };
    cudaError_t e;
    if ((e = mark(0)) != cudaSuccess) return e;
    {   // everything the tick needs at zero, in one launch
        mk::ZeroList z{};
        z.add(b.diag, sizeof(GpuDiagnostics));
        z.add(b.counts, mk::kCountResetBytes);
        z.add(b.tickets, 16 * sizeof(uint32_t));
        if (h->residual) z.add(b.solve_stats, sizeof(mk::SolveStats));
        if (h->collisions) {
            z.add(b.deltas, sizeof(int32_t) * 6ull * std::max(h->B, 1u));
            z.add(b.scene_bounds, 8 * sizeof(uint32_t));
            z.add(b.grid_barrier, 64 * sizeof(uint32_t));
            z.add(b.ground_tile_count, sizeof(uint32_t) * ((h->C + 1023) / 1024));
            z.add(b.lookback, sizeof(uint64_t) * 4 * b.lookback_words);
            void* r = nullptr;
            uint64_t rb = 0;
            const uint32_t key_bits = mk::sort_key_bits(h->launch.morton_mode, h->params.scene_bits);
            mk::sort_clear_region(b.sort_scratch, h->C, key_bits, true, &r, &rb);
            z.add(r, rb);
            mk::sort_clear_region(b.pair_sort_scratch, h->pair_capacity, 2 * h->params.pair_shift, false, &r, &rb);
            z.add(r, rb);
        }
        if (h->mechanism_active) z.add(h->mech.deltas, 24ull * std::max(h->B, 1u));
        if (h->mechanism_active) {   // the closure loop's barrier word and per-step maxima
            void* mp[2];
            uint64_t mb[2];
            uint32_t mc = 0;
            mk::mechanism_tick_clears(h->mech, h->mech_params, mp, mb, &mc);
            for (uint32_t k = 0; k < mc; ++k) z.add(mp[k], mb[k]);
        }
        if (z.dropped) return cudaErrorInvalidValue;   // more per-tick clears than the list holds
        cudaError_t ez = mk::launch_tick_reset(z, h->sm_count, s);
        if (ez != cudaSuccess) return ez;
    }
    const bool fuse = !h->mechanism_active;
    mk::StepLaunch l = h->launch;
    l.fuse_world_mass = fuse;
    if ((e = mk::launch_integrate(b, h->params, l, s)) != cudaSuccess) return e;
    if ((e = mark(1)) != cudaSuccess) return e;
    if (h->mechanism_active) {
        if ((e = mk::enqueue_mechanism(h->mech, b, h->mech_params, s)) != cudaSuccess) return e;
    }
    if ((e = mark(2)) != cudaSuccess) return e;
    if (h->collisions) {
        if (!fuse && (e = mk::launch_world_masses(b, h->params, s)) != cudaSuccess) return e;
        if ((e = mk::launch_broadphase(b, h->params, l, parity, s)) != cudaSuccess) return e;
        if ((e = mark(3)) != cudaSuccess) return e;
        if ((e = mk::launch_narrowphase(b, h->params, l, parity, s)) != cudaSuccess) return e;
        if ((e = mark(4)) != cudaSuccess) return e;
        if (h->mechanism_active && h->mech_params.has_dynamic_root) {
            if ((e = mk::enqueue_contact_solver_with_bearings(h->mech, b, h->params, h->mech_params, l, parity, s)) !=
                cudaSuccess)
                return e;
        } else {
            std::function<cudaError_t()> warm;
            if (h->residual) {
                warm = [&]() -> cudaError_t {
                    cudaError_t ew = mk::launch_warm_features(b, h->params, l, parity, s);
                    if (ew != cudaSuccess || !l.learned_warm) return ew;
                    // network output (one column) into lam_alt, which the solve overwrites later
                    ew = mk::mlp::forward(h->warm_params, reinterpret_cast<const float*>(b.warm_features), 0,
                                          &b.counts->active, h->pair_capacity, b.lam_alt, 1, h->mlp_scratch,
                                          &b.diag->error_flags, s);
                    if (ew != cudaSuccess) return ew;
                    return mk::launch_warm_impulses(b, l, b.lam_alt, s);
                };
            }
            if ((e = mk::launch_contact_solver(b, h->params, l, parity, s, warm)) != cudaSuccess) return e;
        }
        if (h->mechanism_active) {
            if ((e = mk::enqueue_post_contact(h->mech, b, h->mech_params, s)) != cudaSuccess) return e;
        }
    } else {
        if ((e = mark(3)) != cudaSuccess) return e;
        if ((e = mark(4)) != cudaSuccess) return e;
    }
    if ((e = mark(5)) != cudaSuccess) return e;
    if (h->mechanism_active) mk::enqueue_validate_state(h->mech, b, h->mech_params, s);
    if (h->J > 0) mk::enqueue_validate_bearings(h->mech, b, h->mech_params, h->mechanism_active, s);
    if ((e = mark(6)) != cudaSuccess) return e;
    if (!fuse && (e = mk::launch_snapshot(b, h->params, s)) != cudaSuccess) return e;
    if (h->collisions && (e = mk::launch_finish_tick(b, h->params, parity, s)) != cudaSuccess) return e;
    {
        HostRows r{};
        auto add = [&](const void* src, void* dst, size_t bytes) {
            r.src[r.count] = static_cast<const uint32_t*>(src);
            r.dst[r.count] = static_cast<uint32_t*>(dst);
            r.words[r.count] = (uint32_t)(bytes / 4);
            ++r.count;
        };
        add(b.diag, h->d_diag, sizeof(GpuDiagnostics));
        if (h->residual) add(b.solve_stats, h->d_stats, sizeof(mk::SolveStats));
        if (h->mechanism_active && mk::pcg_residual_mode(h->mech_params))
            add(h->mech.cstate, h->d_cstate, sizeof(mk::ClosureState));
        k_publish_host_rows<<<1, 32, 0, s>>>(r);
    }
    if ((e = mark(7)) != cudaSuccess) return e;
    return cudaGetLastError();
}

bool build_graphs(MkHandle* h, MkError* err) {
    for (int p = 0; p < 2; ++p) {
        cudaGraph_t g = nullptr;
        if (!check(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), err, "begin capture"))
            return false;
        cudaError_t e = enqueue_tick(h, p, true);
        cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        if (!check(e, err, "capture tick") || !check(e2, err, "end capture")) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        size_t nodes = 0;
        cudaGraphGetNodes(g, nullptr, &nodes);
        std::vector<cudaGraphNode_t> list(nodes);
        cudaGraphGetNodes(g, list.data(), &nodes);
        uint32_t kernels = 0;
        for (cudaGraphNode_t n : list) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(n, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
        }
        h->kernels_per_tick = kernels;
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (!check(e, err, "instantiate tick graph")) return false;
        h->graph[p] = exec;
    }
    return true;
}

template <class T>
cudaError_t upload(T* dst, const void* src, uint64_t count, cudaStream_t s) {
    if (!src || count == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
}

// Generation of a loaded scene (runtime.rs:139, changes whenever a scene is
// loaded): one process-wide counter for handle creation and state loads.
uint64_t next_generation() {
    static std::atomic<uint64_t> counter{0};
    return counter.fetch_add(1) + 1;
}

// Render hand-off between the published pair of snapshot slots: positions
// lerp(p0, p1, alpha); rotations the shortest-arc slerp of q0 and q1 (q1
// negated when q0 . q1 < 0), a normalised lerp when they are within 0.0316
// rad (dot > 0.9995), where slerp's sin(theta) loses its digits.
__global__ void k_interpolate_snapshot(const float4* __restrict__ p0, const float4* __restrict__ q0,
                                       const float4* __restrict__ p1, const float4* __restrict__ q1, float alpha,
                                       float4* __restrict__ pos_out, float4* __restrict__ rot_out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(p0 + i), b = __ldg(p1 + i);
    pos_out[i] = make_float4(a.x + (b.x - a.x) * alpha, a.y + (b.y - a.y) * alpha, a.z + (b.z - a.z) * alpha, 0.0f);
    const float4 r = __ldg(q0 + i);
    float4 t = __ldg(q1 + i);
    float d = r.x * t.x + r.y * t.y + r.z * t.z + r.w * t.w;
    if (d < 0.0f) {
        t = make_float4(-t.x, -t.y, -t.z, -t.w);
        d = -d;
    }
    float s0, s1;
    if (d > 0.9995f) {
        s0 = 1.0f - alpha;
        s1 = alpha;
    } else {
        const float theta = acosf(fminf(d, 1.0f));
        const float inv = 1.0f / sinf(theta);
        s0 = sinf((1.0f - alpha) * theta) * inv;
        s1 = sinf(alpha * theta) * inv;
    }
    float4 q = make_float4(r.x * s0 + t.x * s1, r.y * s0 + t.y * s1, r.z * s0 + t.z * s1, r.w * s0 + t.w * s1);
    const float inv_len = 1.0f / sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    rot_out[i] = make_float4(q.x * inv_len, q.y * inv_len, q.z * inv_len, q.w * inv_len);
}

// Interleaves float4 pos/rot rows into GpuTransform rows on the device.
__global__ void k_interleave(const float4* a, const float4* b, float4* out, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2ull * i] = a[i];
    out[2ull * i + 1] = b[i];
}
__global__ void k_deinterleave(const float4* in, float4* a, float4* b, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = in[2ull * i];
    b[i] = in[2ull * i + 1];
}

void destroy_handle(MkHandle* h) {
    if (!h) return;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    for (auto& gx : h->graph)
        if (gx) cudaGraphExecDestroy(gx);
    for (uint32_t i = 0; i < 3; ++i) {
        if (h->slot_written[i]) cudaEventDestroy(h->slot_written[i]);
        if (h->slot_read[i]) cudaEventDestroy(h->slot_read[i]);
        if (h->slot_interp[i]) cudaEventDestroy(h->slot_interp[i]);
    }
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    for (auto& e : h->tick_done)
        if (e) cudaEventDestroy(e);
    for (auto& e : h->stage)
        if (e) cudaEventDestroy(e);
    if (h->arena) cudaFree(h->arena);
    if (h->h_tick) cudaFreeHost(h->h_tick);
    if (h->h_diag) cudaFreeHost(h->h_diag);
    if (h->h_stats) cudaFreeHost(h->h_stats);
    if (h->h_cstate) cudaFreeHost(h->h_cstate);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// Several independent scenes as one creation: rows concatenated scene by
// scene with their indices offset (bodies, bearings, coordinates, mechanism
// components); each collider keeps the index of its scene.
struct Batch {
    MkCreation creation{};
    std::vector<GpuTransform> transforms;
    std::vector<GpuVelocity> velocities;
    std::vector<GpuMass> masses;
    std::vector<GpuSpatialInertia> inertias;
    std::vector<GpuCollider> colliders;
    std::vector<GpuBearing> bearings;
    std::vector<GpuPair> suppressed;
    std::vector<GpuMechanismBody> mech;
    std::vector<uint32_t> roots, preorder, components;
    std::vector<GpuMechanismDrive> drives;
    std::vector<uint32_t> collider_scene, body_offsets, collider_offsets;
    uint32_t scene_count = 0;
};

bool concatenate(const MkCreation* sc, uint32_t n, Batch& out, std::string& why) {
    uint64_t B = 0, C = 0, J = 0, S = 0, Q = 0;
    bool any_vel = false, any_inertia = false, any_mech = false;
    for (uint32_t i = 0; i < n; ++i) {
        const MkCreation& c = sc[i];
        if (c.body_count == 0 || !c.transforms || !c.masses || (c.collider_count && !c.colliders) ||
            (c.bearing_count && !c.bearings) || (c.suppression_count && !c.suppressed_pairs) ||
            (c.max_depth > 0 && (!c.mechanism_bodies || !c.preorder))) {
            char msg[128];
            std::snprintf(msg, sizeof(msg), "scene %u: creation arrays missing for the given counts", i);
            why = msg;
            return false;
        }
        B += c.body_count; C += c.collider_count; J += c.bearing_count; S += c.suppression_count;
        Q += c.coordinate_count;
        any_vel |= c.velocities != nullptr;
        any_inertia |= c.spatial_inertias != nullptr;
        any_mech |= c.max_depth > 0;
    }
    if (B > 0xffffffffull || C > 0xffffffffull || J > 0xffffffffull) {
        why = "batch exceeds 2^32 rows";
        return false;
    }
    out.scene_count = n;
    MkCreation& r = out.creation;
    std::memset(&r, 0, sizeof(r));
    uint32_t bo = 0, co = 0, jo = 0, qo = 0, comp_o = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const MkCreation& c = sc[i];
        out.body_offsets.push_back(bo);
        out.collider_offsets.push_back(co);
        out.transforms.insert(out.transforms.end(), c.transforms, c.transforms + c.body_count);
        if (any_vel) {
            if (c.velocities) out.velocities.insert(out.velocities.end(), c.velocities, c.velocities + c.body_count);
            else out.velocities.resize(out.velocities.size() + c.body_count, GpuVelocity{});
        }
        out.masses.insert(out.masses.end(), c.masses, c.masses + c.body_count);
        if (any_inertia) {
            if (c.spatial_inertias)
                out.inertias.insert(out.inertias.end(), c.spatial_inertias, c.spatial_inertias + c.body_count);
            else out.inertias.resize(out.inertias.size() + c.body_count, GpuSpatialInertia{});
        }
        for (uint32_t k = 0; k < c.collider_count; ++k) {
            GpuCollider g = c.colliders[k];
            g.metadata[0] += bo;
            out.colliders.push_back(g);
            out.collider_scene.push_back(i);
        }
        for (uint32_t k = 0; k < c.bearing_count; ++k) {
            GpuBearing g = c.bearings[k];
            g.metadata[0] += bo;
            g.metadata[1] += bo;
            if (g.metadata[2] != 0xffffffffu) g.metadata[2] += qo;
            out.bearings.push_back(g);
        }
        for (uint32_t k = 0; k < c.suppression_count; ++k) {
            GpuPair g = c.suppressed_pairs[k];
            g.collider_a += bo;   // suppression rows hold body pairs (lbvh.wgsl:325-345)
            g.collider_b += bo;
            out.suppressed.push_back(g);
        }
        uint32_t comp_max = 0;
        for (uint32_t k = 0; k < c.body_count; ++k) {
            const uint32_t comp = c.body_components ? c.body_components[k] : k;
            out.components.push_back(comp + comp_o);
            comp_max = std::max(comp_max, comp + 1);
            out.roots.push_back(c.root_flags ? c.root_flags[k] : 1u);
        }
        if (any_mech) {
            for (uint32_t k = 0; k < c.body_count; ++k) {
                GpuMechanismBody g{};
                if (c.max_depth > 0) {
                    g = c.mechanism_bodies[k];
                    g.metadata[0] += bo;
                    if (g.metadata[1] != 0xffffffffu) g.metadata[1] += jo;
                    g.traversal[0] += comp_o;
                    g.traversal[2] += bo;
                    g.traversal[3] += bo;
                    out.preorder.push_back(c.preorder[k] + bo);
                } else {   // a free body: its own root (device.rs:1699-1760 for a body without bearings)
                    g.metadata[0] = bo + k;
                    g.metadata[1] = 0xffffffffu;
                    g.metadata[3] = 1u;
                    g.traversal[0] = (c.body_components ? c.body_components[k] : k) + comp_o;
                    g.traversal[2] = bo + k;
                    g.traversal[3] = bo + k;
                    g.bind_relative_rotation[3] = 1.0f;
                    out.preorder.push_back(bo + k);
                }
                out.mech.push_back(g);
            }
        }
        for (uint32_t k = 0; k < c.coordinate_count; ++k) {
            GpuMechanismDrive d{};
            if (c.drives) d = c.drives[k];
            else { d.min_angle = -INFINITY; d.max_angle = INFINITY; }   // GpuMechanismDrive::PASSIVE (abi.rs:266-275)
            out.drives.push_back(d);
        }
        r.max_depth = std::max(r.max_depth, c.max_depth);
        r.closure_count += c.closure_count;
        r.has_dynamic_root |= c.has_dynamic_root;
        bo += c.body_count; co += c.collider_count; jo += c.bearing_count; qo += c.coordinate_count;
        comp_o += comp_max;
    }
    out.body_offsets.push_back(bo);
    out.collider_offsets.push_back(co);
    r.body_count = bo;
    r.collider_count = co;
    r.bearing_count = jo;
    r.suppression_count = (uint32_t)out.suppressed.size();
    r.coordinate_count = qo;
    r.transforms = out.transforms.data();
    r.velocities = any_vel ? out.velocities.data() : nullptr;
    r.masses = out.masses.data();
    r.spatial_inertias = any_inertia ? out.inertias.data() : nullptr;
    r.colliders = out.colliders.empty() ? nullptr : out.colliders.data();
    r.bearings = out.bearings.empty() ? nullptr : out.bearings.data();
    r.suppressed_pairs = out.suppressed.empty() ? nullptr : out.suppressed.data();
    r.mechanism_bodies = any_mech ? out.mech.data() : nullptr;
    r.root_flags = out.roots.data();
    r.preorder = any_mech ? out.preorder.data() : nullptr;
    r.body_components = out.components.data();
    r.drives = out.drives.empty() ? nullptr : out.drives.data();
    return true;
}

int create_impl(const MkCreation* cr, const MkConfig* config, const MkCapacities* caps, MkHandle** out, MkError* err,
                const Batch* batch) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!cr || !out) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "creation and out must be non-null");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    // Capacity checks (device.rs:405-422).
    const uint32_t max_bodies = caps ? pick(caps->max_bodies, cr->body_count) : MK_DEFAULT_MAX_BODIES;
    const uint32_t max_bearings = caps ? pick(caps->max_bearings, cr->bearing_count) : MK_DEFAULT_MAX_BEARINGS;
    const uint32_t max_colliders = caps ? pick(caps->max_colliders, cr->collider_count) : MK_DEFAULT_MAX_COLLIDERS;
    const uint32_t pair_capacity = caps ? pick(caps->pair_capacity, MK_DEFAULT_MAX_CONTACT_PAIRS)
                                        : MK_DEFAULT_MAX_CONTACT_PAIRS;
    if (cr->body_count > max_bodies) {
        set_error(err, MK_ERR_BODY_CAPACITY, "scene requires %u bodies but capacity is %u", cr->body_count, max_bodies);
        err ? (err->required = cr->body_count, err->capacity = max_bodies) : 0;
        return MK_ERR_BODY_CAPACITY;
    }
    if (cr->bearing_count > max_bearings) {
        set_error(err, MK_ERR_BEARING_CAPACITY, "scene requires %u bearings but capacity is %u", cr->bearing_count,
                  max_bearings);
        err ? (err->required = cr->bearing_count, err->capacity = max_bearings) : 0;
        return MK_ERR_BEARING_CAPACITY;
    }
    if (cr->collider_count > max_colliders) {
        set_error(err, MK_ERR_COLLIDER_CAPACITY, "scene requires %u colliders but capacity is %u", cr->collider_count,
                  max_colliders);
        err ? (err->required = cr->collider_count, err->capacity = max_colliders) : 0;
        return MK_ERR_COLLIDER_CAPACITY;
    }
    if (cr->body_count == 0 || !cr->transforms || !cr->masses ||
        (cr->collider_count && !cr->colliders) || (cr->bearing_count && !cr->bearings) ||
        (cr->suppression_count && !cr->suppressed_pairs) ||
        (cr->max_depth > 0 && (!cr->mechanism_bodies || !cr->preorder))) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "creation arrays missing for the given counts");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (config && !valid_morton_mode(config->morton_mode)) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "unknown morton_mode %u", config->morton_mode);
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (pair_capacity == 0 || pair_capacity > (1u << 30)) {
        set_error(err, MK_ERR_PAIR_CAPACITY, "pair capacity %u outside 1..2^30", pair_capacity);
        return MK_ERR_PAIR_CAPACITY;
    }
    MkHandle* h = new MkHandle();
    if (config) h->config = *config;
    else mk_config_default(&h->config);
    h->device = h->config.device;
    DeviceGuard guard(h->device);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || h->device < 0 || h->device >= ndev) {
        set_error(err, MK_ERR_DEVICE_FAILURE, "CUDA device %d unavailable", h->device);
        delete h;
        return MK_ERR_DEVICE_FAILURE;
    }
    cudaSetDevice(h->device);
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    h->B = cr->body_count;
    h->C = cr->collider_count;
    h->J = cr->bearing_count;
    h->S = cr->suppression_count;
    h->Q = cr->coordinate_count;
    h->max_depth = cr->max_depth;
    h->closure_count = cr->closure_count;
    h->pair_capacity = pair_capacity;
    if (batch && batch->scene_count > 1) {
        h->scene_count = batch->scene_count;
        h->scene_body_offsets = batch->body_offsets;
        h->scene_collider_offsets = batch->collider_offsets;
        uint32_t bits = 0;
        while ((1u << bits) < batch->scene_count) ++bits;
        h->params.scene_bits = bits;
    }
    h->mechanism_active = cr->max_depth > 0;
    h->collisions = h->config.collisions_enabled && h->C > 0;
    const MkConfig& c = h->config;
    h->params.dt = c.delta_seconds != 0.0f ? c.delta_seconds : 1.0f / 60.0f;
    h->params.gravity = c.gravity_y != 0.0f ? c.gravity_y : -9.81f;
    h->params.lin_damp = c.linear_damping != 0.0f ? c.linear_damping : 0.999f;
    h->params.ang_damp = c.angular_damping != 0.0f ? c.angular_damping : 0.98f;
    h->params.body_count = h->B;
    h->params.collider_count = h->C;
    h->params.pair_capacity = pair_capacity;
    h->params.suppression_count = h->S;
    {
        uint32_t shift = 1;
        while (shift < 31 && (1ull << shift) < (uint64_t)h->C) ++shift;
        h->params.pair_shift = shift;
    }
    h->params.clipped_manifold = c.contact_manifold == MK_MANIFOLD_CLIPPED ? 1u : 0u;
    h->params.contact_tol = c.contact_tolerance > 0.0f ? c.contact_tolerance : 0.0f;
    h->params.contact_max_iterations = c.contact_max_iterations ? c.contact_max_iterations : 512u;
    // the interleaved bearing form (dynamic-root mechanisms) keeps the fixed passes
    h->residual = h->params.contact_tol > 0.0f && !(cr->max_depth > 0 && cr->has_dynamic_root);
    if (!h->residual) h->params.contact_tol = 0.0f;
    h->launch.learned_warm = h->residual && c.warm_start == MK_WARM_LEARNED;
    h->launch.sm_count = h->sm_count;
    h->launch.morton_mode = c.morton_mode;
    h->launch.iterations = std::max(1u, c.solver_iterations ? c.solver_iterations : 8u);
    h->launch.collisions = h->collisions;
    h->mech_params = mk::make_mech_params(cr, h->params, h->launch.iterations, c.closure_mode, c.closure_tolerance,
                                          c.closure_max_iterations, c.preconditioner);
    // a batch keeps the parallel contact form (device.rs:1370-1373 picks the serial one for
    // small mechanisms): one scene's path must not depend on the batch it is stepped in
    if (h->scene_count > 1) h->mech_params.serial_contacts = 0;
    const mk::MechTopology topo = mk::derive_topology(cr, h->mech_params);

    bool ok = check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), err, "stream");
    ok = ok && check(mk::sort_prepare(), err, "sort kernel attributes");
    if (ok && (h->residual || h->mech_params.learned_precond))
        ok = check(mk::mlp::init(), err, "network kernel attributes");
    const uint64_t bytes = ok ? carve(h, nullptr) : 0;
    ok = ok && check(cudaMalloc(&h->arena, bytes), err, "device arena");
    if (ok) {
        h->arena_bytes = bytes;
        carve(h, (char*)h->arena);
        ok = check(cudaMemsetAsync(h->arena, 0, bytes, h->stream), err, "clear arena");
    }
    ok = ok && check(cudaMallocHost(&h->h_tick, sizeof(mk::DevTick) * kTickRing), err, "pinned tick ring");
    ok = ok && check(cudaMallocHost(&h->h_diag, sizeof(GpuDiagnostics)), err, "pinned diagnostics");
    ok = ok && check(cudaMallocHost(&h->h_stats, sizeof(mk::SolveStats)), err, "pinned solve stats");
    ok = ok && check(cudaMallocHost(&h->h_cstate, sizeof(mk::ClosureState)), err, "pinned closure state");
    ok = ok && check(cudaHostGetDevicePointer((void**)&h->d_diag, h->h_diag, 0), err, "mapped diagnostics");
    ok = ok && check(cudaHostGetDevicePointer((void**)&h->d_stats, h->h_stats, 0), err, "mapped solve stats");
    ok = ok && check(cudaHostGetDevicePointer((void**)&h->d_cstate, h->h_cstate, 0), err, "mapped closure state");
    for (uint32_t i = 0; ok && i < kTickRing; ++i)
        ok = check(cudaEventCreateWithFlags(&h->tick_done[i], cudaEventDisableTiming), err, "event");
    for (uint32_t i = 0; ok && i < kStageEvents; ++i) ok = check(cudaEventCreate(&h->stage[i]), err, "event");
    ok = ok && check(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), err, "copy stream");
    for (uint32_t i = 0; ok && i < 3; ++i) {
        ok = check(cudaEventCreateWithFlags(&h->slot_written[i], cudaEventDisableTiming), err, "event");
        ok = ok && check(cudaEventCreateWithFlags(&h->slot_read[i], cudaEventDisableTiming), err, "event");
        ok = ok && check(cudaEventCreateWithFlags(&h->slot_interp[i], cudaEventDisableTiming), err, "event");
    }
    h->pub_generation = next_generation();
    if (!ok) {
        destroy_handle(h);
        return MK_ERR_DEVICE_FAILURE;
    }
    std::memset(h->h_diag, 0, sizeof(GpuDiagnostics));
    std::memset(h->h_stats, 0, sizeof(mk::SolveStats));
    std::memset(h->h_cstate, 0, sizeof(mk::ClosureState));
    // Upload rows (device.rs:429-523): transforms de-interleaved into SoA.
    mk::StepBuffers& b = h->buf;
    cudaStream_t s = h->stream;
    std::vector<float4> tmp(2ull * h->B);
    std::memcpy(tmp.data(), cr->transforms, sizeof(GpuTransform) * h->B);
    ok = check(upload<float4>(h->staging, tmp.data(), 2ull * h->B, s), err, "upload transforms");
    if (ok) k_deinterleave<<<(h->B + 255) / 256, 256, 0, s>>>(h->staging, b.pos, b.rot, h->B);
    if (ok && cr->velocities) {
        std::memcpy(tmp.data(), cr->velocities, sizeof(GpuVelocity) * h->B);
        ok = check(cudaStreamSynchronize(s), err, "sync");
        ok = ok && check(upload<float4>(h->staging, tmp.data(), 2ull * h->B, s), err, "upload velocities");
        if (ok) k_deinterleave<<<(h->B + 255) / 256, 256, 0, s>>>(h->staging, b.lin, b.ang, h->B);
    }
    std::vector<float> inv(h->B);
    std::vector<uint32_t> roots(h->B, 1u);
    for (uint32_t i = 0; i < h->B; ++i) inv[i] = cr->masses[i].inverse_mass[0];
    if (cr->root_flags) std::memcpy(roots.data(), cr->root_flags, 4ull * h->B);
    ok = ok && check(upload<float>(const_cast<float*>(b.inv_mass), inv.data(), h->B, s), err, "upload inverse masses");
    ok = ok && check(upload<float4>(const_cast<float4*>(b.mass), cr->masses, 4ull * h->B, s), err, "upload masses");
    ok = ok && check(upload<uint32_t>(const_cast<uint32_t*>(b.root_flags), roots.data(), h->B, s), err, "upload roots");
    ok = ok && check(upload<float4>(const_cast<float4*>(b.colliders), cr->colliders, 4ull * h->C, s), err,
                     "upload colliders");
    if (ok && h->C) {   // the traversal's same-body test reads 4 bytes per collider, not a box row
        std::vector<uint32_t> cbody(h->C);
        for (uint32_t i = 0; i < h->C; ++i) cbody[i] = cr->colliders[i].metadata[0];
        ok = check(upload<uint32_t>(const_cast<uint32_t*>(b.collider_body), cbody.data(), h->C, s), err,
                   "collider bodies");
        ok = ok && check(cudaStreamSynchronize(s), err, "sync");
    }
    if (ok && batch && h->scene_count > 1 && h->C) {
        // scene s owns sorted leaf positions [collider_offsets[s], collider_offsets[s + 1]): its
        // colliders' keys carry s in their top bits
        ok = check(upload<uint32_t>(b.collider_scene, batch->collider_scene.data(), h->C, s), err, "collider scenes");
        ok = ok && check(upload<uint32_t>(b.scene_end, batch->collider_offsets.data() + 1, h->scene_count, s), err,
                         "scene ends");
    }
    ok = ok && check(upload<uint2>(const_cast<uint2*>(b.suppressed), cr->suppressed_pairs, h->S, s), err,
                     "upload suppression");
    if (ok && b.components) {
        std::vector<uint32_t> comp(h->B);
        for (uint32_t i = 0; i < h->B; ++i) comp[i] = cr->body_components ? cr->body_components[i] : i;
        ok = check(upload<uint32_t>(const_cast<uint32_t*>(b.components), comp.data(), h->B, s), err, "components");
        ok = ok && check(cudaStreamSynchronize(s), err, "sync");
    }
    if (ok && (h->mechanism_active || h->J > 0)) ok = mk::upload_mechanism(h->mech, h->mech_params, topo, cr, s, err);
    h->mech_level_offsets = topo.level_offsets;
    h->mech.level_offsets = h->mech_level_offsets.data();
    h->mech.level_count = h->mech_level_offsets.empty() ? 0u : (uint32_t)h->mech_level_offsets.size() - 1u;
    ok = ok && check(cudaStreamSynchronize(s), err, "upload sync");
    // Snapshot ring starts as the initial pose (device.rs:666-684).
    for (uint32_t slot = 0; ok && slot < 3; ++slot) {
        ok = check(cudaMemcpyAsync(b.snap_pos + (size_t)slot * h->B, b.pos, 16ull * h->B, cudaMemcpyDeviceToDevice, s),
                   err, "snapshot init");
        ok = ok && check(cudaMemcpyAsync(b.snap_rot + (size_t)slot * h->B, b.rot, 16ull * h->B,
                                         cudaMemcpyDeviceToDevice, s), err, "snapshot init");
    }
    if (ok && h->residual) ok = check(mk::mlp::pack(h->warm_params, h->mlp_scratch, s), err, "pack network");
    ok = ok && check(cudaStreamSynchronize(s), err, "create sync");
    if (ok && h->config.use_graph) ok = build_graphs(h, err);
    if (!ok) {
        destroy_handle(h);
        return err ? err->code : MK_ERR_DEVICE_FAILURE;
    }
    *out = h;
    return MK_OK;
}

}  // namespace

extern "C" {

void mk_config_default(MkConfig* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->collisions_enabled = 1;
    c->mechanism_self_collisions = 1;
    c->solver_iterations = 8;
    c->morton_mode = MK_MORTON_39;
    c->closure_mode = MK_CLOSURE_REFERENCE;
    c->use_graph = 1;
}

const char* mk_version(void) { return "mechanic_b200 0.1.0 sm_100a"; }

int mk_set_tuning(uint32_t key, uint32_t value) {
    static uint32_t sort_items = 0;
    if (key == MK_TUNE_SORT_ITEMS) {
        const uint32_t prev = sort_items;
        sort_items = value;
        mk::set_sort_items(value);
        return (int)prev;
    }
    if (key == MK_TUNE_CLOSURE_GRID) {
        const uint32_t prev = mk::closure_grid_mode();
        mk::set_closure_grid(value);
        return (int)prev;
    }
    if (key == MK_TUNE_HEAVY_SOLVE) {
        const uint32_t prev = mk::heavy_solve_form();
        mk::set_heavy_solve_form(value);
        return (int)prev;
    }
    if (key == MK_TUNE_PAIR_SORT_ITEMS) {
        const uint32_t prev = mk::pair_sort_items();
        mk::set_pair_sort_items(value);
        return (int)prev;
    }
    return -1;
}

const char* mk_last_error(void) { return g_last_error.c_str(); }

int mk_create(const MkCreation* cr, const MkConfig* config, const MkCapacities* caps, MkHandle** out, MkError* err) {
    return create_impl(cr, config, caps, out, err, nullptr);
}

int mk_create_batch(const MkCreation* scenes, uint32_t scene_count, const MkConfig* config, const MkCapacities* caps,
                    MkHandle** out, MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!scenes || !out || scene_count == 0) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "scenes, out and scene_count > 0 required");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (scene_count > (1u << 16)) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "at most 65536 scenes per batch, %u given", scene_count);
        return MK_ERR_INVALID_ARGUMENT;
    }
    Batch batch;
    std::string why;
    if (!concatenate(scenes, scene_count, batch, why)) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "%s", why.c_str());
        return MK_ERR_INVALID_ARGUMENT;
    }
    return create_impl(&batch.creation, config, caps, out, err, &batch);
}

int mk_scene_offsets(const MkHandle* h, uint32_t* body_offsets, uint32_t* collider_offsets, uint32_t capacity) {
    if (!h) return -1;
    const uint32_t n = (uint32_t)h->scene_body_offsets.size();
    if (n == 0) {   // single scene
        if (capacity >= 2) {
            if (body_offsets) body_offsets[0] = 0, body_offsets[1] = h->B;
            if (collider_offsets) collider_offsets[0] = 0, collider_offsets[1] = h->C;
        }
        return 1;
    }
    for (uint32_t i = 0; i < n && i < capacity; ++i) {
        if (body_offsets) body_offsets[i] = h->scene_body_offsets[i];
        if (collider_offsets) collider_offsets[i] = h->scene_collider_offsets[i];
    }
    return (int)n - 1;
}


void mk_destroy(MkHandle* h) { destroy_handle(h); }

int mk_dispatch_tick(MkHandle* h, uint64_t tick_index, MkSubmission* out) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    const uint64_t sub = ++h->submissions;
    const uint32_t slot = (uint32_t)(sub % kTickRing);
    if (h->tick_sub[slot]) cudaEventSynchronize(h->tick_done[slot]);
    mk::DevTick& t = h->h_tick[slot];
    std::memset(&t, 0, sizeof(t));
    t.tick_index = (uint32_t)tick_index;    // wrapping_u32 (device.rs:868)
    t.snapshot_slot = (uint32_t)(tick_index % 3);
    t.generation = (uint32_t)sub;
    const uint32_t snap = t.snapshot_slot;
    cudaError_t e = cudaSuccess;
    if (h->slot_read_pending[snap]) {   // a read of this snapshot slot may still be copying it
        e = cudaStreamWaitEvent(h->stream, h->slot_read[snap], 0);
        h->slot_read_pending[snap] = false;
    }
    if (e == cudaSuccess && h->slot_interp_pending[snap]) {   // or an interpolation reading it
        e = cudaStreamWaitEvent(h->stream, h->slot_interp[snap], 0);
        h->slot_interp_pending[snap] = false;
    }
    if (e == cudaSuccess) {
        k_set_tick<<<1, 32, 0, h->stream>>>(h->buf.tick, t);
        e = cudaGetLastError();
    }
    const int parity = h->parity;
    if (e == cudaSuccess) {
        if (h->graph[parity]) e = cudaGraphLaunch(h->graph[parity], h->stream);
        else e = enqueue_tick(h, parity, false);
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->tick_done[slot], h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->slot_written[snap], h->stream);
    if (e != cudaSuccess) {
        set_error(nullptr, MK_ERR_DEVICE_FAILURE, "dispatch_tick: %s", cudaGetErrorString(e));
        return MK_ERR_DEVICE_FAILURE;
    }
    h->tick_sub[slot] = sub;
    h->last_submission = sub;
    h->pub_prev_slot = h->pub_cur_slot;
    h->pub_prev_tick = h->pub_cur_tick;
    h->pub_cur_slot = (uint8_t)snap;
    h->pub_cur_tick = tick_index;
    h->parity ^= (h->collisions ? 1 : 0);
    h->any_tick = true;
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->tick_index = tick_index;
        out->snapshot_slot = (uint8_t)(tick_index % 3);
        out->submission_index = sub;
    }
    return MK_OK;
}

int mk_wait(MkHandle* h, uint64_t submission) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    cudaError_t e = cudaSuccess;
    if (submission == 0 || submission >= h->last_submission) {
        e = cudaStreamSynchronize(h->stream);
    } else {
        const uint32_t slot = (uint32_t)(submission % kTickRing);
        if (h->tick_sub[slot] == submission) e = cudaEventSynchronize(h->tick_done[slot]);
    }
    if (e != cudaSuccess) {
        set_error(nullptr, MK_ERR_DEVICE_FAILURE, "wait: %s", cudaGetErrorString(e));
        return MK_ERR_DEVICE_FAILURE;
    }
    return MK_OK;
}

int mk_read_last_tick(MkHandle* h, MkTickReadback* out) {
    if (!h || !out) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        set_error(nullptr, MK_ERR_DEVICE_FAILURE, "read_last_tick: %s", cudaGetErrorString(e));
        return MK_ERR_DEVICE_FAILURE;
    }
    std::memset(out, 0, sizeof(*out));
    const GpuDiagnostics d = *h->h_diag;
    out->has_timestamps = 1;
    out->error_flags = d.error_flags;
    out->pair_count = d.pair_count;
    out->contact_count = d.contact_count;
    out->active_contact_count = d.active_contact_count;
    // diagnostic_units: micro-units to units (device.rs:1520-1521).
    out->anchor_residual_meters = (float)((double)d.max_anchor_micrometers / 1.0e6);
    out->axis_residual_degrees = (float)((double)d.max_axis_microdegrees / 1.0e6);
    if (h->any_tick) {
        float ms[kStageEvents - 1] = {};
        for (uint32_t i = 0; i + 1 < kStageEvents; ++i)
            if (cudaEventElapsedTime(&ms[i], h->stage[i], h->stage[i + 1]) != cudaSuccess) ms[i] = 0.0f;
        cudaGetLastError();
        out->kernel_timings.integration_ms = ms[0];
        out->kernel_timings.mechanism_ms = ms[1];
        out->kernel_timings.broadphase_ms = ms[2];
        out->kernel_timings.narrowphase_ms = ms[3];
        out->kernel_timings.contact_solver_ms = ms[4];
        out->kernel_timings.bearings_ms = ms[5];
        out->kernel_timings.snapshot_ms = ms[6];
        double total = 0;
        for (float m : ms) total += m;
        out->gpu_tick_ms = total;
    }
    mk::read_mechanism_readback(h->mech, h->mech_params, d, h->h_cstate, out);
    if (h->residual) {
        const mk::SolveStats st = *h->h_stats;
        out->contact_iterations = st.iterations;
        out->warm_start_used = h->launch.learned_warm ? (st.chosen ? MK_WARM_LEARNED : 2u) : MK_WARM_CACHED;
        out->contact_relative_residual = st.s0 > 0.0 ? std::sqrt(st.sk / st.s0) : 0.0;
    } else if (h->collisions && d.active_contact_count > 0) {
        out->contact_iterations = h->launch.iterations;
    }
    return MK_OK;
}

int mk_set_warm_start_network(MkHandle* h, const float* params, uint32_t count, MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!h || !params) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "handle and params must be non-null");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (!h->residual) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "the warm-start network needs contact_tolerance > 0");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (count != mk::mlp::kParams) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "network has %u parameters, %u given", mk::mlp::kParams, count);
        if (err) err->required = mk::mlp::kParams, err->provided = count;
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    cudaError_t e = cudaMemcpyAsync(h->warm_params, params, sizeof(float) * count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = mk::mlp::pack(h->warm_params, h->mlp_scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return check(e, err, "set_warm_start_network") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_set_preconditioner_network(MkHandle* h, const float* params, uint32_t count, MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!h || !params) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "handle and params must be non-null");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (!h->mech.precond_params) {
        set_error(err, MK_ERR_INVALID_ARGUMENT,
                  "the preconditioner network needs closure_mode = MK_CLOSURE_PCG_RESIDUAL, "
                  "preconditioner = MK_PRECOND_LEARNED and at least one closure");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (count != mk::mlp::kParams) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "network has %u parameters, %u given", mk::mlp::kParams, count);
        if (err) err->required = mk::mlp::kParams, err->provided = count;
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    cudaError_t e = cudaMemcpyAsync(h->mech.precond_params, params, sizeof(float) * count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = mk::mlp::pack(h->mech.precond_params, h->mech.mlp_scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return check(e, err, "set_preconditioner_network") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_read_warm_start_samples(MkHandle* h, float* features, float* targets, uint32_t capacity, uint32_t* count,
                               MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!h || !count) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "handle and count must be non-null");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *count = 0;
    if (!h->residual || !h->collisions) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "warm-start samples need collisions and contact_tolerance > 0");
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    cudaError_t e = cudaStreamSynchronize(s);
    if (!check(e, err, "read_warm_start_samples")) return MK_ERR_DEVICE_FAILURE;
    const uint32_t A = h->any_tick ? h->h_diag->active_contact_count : 0u;
    const uint32_t n = std::min(A, capacity);
    *count = A;
    if (n == 0 || !features || !targets) return MK_OK;
    mk::StepBuffers& b = h->buf;
    const int last = h->parity ^ 1;
    e = mk::launch_warm_targets(b, last, n, b.warm_pred, s);   // warm_pred is free between ticks
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(features, b.warm_features, 64ull * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(targets, b.warm_pred, 4ull * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return check(e, err, "read_warm_start_samples") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_read_snapshot(MkHandle* h, uint8_t slot, GpuTransform* out, uint32_t capacity, MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    if (slot >= 3) {
        set_error(err, MK_ERR_INVALID_SNAPSHOT_SLOT, "snapshot slot %u is outside the published ring", slot);
        if (err) err->slot = slot;
        return MK_ERR_INVALID_SNAPSHOT_SLOT;
    }
    if (!out || capacity < h->B) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "output holds %u rows, %u needed", capacity, h->B);
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    // on the copy stream, after the tick that last wrote this slot only: ticks
    // dispatched later keep running while the slot is copied
    cudaStream_t s = h->copy_stream;
    cudaError_t e = cudaStreamWaitEvent(s, h->slot_written[slot], 0);
    if (e == cudaSuccess) {
        k_interleave<<<(h->B + 255) / 256, 256, 0, s>>>(h->buf.snap_pos + (size_t)slot * h->B,
                                                         h->buf.snap_rot + (size_t)slot * h->B, h->snap_staging,
                                                         h->B);
        e = cudaMemcpyAsync(out, h->snap_staging, sizeof(GpuTransform) * h->B, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->slot_read[slot], s);
    if (e == cudaSuccess) {
        h->slot_read_pending[slot] = true;
        e = cudaEventSynchronize(h->slot_read[slot]);
    }
    if (!check(e, err, "read_snapshot")) return MK_ERR_DEVICE_FAILURE;
    return MK_OK;
}

int mk_published_state(MkHandle* h, MkPublishedState* out) {
    if (!h || !out) return MK_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->generation = h->pub_generation;
    out->previous_slot = h->pub_prev_slot;
    out->current_slot = h->pub_cur_slot;
    out->previous_tick = h->pub_prev_tick;
    out->current_tick = h->pub_cur_tick;
    out->body_count = h->B;
    out->ticks_published = h->any_tick ? (h->last_submission >= 2 ? 2u : 1u) : 0u;
    return MK_OK;
}

int mk_interpolate_snapshot(MkHandle* h, float alpha, void* positions_out, void* rotations_out, void* stream,
                            MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    if (!positions_out || !rotations_out || !(alpha >= 0.0f && alpha <= 1.0f)) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "interpolate_snapshot: null output or alpha outside [0, 1]");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if ((((uintptr_t)positions_out) | ((uintptr_t)rotations_out)) & 15u) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "interpolate_snapshot: outputs must be 16-byte aligned");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (h->B == 0) return MK_OK;
    DeviceGuard guard(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint8_t a = h->pub_prev_slot, b = h->pub_cur_slot;
    // after the ticks that wrote both slots; the next tick that rewrites either waits for this
    cudaError_t e = cudaStreamWaitEvent(s, h->slot_written[a], 0);
    if (e == cudaSuccess && b != a) e = cudaStreamWaitEvent(s, h->slot_written[b], 0);
    if (e == cudaSuccess) {
        const size_t B = h->B;
        k_interpolate_snapshot<<<(h->B + 255) / 256, 256, 0, s>>>(
            h->buf.snap_pos + a * B, h->buf.snap_rot + a * B, h->buf.snap_pos + b * B, h->buf.snap_rot + b * B, alpha,
            (float4*)positions_out, (float4*)rotations_out, h->B);
        e = cudaGetLastError();
    }
    for (uint8_t slot : {a, b}) {
        if (e == cudaSuccess) e = cudaEventRecord(h->slot_interp[slot], s);
        if (e == cudaSuccess) h->slot_interp_pending[slot] = true;
    }
    if (!check(e, err, "interpolate_snapshot")) return MK_ERR_DEVICE_FAILURE;
    return MK_OK;
}

int mk_snapshot_buffers(MkHandle* h, uint8_t slot, void** positions, void** rotations, MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    if (slot >= 3) {
        set_error(err, MK_ERR_INVALID_SNAPSHOT_SLOT, "snapshot slot %u is outside the published ring", slot);
        if (err) err->slot = slot;
        return MK_ERR_INVALID_SNAPSHOT_SLOT;
    }
    if (positions) *positions = h->buf.snap_pos + (size_t)slot * h->B;
    if (rotations) *rotations = h->buf.snap_rot + (size_t)slot * h->B;
    return MK_OK;
}

int mk_apply_impulse(MkHandle* h, uint32_t body, const float p[3], const float J[3], MkError* err) {
    if (!h || !p || !J) return MK_ERR_INVALID_ARGUMENT;
    if (body >= h->B) {
        set_error(err, MK_ERR_BODY_INDEX_OUT_OF_RANGE, "body index %u is outside the uploaded body count %u", body, h->B);
        if (err) { err->body_index = body; err->body_count = h->B; }
        return MK_ERR_BODY_INDEX_OUT_OF_RANGE;
    }
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(p[k]) || !std::isfinite(J[k])) {
            set_error(err, MK_ERR_NON_FINITE, "external impulse point and vector must be finite");
            return MK_ERR_NON_FINITE;
        }
    DeviceGuard guard(h->device);
    cudaError_t e = mk::launch_apply_impulse(h->buf, body, make_float3(p[0], p[1], p[2]), make_float3(J[0], J[1], J[2]),
                                             h->stream);
    return check(e, err, "apply_impulse") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_write_drives(MkHandle* h, const GpuMechanismDrive* drives, uint32_t count, MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    if (count != h->Q) {
        set_error(err, MK_ERR_DRIVE_STATE_COUNT, "drive state has %u rows but scene requires %u", count, h->Q);
        if (err) { err->provided = count; err->required = h->Q; }
        return MK_ERR_DRIVE_STATE_COUNT;
    }
    if (count == 0) return MK_OK;
    DeviceGuard guard(h->device);
    cudaError_t e = cudaMemcpyAsync(h->mech.drives, drives, sizeof(GpuMechanismDrive) * count, cudaMemcpyHostToDevice,
                                    h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return check(e, err, "write_drives") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_init_coordinates(MkHandle* h, const GpuMechanismCoordinate* coords, uint32_t count, MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    if (count != h->Q) {
        set_error(err, MK_ERR_COORDINATE_STATE_COUNT, "coordinate state has %u rows but scene requires %u", count,
                  h->Q);
        if (err) { err->provided = count; err->required = h->Q; }
        return MK_ERR_COORDINATE_STATE_COUNT;
    }
    if (count == 0) return MK_OK;
    DeviceGuard guard(h->device);
    cudaError_t e = cudaMemcpyAsync(h->mech.coords, coords, sizeof(GpuMechanismCoordinate) * count,
                                    cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return check(e, err, "init_coordinates") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

uint32_t mk_body_count(const MkHandle* h) { return h ? h->B : 0u; }

uint32_t mk_tick_kernel_count(const MkHandle* h) { return h ? h->kernels_per_tick : 0u; }

int mk_get_handle_tuning(const MkHandle* h, MkTuning* out) {
    if (!h || !out) return MK_ERR_INVALID_ARGUMENT;
    out->sort_items = h->launch.sort_items ? h->launch.sort_items : mk::sort_items_for(h->C, h->sm_count);
    out->sort_ctas_per_sm = h->launch.sort_ctas ? h->launch.sort_ctas : mk::default_sort_ctas(out->sort_items);
    out->append_ctas_per_sm = h->launch.append_ctas ? h->launch.append_ctas : 8u;
    out->solve_items = h->launch.solve_items;
    out->morton_mode = h->launch.morton_mode;
    return MK_OK;
}

int mk_set_handle_tuning(MkHandle* h, const MkTuning* t, MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!h || !t) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "handle and tuning must be non-null");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const bool ok_items = t->sort_items == 0 || mk::valid_sort_items(t->sort_items);
    if (!ok_items || t->sort_ctas_per_sm > 32 || t->append_ctas_per_sm > 64 || t->solve_items > 64 ||
        !valid_morton_mode(t->morton_mode)) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "tuning outside the supported shapes");
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    if (!check(cudaStreamSynchronize(h->stream), err, "set_handle_tuning sync")) return MK_ERR_DEVICE_FAILURE;
    h->launch.sort_items = t->sort_items;
    h->launch.sort_ctas = t->sort_ctas_per_sm;
    h->launch.append_ctas = t->append_ctas_per_sm;
    h->launch.solve_items = t->solve_items;
    h->launch.morton_mode = t->morton_mode;   // the sort's scratch holds 63-bit keys: any mode fits
    if (!h->config.use_graph) return MK_OK;
    for (auto& gx : h->graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    return build_graphs(h, err) ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_autotune(MkHandle* h, uint32_t ticks, MkTuning* best, double* best_ms, MkError* err) {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!h || ticks == 0) {
        set_error(err, MK_ERR_INVALID_ARGUMENT, "handle and ticks > 0 required");
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    if (!check(cudaStreamSynchronize(s), err, "autotune sync")) return MK_ERR_DEVICE_FAILURE;
    // the state every candidate starts from
    mk::DevCounts counts{};
    if (!check(cudaMemcpy(&counts, h->buf.counts, sizeof(counts), cudaMemcpyDeviceToHost), err, "autotune counts"))
        return MK_ERR_DEVICE_FAILURE;
    const uint32_t rows = h->collisions ? std::max(counts.contacts, 1u) : 1u;
    std::vector<GpuTransform> tr(h->B);
    std::vector<GpuVelocity> vel(h->B);
    std::vector<GpuMechanismCoordinate> coords(std::max(h->Q, 1u));
    std::vector<GpuContact> man(rows);
    MkHostState st{tr.data(), vel.data(), coords.data(), man.data(), rows, 0, 0};
    int rc = mk_save_state(h, &st, err);
    if (rc != MK_OK) return rc;
    const uint64_t base_tick = st.manifold_tick;
    MkHostState load = st;
    if (!h->collisions || st.manifold_count == 0) load.manifold_contacts = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto measure = [&](const MkTuning& t, double* ms) -> int {
        int r = mk_set_handle_tuning(h, &t, err);
        if (r != MK_OK) return r;
        r = mk_load_state(h, &load, err);
        if (r != MK_OK) return r;
        for (auto& gx : h->graph)
            if (gx && !check(cudaGraphUpload(gx, s), err, "graph upload")) return MK_ERR_DEVICE_FAILURE;
        MkSubmission sub;
        cudaEventRecord(e0, s);
        for (uint32_t k = 0; k < ticks; ++k)
            if ((r = mk_dispatch_tick(h, base_tick + 1 + k, &sub)) != MK_OK) return r;
        cudaEventRecord(e1, s);
        if (!check(cudaEventSynchronize(e1), err, "autotune timing")) return MK_ERR_DEVICE_FAILURE;
        float f = 0.0f;
        cudaEventElapsedTime(&f, e0, e1);
        *ms = f;
        return MK_OK;
    };
    MkTuning cur;
    mk_get_handle_tuning(h, &cur);
    double cur_ms = 0.0;
    rc = measure(cur, &cur_ms);
    // coordinate descent over the launch shapes, two sweeps
    const uint32_t sort_items[] = {4, 6, 8, 11, 16};
    const uint32_t sort_ctas[] = {1, 2, 3, 4, 6};
    const uint32_t append_ctas[] = {4, 8, 16};
    const uint32_t solve_items[] = {0, 1, 2, 4};
    // the key mode: between the two scene-adaptive widths of a handle that uses
    // one of them (every mode yields the same pairs); other modes are kept
    const uint32_t key_modes[] = {MK_MORTON_39, MK_MORTON_30_ADAPTIVE};
    const bool tune_keys = cur.morton_mode == MK_MORTON_39 || cur.morton_mode == MK_MORTON_30_ADAPTIVE;
    for (int sweep = 0; sweep < 2 && rc == MK_OK; ++sweep) {
        for (int field = 0; field < 5 && rc == MK_OK; ++field) {
            if (field == 4 && !tune_keys) continue;
            const uint32_t* vals = field == 0 ? sort_items : field == 1 ? sort_ctas : field == 2 ? append_ctas
                                   : field == 3 ? solve_items : key_modes;
            const int nv = field == 0 ? 5 : field == 1 ? 5 : field == 2 ? 3 : field == 3 ? 4 : 2;
            for (int i = 0; i < nv && rc == MK_OK; ++i) {
                MkTuning cand = cur;
                uint32_t* slot = field == 0 ? &cand.sort_items : field == 1 ? &cand.sort_ctas_per_sm
                                 : field == 2 ? &cand.append_ctas_per_sm : field == 3 ? &cand.solve_items
                                 : &cand.morton_mode;
                if (*slot == vals[i]) continue;
                *slot = vals[i];
                double ms = 0.0;
                rc = measure(cand, &ms);
                if (rc == MK_OK && ms < 0.98 * cur_ms) {   // a change must win by 2% (timing noise)
                    cur = cand;
                    cur_ms = ms;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != MK_OK) return rc;
    rc = mk_set_handle_tuning(h, &cur, err);
    if (rc == MK_OK) rc = mk_load_state(h, &load, err);
    if (rc == MK_OK && !check(cudaStreamSynchronize(s), err, "autotune restore")) rc = MK_ERR_DEVICE_FAILURE;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms / ticks;
    return rc;
}

int mk_has_gpu_timestamps(const MkHandle* h) { return h ? 1 : 0; }

int mk_state_buffers(MkHandle* h, MkDeviceState* out) {
    if (!h || !out) return MK_ERR_INVALID_ARGUMENT;
    out->positions = h->buf.pos;
    out->rotations = h->buf.rot;
    out->linear_velocities = h->buf.lin;
    out->angular_velocities = h->buf.ang;
    out->inverse_masses = const_cast<float*>(h->buf.inv_mass);
    out->coordinates = h->mech.coords;
    out->diagnostics = h->buf.diag;
    out->stream = h->stream;
    return MK_OK;
}

int mk_save_state(MkHandle* h, MkHostState* st, MkError* err) {
    if (!h || !st) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    cudaError_t e = cudaStreamSynchronize(s);
    const uint32_t B = h->B;
    if (e == cudaSuccess && st->transforms) {
        k_interleave<<<(B + 255) / 256, 256, 0, s>>>(h->buf.pos, h->buf.rot, h->staging, B);
        e = cudaMemcpyAsync(st->transforms, h->staging, 32ull * B, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess && st->velocities) {
        k_interleave<<<(B + 255) / 256, 256, 0, s>>>(h->buf.lin, h->buf.ang, h->staging, B);
        e = cudaMemcpyAsync(st->velocities, h->staging, 32ull * B, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess && st->coordinates && h->Q)
        e = cudaMemcpy(st->coordinates, h->mech.coords, sizeof(GpuMechanismCoordinate) * h->Q, cudaMemcpyDeviceToHost);
    st->manifold_count = 0;
    st->manifold_tick = 0;
    if (e == cudaSuccess && h->collisions) {
        mk::DevCounts counts;
        e = cudaMemcpy(&counts, h->buf.counts, sizeof(counts), cudaMemcpyDeviceToHost);
        const int prev = h->parity ^ 1;   // buffer written by the last completed tick
        if (e == cudaSuccess && counts.prev_valid) {
            const uint32_t n = counts.prev_contacts;
            std::vector<GpuContact> rows(n);
            std::vector<uint64_t> keys(n);
            std::vector<uint32_t> feat(n);
            e = cudaMemcpy(rows.data(), h->buf.contacts[prev], sizeof(GpuContact) * n, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess)
                e = cudaMemcpy(keys.data(), h->buf.contact_keys[prev], 8ull * n, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(feat.data(), h->buf.features[prev], 4ull * n, cudaMemcpyDeviceToHost);
            std::vector<uint32_t> order;
            for (uint32_t k = 0; k < n; ++k)
                if (feat[k] & (1u << 24)) order.push_back(k);
            std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b2) { return keys[a] < keys[b2]; });
            uint32_t m = 0;
            for (uint32_t k : order) {
                if (st->manifold_contacts && m < st->manifold_capacity) {
                    GpuContact c = rows[k];
                    c.metadata[2] = (uint32_t)(keys[k] >> 32);
                    c.metadata[3] = (uint32_t)keys[k];
                    std::memset(c.arm_b, 0, sizeof(c.arm_b));
                    st->manifold_contacts[m] = c;
                }
                ++m;
            }
            st->manifold_count = m;
            st->manifold_tick = counts.prev_tick;
        }
    }
    return check(e, err, "save_state") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_load_state(MkHandle* h, const MkHostState* st, MkError* err) {
    if (!h || !st) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    cudaStream_t s = h->stream;
    cudaError_t e = cudaStreamSynchronize(s);
    const uint32_t B = h->B;
    if (e == cudaSuccess && st->transforms) {
        e = cudaMemcpyAsync(h->staging, st->transforms, 32ull * B, cudaMemcpyHostToDevice, s);
        k_deinterleave<<<(B + 255) / 256, 256, 0, s>>>(h->staging, h->buf.pos, h->buf.rot, B);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess && st->velocities) {
        e = cudaMemcpyAsync(h->staging, st->velocities, 32ull * B, cudaMemcpyHostToDevice, s);
        k_deinterleave<<<(B + 255) / 256, 256, 0, s>>>(h->staging, h->buf.lin, h->buf.ang, B);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess && st->coordinates && h->Q)
        e = cudaMemcpy(h->mech.coords, st->coordinates, sizeof(GpuMechanismCoordinate) * h->Q, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h->collisions) {
        // The next tick reads the buffer of parity ^ 1 as its manifold.
        const int prev = h->parity ^ 1;
        const uint32_t n = st->manifold_contacts ? st->manifold_count : 0u;
        if (n > h->pair_capacity) {
            set_error(err, MK_ERR_INVALID_ARGUMENT, "manifold rows %u exceed pair capacity %u", n, h->pair_capacity);
            return MK_ERR_INVALID_ARGUMENT;
        }
        std::vector<uint32_t> order(n);
        std::vector<uint64_t> key(n);
        for (uint32_t k = 0; k < n; ++k) {
            order[k] = k;
            key[k] = ((uint64_t)st->manifold_contacts[k].metadata[2] << 32) | st->manifold_contacts[k].metadata[3];
        }
        // narrowphase rows first, then ground rows, each sorted by key
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b2) {
            const bool ga = (uint32_t)key[a] == 0xffffffffu, gb = (uint32_t)key[b2] == 0xffffffffu;
            if (ga != gb) return !ga;
            return key[a] < key[b2];
        });
        std::vector<GpuContact> rows(n);
        std::vector<uint64_t> keys(n);
        std::vector<uint32_t> feat(n, 1u << 24);
        uint32_t narrow = 0;
        for (uint32_t k = 0; k < n; ++k) {
            rows[k] = st->manifold_contacts[order[k]];
            keys[k] = key[order[k]];
            rows[k].metadata[2] = k;
            rows[k].metadata[3] = 1;
            if ((uint32_t)keys[k] != 0xffffffffu) ++narrow;
        }
        if (n) {
            e = cudaMemcpy(h->buf.contacts[prev], rows.data(), sizeof(GpuContact) * n, cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(h->buf.contact_keys[prev], keys.data(), 8ull * n, cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(h->buf.features[prev], feat.data(), 4ull * n, cudaMemcpyHostToDevice);
        }
        mk::DevCounts counts;
        if (e == cudaSuccess) e = cudaMemcpy(&counts, h->buf.counts, sizeof(counts), cudaMemcpyDeviceToHost);
        counts.prev_narrow = narrow;
        counts.prev_contacts = n;
        counts.prev_tick = (uint32_t)st->manifold_tick;
        counts.prev_valid = st->manifold_contacts ? 1u : 0u;
        counts.prev_indexed = 0u;   // a loaded list has no run index: prepare searches it
        if (e == cudaSuccess) e = cudaMemcpy(h->buf.counts, &counts, sizeof(counts), cudaMemcpyHostToDevice);
    }
    return check(e, err, "load_state") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

int mk_read_buffer(MkHandle* h, uint32_t id, void* host, uint64_t cap_bytes, uint64_t* count, MkError* err) {
    if (!h) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(h->device);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (!check(e, err, "read_buffer sync")) return MK_ERR_DEVICE_FAILURE;
    mk::DevCounts counts{};
    e = cudaMemcpy(&counts, h->buf.counts, sizeof(counts), cudaMemcpyDeviceToHost);
    const int last = h->parity ^ (h->collisions ? 1 : 0);   // parity written by the last tick
    const void* src = nullptr;
    uint64_t n = 0, row = 0;
    const mk::StepBuffers& b = h->buf;
    switch (id) {
        case MK_BUF_SORTED_KEYS: src = b.skeys; n = h->C; row = 8; break;
        case MK_BUF_SORTED_VALUES: src = b.svals; n = h->C; row = 4; break;
        case MK_BUF_COLLIDER_AABBS: src = b.aabbs; n = h->C; row = 32; break;
        case MK_BUF_NODE_CHILDREN: src = b.children; n = h->C ? h->C - 1 : 0; row = 8; break;
        case MK_BUF_NODE_AABBS: src = b.node_aabbs; n = h->C ? 2ull * h->C - 1 : 0; row = 32; break;
        case MK_BUF_NODE_RECORDS: src = b.node_records; n = h->C > 1 ? h->C - 1ull : 0; row = 128; break;
        case MK_BUF_PAIRS: src = b.pair_keys; n = counts.pairs; row = 8; break;
        case MK_BUF_CONTACTS: src = b.contacts[last]; n = counts.contacts; row = 64; break;
        case MK_BUF_ACTIVE: src = b.active; n = counts.active; row = 4; break;
        case MK_BUF_COLLIDER_KEYS: src = b.keys; n = h->C; row = 8; break;
        case MK_BUF_CONTACT_FEATURES: src = b.features[last]; n = counts.contacts; row = 4; break;
        case MK_BUF_CONTACT_KEYS: src = b.contact_keys[last]; n = counts.contacts; row = 8; break;
        case MK_BUF_WORLD_MASSES: src = b.world_mass; n = h->B; row = 48; break;
        case MK_BUF_LINKS: src = h->mech.links_final; n = h->mech.links_final ? h->B : 0; row = 48; break;
        case MK_BUF_WARM_PREDICTIONS: src = b.warm_pred; n = b.warm_pred ? counts.active : 0; row = 4; break;
        case MK_BUF_WARM_FEATURES: src = b.warm_features; n = b.warm_features ? counts.active : 0; row = 64; break;
        case MK_BUF_CLOSURE_SLOTS: src = h->mech.slot_v; n = h->mech.slot_v ? h->mech_params.slots : 0; row = 32; break;
        case MK_BUF_CLOSURE_BLOCKS:   // computed for the 2 x 2 block preconditioners only
            src = h->mech.blk_feat;
            n = (h->mech.blk_feat && (h->mech_params.precond == MK_PRECOND_LEARNED ||
                                      h->mech_params.precond == MK_PRECOND_PAIR_BLOCKS))
                    ? h->mech_params.blocks : 0;
            row = 64;
            break;
        case MK_BUF_CLOSURE_BLOCK_OUTPUTS:
            src = h->mech.blk_hist;
            n = h->mech.blk_hist ? 12ull * h->mech_params.blocks : 0;
            row = 12;
            break;
        default:
            set_error(err, MK_ERR_INVALID_ARGUMENT, "unknown buffer id %u", id);
            return MK_ERR_INVALID_ARGUMENT;
    }
    if (count) *count = n;
    if (!host) return MK_OK;
    const uint64_t bytes = std::min<uint64_t>(n * row, cap_bytes);
    if (e == cudaSuccess && bytes && src) e = cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && id == MK_BUF_PAIRS) {
        // pair keys (a << shift | b) to GpuPair rows
        const uint32_t shift = h->params.pair_shift;
        uint64_t* k = reinterpret_cast<uint64_t*>(host);
        for (uint64_t r = 0; r < bytes / 8; ++r) {
            const uint64_t key = k[r];
            GpuPair pr{(uint32_t)(key >> shift), (uint32_t)(key & ((1ull << shift) - 1))};
            std::memcpy(&k[r], &pr, sizeof(pr));
        }
    }
    return check(e, err, "read_buffer") ? MK_OK : MK_ERR_DEVICE_FAILURE;
}

uint64_t mk_op_sort_scratch_bytes(uint32_t n) { return mk::sort_scratch_bytes(n, 63); }

int mk_op_sort_keys(const uint64_t* keys_in, const uint32_t* values_in, uint64_t* keys_out, uint32_t* values_out,
                    uint32_t n, uint32_t key_bits, void* scratch, uint64_t scratch_bytes, void* stream) {
    if (n == 0) return MK_OK;
    if (!keys_in || !values_in || !keys_out || !values_out || !scratch || key_bits == 0 || key_bits > 64) {
        set_error(nullptr, MK_ERR_INVALID_ARGUMENT, "sort: null pointer or key_bits outside 1..64");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (scratch_bytes < mk::sort_scratch_bytes(n, key_bits) || ((uintptr_t)scratch & 255u)) {
        set_error(nullptr, MK_ERR_INVALID_ARGUMENT, "sort: scratch too small or not 256-byte aligned");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (mk::sort_buffers_overlap(keys_in, values_in, keys_out, values_out, n)) {
        set_error(nullptr, MK_ERR_INVALID_ARGUMENT, "sort: input and output buffers overlap");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // The error word lives at the end of the caller's scratch (inside the size).
    uint32_t* flags = nullptr;
    cudaError_t e = mk::launch_sort(keys_in, values_in, keys_out, values_out, n, nullptr, key_bits, scratch,
                                    scratch_bytes, flags, (cudaStream_t)stream, sms);
    if (e != cudaSuccess) {
        set_error(nullptr, MK_ERR_DEVICE_FAILURE, "sort: %s", cudaGetErrorString(e));
        return MK_ERR_DEVICE_FAILURE;
    }
    return MK_OK;
}

int mk_op_obb_sat(const float* boxes_a, const float* boxes_b, uint32_t count, float* np, uint32_t* features,
                  void* stream) {
    if (count == 0) return MK_OK;
    if (!boxes_a || !boxes_b || !np || !features) return MK_ERR_INVALID_ARGUMENT;
    cudaError_t e = mk::launch_obb_sat(boxes_a, boxes_b, count, np, features, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        set_error(nullptr, MK_ERR_DEVICE_FAILURE, "obb_sat: %s", cudaGetErrorString(e));
        return MK_ERR_DEVICE_FAILURE;
    }
    return MK_OK;
}

}  // extern "C"
