// mk_device.cuh — device-side vector math, rows and shared primitives of the
// B200 rigid-body step.
//
// Every kernel that produces a parity-checked float is compiled with
// --fmad=false -prec-div=true -prec-sqrt=true -ftz=false: each source
// add/mul/div/sqrt is one IEEE-754 operation, so results are reproducible
// bit-for-bit and follow the operation order of the reference WGSL
// (crates/mechanic-gpu/src/kernels/*.wgsl), which evaluates vector
// expressions left to right.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mechanic_b200.h"

namespace mk {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr float kFloatMax = 3.402823e+38f;   // the literal the WGSL kernels use

// -------------------------------------------------------------- float3 ops
struct f3 { float x, y, z; };

__device__ __forceinline__ f3 mkf3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(const float4& a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ float4 f4(const f3& a, float w) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
// inverseSqrt is evaluated as an IEEE division of 1 by an IEEE sqrt.
__device__ __forceinline__ float rsqrt_ieee(float x) { return 1.0f / sqrtf(x); }
__device__ __forceinline__ f3 normalize(f3 a) { return a * rsqrt_ieee(dot(a, a)); }
__device__ __forceinline__ float4 normalize4(float4 a) {
    float s = rsqrt_ieee(dot4(a, a));
    return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
// min/max/clamp with a fixed operand choice on ties (signed zeros stay reproducible).
__device__ __forceinline__ float mxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float mnf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return mnf(mxf(x, lo), hi); }
__device__ __forceinline__ float sgnf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ __forceinline__ f3 absf3(f3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }

// Transcendentals: evaluated in double and rounded once to float, so the value
// is the correctly rounded one (bar double-rounding ties) on host and device.
__device__ __forceinline__ float sin_cr(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float cos_cr(float x) { return (float)cos((double)x); }
__device__ __forceinline__ float acos_cr(float x) { return (float)acos((double)x); }
__device__ __forceinline__ float atan2_cr(float y, float x) { return (float)atan2((double)y, (double)x); }

// Quaternion product / rotation (physics.wgsl:46-56; same helpers in every kernel file).
__device__ __forceinline__ float4 quat_multiply(float4 a, float4 b) {
    f3 av = xyz(a), bv = xyz(b);
    f3 v = a.w * bv + b.w * av + cross(av, bv);
    return make_float4(v.x, v.y, v.z, a.w * b.w - dot(av, bv));
}
__device__ __forceinline__ f3 quat_rotate(float4 q, f3 v) {
    f3 t = 2.0f * cross(xyz(q), v);
    return v + q.w * t + cross(xyz(q), t);
}
__device__ __forceinline__ float4 conjq(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }

__device__ __forceinline__ bool finite4(float4 v) {
    return v.x == v.x && v.y == v.y && v.z == v.z && v.w == v.w && fabsf(v.x) < kFloatMax &&
           fabsf(v.y) < kFloatMax && fabsf(v.z) < kFloatMax && fabsf(v.w) < kFloatMax;
}

// i32(round(x)) with WGSL round-half-to-even and a saturating conversion.
__device__ __forceinline__ int32_t fixed_i32(float x) {
    float r = rintf(x);
    if (r != r) return 0;
    if (r >= 2147483647.0f) return INT32_MAX;
    if (r <= -2147483648.0f) return INT32_MIN;
    return (int32_t)r;
}
__device__ __forceinline__ uint32_t round_u32(float x) {
    float r = rintf(x);
    if (!(r > 0.0f)) return 0u;
    if (r >= 4294967295.0f) return 0xffffffffu;
    return (uint32_t)r;
}

// An apply of zero deltas, f4(xyz(v) + 0.0f, 0.0f), reproduces v bit for bit
// unless a component is -0.0 (it becomes +0.0) or NaN (it may come back with
// another payload), or w is not +0.0: then the row must still be written.
__device__ __forceinline__ bool zero_apply_is_identity(float4 v) {
    const uint32_t nz = 0x80000000u;
    return __float_as_uint(v.x) != nz && __float_as_uint(v.y) != nz && __float_as_uint(v.z) != nz &&
           v.x == v.x && v.y == v.y && v.z == v.z && __float_as_uint(v.w) == 0u;
}

// ------------------------------------------------------------- loads/stores
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float4 ld4(const float4* p) { return *p; }

// Oriented box in world space as stored once per collider per tick:
// row0 = {center, half.x}, row1 = {axis_x, half.y}, row2 = {axis_y, half.z},
// row3 = {axis_z, bits(body)}.  64 bytes: one 4 x 128-bit load per box.
struct WorldBox { float4 r0, r1, r2, r3; };

__device__ __forceinline__ WorldBox load_box(const float4* boxes, uint32_t i) {
    const float4* p = boxes + 4ull * i;
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)};
}

// ------------------------------------------------------------ warp helpers
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if ((int)lane_id() >= o) v += n;
    }
    return v;
}

// Block-wide exclusive scan of one uint32 per thread (blockDim.x <= 1024,
// multiple of 32).  Returns the exclusive prefix; *total gets the block sum.
// `scratch` holds >= 33 words of shared memory.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scratch, uint32_t* total) {
    uint32_t inc = warp_inclusive_scan(v);
    uint32_t w = warp_id(), nw = blockDim.x >> 5;
    if (lane_id() == 31u) scratch[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane_id() < nw ? scratch[lane_id()] : 0u;
        uint32_t si = warp_inclusive_scan(s);
        if (lane_id() < nw) scratch[lane_id()] = si - s;
        if (lane_id() == 31u) scratch[32] = si;
    }
    __syncthreads();
    uint32_t r = scratch[w] + inc - v;
    *total = scratch[32];
    __syncthreads();
    return r;
}

// --------------------------------------------------- ordered tile look-back
// Decoupled look-back over tiles handed out in ticket order.  Each 64-bit
// word packs status (bits 62-63: 1 = aggregate, 2 = inclusive prefix) and a
// 62-bit count.  Waits are bounded: after kSpinLimit polls (a smaller limit
// only in the bounded-wait self-test) the tile gives up,
// raises MK_DEVICE_WAIT_TIMEOUT_FLAG and treats the missing predecessor as 0
// (results are then wrong but the GPU never hangs).
constexpr uint64_t kStatusAggregate = 1ull << 62;
constexpr uint64_t kStatusInclusive = 2ull << 62;
constexpr uint64_t kCountMask = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 20;

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
// Coherent GPU-scope stores / loads with no ordering (a word written and read
// for its own value only: no fence, unlike a release store).
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Fetch-add with acquire-release semantics at GPU scope: orders this thread's
// earlier writes before the add and makes writes released by earlier adds on
// the same word visible after it (the bottom-up refit's arrival counter).
__device__ __forceinline__ uint32_t atomic_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Called by warp 0 of a block (all 32 lanes).  Returns the exclusive prefix
// of `tile` and publishes its inclusive prefix.  The words are stored and read
// relaxed: each carries its own status and count, nothing else is published
// through them, and a release store's fence costs an L2 round trip per tile.
__device__ __forceinline__ uint64_t tile_lookback(uint64_t* states, uint32_t tile, uint64_t aggregate,
                                                  uint32_t* error_flags, uint32_t spin_limit = kSpinLimit) {
    const uint32_t lane = lane_id();
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(states, kStatusInclusive | aggregate);
        return 0;
    }
    if (lane == 0) st_relaxed_u64(states + tile, kStatusAggregate | aggregate);
    uint64_t exclusive = 0;
    int64_t base = (int64_t)tile - 1;
    uint32_t spins = 0;
    bool timed_out = false;
    while (base >= 0) {
        int64_t idx = base - (int64_t)lane;
        uint64_t v = idx >= 0 ? ld_relaxed_u64(states + idx) : kStatusInclusive;
        uint32_t ready = __ballot_sync(0xffffffffu, (v >> 62) != 0);
        if (ready != 0xffffffffu) {
            if (++spins > spin_limit) { timed_out = true; v = (v >> 62) ? v : kStatusInclusive; }
            else continue;
        }
        uint32_t inclusive = __ballot_sync(0xffffffffu, (v >> 62) == 2);
        uint32_t stop = inclusive ? (__ffs(inclusive) - 1) : 32u;   // first lane (nearest tile) with a prefix
        uint64_t contrib = lane <= stop ? (v & kCountMask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, o);
        exclusive += __shfl_sync(0xffffffffu, contrib, 0);
        if (inclusive) break;
        base -= 32;
        spins = 0;
    }
    if (timed_out && lane == 0) atomicOr(error_flags, MK_DEVICE_WAIT_TIMEOUT_FLAG);
    if (lane == 0) st_relaxed_u64(states + tile, kStatusInclusive | (exclusive + aggregate));
    return exclusive;
}

// Grid-wide barrier for a cooperative launch on one 32-bit word that starts at
// zero: block 0 adds 2^31 - (participants - 1), every other block adds 1, so
// the word's top bit flips exactly when the last block arrives and its low
// bits return to zero for the next barrier (one atomic per block, no reset
// step).  The wait is bounded: a block that gives up raises
// MK_DEVICE_WAIT_TIMEOUT_FLAG and carries on.
__device__ __forceinline__ void grid_barrier(uint32_t* state, uint32_t* error_flags, uint32_t participants,
                                             uint32_t spin_limit = kSpinLimit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t add = blockIdx.x == 0 ? 0x80000000u - (participants - 1u) : 1u;
        __threadfence();
        const uint32_t old = atomicAdd(state, add);
        uint32_t spins = 0;
        while (((ld_acquire_u32(state) ^ old) & 0x80000000u) == 0u) {
            if (++spins > spin_limit) {
                atomicOr(error_flags, MK_DEVICE_WAIT_TIMEOUT_FLAG);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
}

}  // namespace mk
