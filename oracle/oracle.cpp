// oracle.cpp — CPU restatement of Mechanic's rigid-body step.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never linked
// into it.  Each function names the reference file:line it restates (paths
// are relative to the jens-hj/mechanic project).  Operation order follows the
// WGSL source left to right; the FP32 build uses -ffp-contract=off so that
// every add/mul/div/sqrt is one IEEE-754 operation, exactly as the CUDA
// kernels compiled with --fmad=false.  Parity is unpinned against the
// reference's own kernels (none can run here); see oracle.h.

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <limits>
#include <map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const uint32_t INVALID = 0xffffffffu;
static int g_threads = 0;

// ---------------------------------------------------------------- math ----
template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

template <class T> static inline V3<T> v3(T x, T y, T z) { return {x, y, z}; }
template <class T> static inline V3<T> xyz(const V4<T>& a) { return {a.x, a.y, a.z}; }
template <class T> static inline V4<T> v4(const V3<T>& a, T w) { return {a.x, a.y, a.z, w}; }
template <class T> static inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> static inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> static inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> static inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> static inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> static inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> static inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> static inline T dot4(V4<T> a, V4<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <class T> static inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> static inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
// normalize(v) = v * inverseSqrt(dot(v, v)); inverseSqrt taken as 1 / sqrt.
template <class T> static inline V3<T> normalize(V3<T> a) { return a * (T(1) / std::sqrt(dot(a, a))); }
template <class T> static inline V4<T> normalize4(V4<T> a) {
    T s = T(1) / std::sqrt(dot4(a, a));
    return {a.x * s, a.y * s, a.z * s, a.w * s};
}
// WGSL min/max/clamp with a fixed answer for equal operands.
template <class T> static inline T mx(T a, T b) { return a > b ? a : b; }
template <class T> static inline T mn(T a, T b) { return a < b ? a : b; }
template <class T> static inline T clampv(T x, T lo, T hi) { return mn(mx(x, lo), hi); }
template <class T> static inline T sgn(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0)); }
template <class T> static inline V3<T> absv(V3<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }

// Transcendentals evaluated in double and rounded once, so the FP32 result
// is the correctly rounded value on both the CPU and the GPU.
template <class T> static inline T tsin(T x) { return T(std::sin(double(x))); }
template <class T> static inline T tcos(T x) { return T(std::cos(double(x))); }
template <class T> static inline T tacos(T x) { return T(std::acos(double(x))); }
template <class T> static inline T tatan2(T y, T x) { return T(std::atan2(double(y), double(x))); }
template <class T> static inline T tlog(T x) { return T(std::log(double(x))); }

// physics.wgsl:46-56, collision.wgsl:97-107 (identical in every kernel file).
template <class T> static inline V4<T> quat_multiply(V4<T> a, V4<T> b) {
    V3<T> av = xyz(a), bv = xyz(b);
    V3<T> v = a.w * bv + b.w * av + cross(av, bv);
    return {v.x, v.y, v.z, a.w * b.w - dot(av, bv)};
}
template <class T> static inline V3<T> quat_rotate(V4<T> q, V3<T> v) {
    V3<T> t = T(2) * cross(xyz(q), v);
    return v + q.w * t + cross(xyz(q), t);
}
template <class T> static inline V4<T> conj(V4<T> q) { return {-q.x, -q.y, -q.z, q.w}; }

template <class T> static inline bool finite4(V4<T> v) {
    const T lim = T(3.402823e+38f);
    return v.x == v.x && v.y == v.y && v.z == v.z && v.w == v.w &&
           std::fabs(v.x) < lim && std::fabs(v.y) < lim && std::fabs(v.z) < lim && std::fabs(v.w) < lim;
}

// i32(round(x)): WGSL round is half-to-even; the conversion saturates and
// sends NaN to 0 (as the GPU's cvt.rni.s32.f32 does).
template <class T> static inline int32_t fixed_i32(T x) {
    T r = std::nearbyint(x);
    if (r != r) return 0;
    if (r >= T(2147483647.0)) return INT32_MAX;
    if (r <= T(-2147483648.0)) return INT32_MIN;
    return (int32_t)r;
}
// i64(round(x)) for the 2^32 fixed point of the residual-mode solve: half to
// even, saturating, NaN to 0 (cvt.rni.s64.f32).
template <class T> static inline int64_t fixed_i64(T x) {
    T r = std::nearbyint(x);
    if (r != r) return 0;
    if (r >= T(9223372036854775807.0)) return INT64_MAX;
    if (r <= T(-9223372036854775808.0)) return INT64_MIN;
    return (int64_t)r;
}
template <class T> static inline uint32_t round_u32(T x) {
    T r = std::nearbyint(x);
    if (!(r > T(0))) return 0;
    if (r >= T(4294967295.0)) return 0xffffffffu;
    return (uint32_t)r;
}

template <class T> static inline V4<T> load4(const float* p) { return {T(p[0]), T(p[1]), T(p[2]), T(p[3])}; }

// ------------------------------------------------------------- world -----
template <class T> struct Collider { V4<T> center, rot, half; uint32_t meta[4]; };
template <class T> struct Mass { T inv_mass; V3<T> ix, iy, iz; };
template <class T> struct WorldMass { V4<T> x, y, z; };  // x.w = inverse mass
template <class T> struct Contact {
    uint32_t meta[4];
    V4<T> np;   // normal, penetration
    V4<T> aa;   // arm a, impulse
    V4<T> ab;   // arm b, near-face axes / -1
};
template <class T> struct Manifold { uint32_t tick, count; V4<T> np; V4<T> pi; };
template <class T> struct Bearing { V4<T> aa, ab, xa, xb; uint32_t meta[4]; };
template <class T> struct MechBody { uint32_t meta[4]; uint32_t trav[4]; V4<T> bpos, brot; };
template <class T> struct Link { V4<T> pos, rot; uint32_t meta[4]; };
struct Drive { uint32_t mode; float max_acc, max_speed, target_speed, target_angle, min_angle, max_angle; };

struct SatResult32 { uint32_t axis; };

template <class T> struct Sat { V3<T> normal; T pen; uint32_t near; uint32_t axis; uint32_t early; };

template <class T> struct Obb { V3<T> c; V3<T> ax[3]; V3<T> h; };

struct WorldBase {
    virtual ~WorldBase() {}
    virtual int step(uint64_t tick) = 0;
    int precision = 32;
};

template <class T> struct World : WorldBase {
    // configuration
    uint32_t B = 0, C = 0, J = 0, S = 0, Q = 0, max_depth = 0, closure_count = 0;
    T dt, gravity, lin_damp, ang_damp;
    uint32_t iterations = 8, morton_mode = 0, collisions = 1, self_collisions = 1, pair_capacity = 0;
    uint32_t has_dynamic_root = 0;
    // rows
    std::vector<V4<T>> pos, rot, lin, ang;
    std::vector<T> inv_mass;
    std::vector<Mass<T>> mass;
    std::vector<Collider<T>> col;
    std::vector<uint32_t> sup;  // 2*S
    std::vector<uint32_t> root;
    std::vector<uint32_t> components;
    std::vector<Bearing<T>> bear;
    std::vector<MechBody<T>> mech;
    std::vector<uint32_t> preorder;
    std::vector<Drive> drives;
    std::vector<V4<T>> coords;  // x angle, y angular velocity
    // per tick
    std::vector<WorldMass<T>> wm;
    std::vector<uint32_t> deltas;  // 6 per body, i32 bit patterns with wrap-around
    std::vector<V4<T>> aabb_min, aabb_max;
    std::vector<uint64_t> keys, skeys;
    std::vector<uint32_t> svals;
    std::vector<uint32_t> pairs;    // 2 per pair
    std::vector<Contact<T>> contacts;
    std::vector<uint64_t> contact_keys;
    std::vector<uint32_t> features;
    std::vector<uint32_t> active;
    std::unordered_map<uint64_t, Manifold<T>> manifold;
    // MK_MANIFOLD_CLIPPED: up to four contacts per collider pair; the previous
    // tick's acquired rows of each pair in row order
    uint32_t clipped = 0;
    std::unordered_map<uint64_t, std::vector<Manifold<T>>> manifold_rows;
    std::vector<V4<T>> snap_pos[3], snap_rot[3];
    GpuDiagnostics diag{};
    uint32_t tick32 = 0;

    // ---------------------------------------------------------- helpers
    V3<T> collider_center(uint32_t i) const {
        const Collider<T>& c = col[i];
        uint32_t b = c.meta[0];
        return xyz(pos[b]) + quat_rotate(rot[b], xyz(c.center));
    }
    V4<T> collider_rotation(uint32_t i) const { return quat_multiply(rot[col[i].meta[0]], col[i].rot); }
    Obb<T> obb(uint32_t i) const {
        Obb<T> o;
        V4<T> r = collider_rotation(i);
        o.c = collider_center(i);
        o.ax[0] = quat_rotate(r, v3<T>(1, 0, 0));
        o.ax[1] = quat_rotate(r, v3<T>(0, 1, 0));
        o.ax[2] = quat_rotate(r, v3<T>(0, 0, 1));
        o.h = xyz(col[i].half);
        return o;
    }

    bool pair_is_suppressed(uint32_t a, uint32_t b) const {  // lbvh.wgsl:325-345
        uint32_t low = std::min(a, b), high = std::max(a, b);
        uint32_t left = 0, right = S;
        while (left < right) {
            uint32_t mid = left + (right - left) / 2;
            uint32_t cx = sup[2 * mid], cy = sup[2 * mid + 1];
            if (cx < low || (cx == low && cy < high)) left = mid + 1; else right = mid;
        }
        return left < S && sup[2 * left] == low && sup[2 * left + 1] == high;
    }

    // ------------------------------------------------- physics.wgsl:92-132
    void integrate() {
        const T gdt = gravity * dt;
        const T half_dt = T(0.5) * dt;
        std::atomic<uint32_t> flag{0};
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)B; ++ii) {
            uint32_t i = (uint32_t)ii;
            V4<T> p = pos[i], q = rot[i], l = lin[i], a = ang[i];
            if (inv_mass[i] > T(0)) {
                l.y += gdt;
                V3<T> lv = xyz(l) * lin_damp; l = v4(lv, l.w);
                V3<T> av = xyz(a) * ang_damp; a = v4(av, a.w);
                if (root[i] != 0) {
                    V3<T> pv = xyz(p) + xyz(l) * dt; p = v4(pv, p.w);
                    V4<T> spin = v4(xyz(a), T(0));
                    V4<T> d = quat_multiply(spin, q);
                    q = {q.x + d.x * half_dt, q.y + d.y * half_dt, q.z + d.z * half_dt, q.w + d.w * half_dt};
                    T ns = dot4(q, q);
                    if (ns > T(1.0e-20f)) {
                        T s = T(1) / std::sqrt(ns);
                        q = {q.x * s, q.y * s, q.z * s, q.w * s};
                    } else {
                        q = {0, 0, 0, 1};
                        flag |= MK_INVALID_NUMERIC_FLAG;
                    }
                }
            }
            if (!(finite4(p) && finite4(q) && finite4(l) && finite4(a))) {
                flag |= MK_INVALID_NUMERIC_FLAG;
                continue;
            }
            pos[i] = p; rot[i] = q; lin[i] = l; ang[i] = a;
        }
        diag.error_flags |= flag.load();
    }

    // --------------------------------------------- collision.wgsl:134-162
    V3<T> world_inverse_inertia_column(uint32_t b, V3<T> axis) const {
        V4<T> r = rot[b];
        V3<T> local = quat_rotate(conj(r), axis);
        const Mass<T>& m = mass[b];
        V3<T> lr = m.ix * local.x + m.iy * local.y + m.iz * local.z;
        return quat_rotate(r, lr);
    }
    void update_world_masses() {
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)B; ++ii) {
            uint32_t b = (uint32_t)ii;
            wm[b].x = v4(world_inverse_inertia_column(b, v3<T>(1, 0, 0)), mass[b].inv_mass);
            wm[b].y = v4(world_inverse_inertia_column(b, v3<T>(0, 1, 0)), T(0));
            wm[b].z = v4(world_inverse_inertia_column(b, v3<T>(0, 0, 1)), T(0));
        }
    }

    // ------------------------------------------------ lbvh.wgsl:84-130
    static uint32_t expand10(uint32_t v) {
        v &= 0x3ffu;
        v = (v | (v << 16)) & 0x030000ffu;
        v = (v | (v << 8)) & 0x0300f00fu;
        v = (v | (v << 4)) & 0x030c30c3u;
        v = (v | (v << 2)) & 0x09249249u;
        return v;
    }
    static uint64_t expand21(uint64_t v) {
        v &= 0x1fffffull;
        v = (v | (v << 32)) & 0x1f00000000ffffull;
        v = (v | (v << 16)) & 0x1f0000ff0000ffull;
        v = (v | (v << 8)) & 0x100f00f00f00f00full;
        v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
        v = (v | (v << 2)) & 0x1249249249249249ull;
        return v;
    }
    static uint32_t morton30(V3<T> c) {
        auto q = [](T x) -> uint32_t {
            T f = clampv(std::floor(x + T(512)), T(0), T(1023));
            return (uint32_t)f;
        };
        return expand10(q(c.x)) | (expand10(q(c.y)) << 1) | (expand10(q(c.z)) << 2);
    }
    // qmax + 1 cells per axis (2^21: 63-bit keys, 2^16: 48-bit keys) over the
    // tick's bounds of the collider centres, one scale from the largest extent
    // (cubic cells).
    static uint64_t morton_frame(V3<T> c, V3<T> lo, T scale, T qmax) {
        auto q = [&](T x, T l) -> uint64_t {
            T f = clampv(std::floor((x - l) * scale), T(0), qmax);
            return (uint64_t)f;
        };
        return expand21(q(c.x, lo.x)) | (expand21(q(c.y, lo.y)) << 1) | (expand21(q(c.z, lo.z)) << 2);
    }
    static T frame_qmax(uint32_t mode) {
        return mode == MK_MORTON_30_ADAPTIVE ? T(1023.0f)
               : mode == MK_MORTON_39      ? T(8191.0f)
               : mode == MK_MORTON_48      ? T(65535.0f)
                                           : T(2097151.0f);
    }
    static uint32_t spatial_key_bits(uint32_t mode) {
        return mode == MK_MORTON_REFERENCE_30 || mode == MK_MORTON_30_ADAPTIVE ? 30u
               : mode == MK_MORTON_39                                        ? 39u
               : mode == MK_MORTON_48                                        ? 48u
                                                                             : 63u;
    }
    // batched scenes: the scene index above the spatial key, whose lowest bits
    // give way when both do not fit in 63 bits
    static uint64_t compose_key(uint32_t mode, uint32_t sb, uint64_t scene, uint64_t key) {
        if (!sb) return key;
        const uint32_t w = spatial_key_bits(mode);
        if (w + sb <= 63u) return (scene << w) | key;
        return (scene << (63u - sb)) | (key >> (w + sb - 63u));
    }
    // floats as unsigned integers in the same order (-0 below +0)
    static uint32_t float_order(float f) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }
    static float float_unorder(uint32_t v) {
        const uint32_t u = (v & 0x80000000u) ? (v & 0x7fffffffu) : ~v;
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }
    void key_frame(const std::vector<V3<T>>& centers, T qmax, V3<T>& lo, T& scale) const {
        uint32_t w[6] = {0, 0, 0, 0, 0, 0};
        for (const V3<T>& c : centers) {
            const float cc[3] = {float(c.x), float(c.y), float(c.z)};
            if (!(std::isfinite(cc[0]) && std::isfinite(cc[1]) && std::isfinite(cc[2]))) continue;
            for (int a = 0; a < 3; ++a) {
                const uint32_t o = float_order(cc[a]);
                w[a] = std::max(w[a], o);
                w[3 + a] = std::max(w[3 + a], ~o);
            }
        }
        lo = v3<T>(T(float_unorder(~w[3])), T(float_unorder(~w[4])), T(float_unorder(~w[5])));
        const V3<T> hi = v3<T>(T(float_unorder(w[0])), T(float_unorder(w[1])), T(float_unorder(w[2])));
        const T extent = mx(mx(hi.x - lo.x, hi.y - lo.y), hi.z - lo.z);
        scale = extent > T(0) ? qmax / extent : T(1);
    }
    void compute_bounds() {
        std::vector<V3<T>> centers(C);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)C; ++ii) centers[ii] = collider_center((uint32_t)ii);
        V3<T> lo = v3<T>(0, 0, 0);
        T scale = T(1);
        const T qmax = frame_qmax(morton_mode);
        if (morton_mode != MK_MORTON_REFERENCE_30) key_frame(centers, qmax, lo, scale);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)C; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<T> c = centers[i];
            V4<T> r = collider_rotation(i);
            V3<T> ax = quat_rotate(r, v3<T>(1, 0, 0));
            V3<T> ay = quat_rotate(r, v3<T>(0, 1, 0));
            V3<T> az = quat_rotate(r, v3<T>(0, 0, 1));
            const V4<T>& h = col[i].half;
            V3<T> e = absv(ax) * h.x + absv(ay) * h.y + absv(az) * h.z;
            aabb_min[i] = v4(c - e, T(0));
            aabb_max[i] = v4(c + e, T(0));
            const uint64_t key = morton_mode == MK_MORTON_REFERENCE_30 ? (uint64_t)morton30(c)
                                                                       : morton_frame(c, lo, scale, qmax);
            keys[i] = compose_key(morton_mode, scene_bits, scene_bits ? col_scene[i] : 0u, key);
        }
        // Stable sort by key == ascending (key, index) order.
        std::vector<uint32_t> perm(C);
        for (uint32_t i = 0; i < C; ++i) perm[i] = i;
        std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
        for (uint32_t i = 0; i < C; ++i) { skeys[i] = keys[perm[i]]; svals[i] = perm[i]; }
    }

    static bool overlaps(const V4<T>& amin, const V4<T>& amax, const V4<T>& bmin, const V4<T>& bmax) {
        return amin.x <= bmax.x && amin.y <= bmax.y && amin.z <= bmax.z &&
               bmin.x <= amax.x && bmin.y <= amax.y && bmin.z <= amax.z;
    }

    // Pair set of lbvh.wgsl:321-398: every collider pair (i < j) of different,
    // non-suppressed bodies whose closed AABBs overlap.  Found here with a
    // uniform grid (an independent method) and emitted in canonical order.
    void broadphase() {
        pairs.clear();
        if (C < 2) return;
        if (C <= 2048) {
            for (uint32_t i = 0; i < C; ++i)
                for (uint32_t j = i + 1; j < C; ++j) consider_pair(i, j, pairs);
        } else {
            grid_pairs();
        }
        uint64_t count = pairs.size() / 2;
        if (count > pair_capacity) {
            diag.error_flags |= MK_PAIR_OVERFLOW_FLAG;
            pairs.resize(2ull * pair_capacity);
        }
        diag.pair_count = (uint32_t)std::min<uint64_t>(count, 0xffffffffull);
    }
    std::vector<uint32_t> col_scene;   // batched scenes: scene of each collider
    uint32_t scene_bits = 0;
    void consider_pair(uint32_t i, uint32_t j, std::vector<uint32_t>& out) const {
        uint32_t a = col[i].meta[0], b = col[j].meta[0];
        if (a == b) return;
        if (scene_bits && col_scene[i] != col_scene[j]) return;
        if (!overlaps(aabb_min[i], aabb_max[i], aabb_min[j], aabb_max[j])) return;
        if (pair_is_suppressed(a, b)) return;
        out.push_back(i);
        out.push_back(j);
    }
    void grid_pairs() {
        // Cell size: twice the median AABB extent, at least 0.05 m.
        std::vector<T> ext(C);
        for (uint32_t i = 0; i < C; ++i)
            ext[i] = mx(mx(aabb_max[i].x - aabb_min[i].x, aabb_max[i].y - aabb_min[i].y), aabb_max[i].z - aabb_min[i].z);
        std::nth_element(ext.begin(), ext.begin() + C / 2, ext.end());
        double cell = std::max(0.05, 2.0 * double(ext[C / 2]));
        double lo[3] = {1e300, 1e300, 1e300};
        for (uint32_t i = 0; i < C; ++i) {
            lo[0] = std::min(lo[0], double(aabb_min[i].x));
            lo[1] = std::min(lo[1], double(aabb_min[i].y));
            lo[2] = std::min(lo[2], double(aabb_min[i].z));
        }
        auto cidx = [&](double v, int d) -> int64_t { return (int64_t)std::floor((v - lo[d]) / cell); };
        // cell key -> colliders; a pair is reported only in the cell holding
        // the max of the two AABB minima, so each pair appears once.
        std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
        grid.reserve(C * 2);
        auto key3 = [](int64_t x, int64_t y, int64_t z) -> uint64_t {
            return ((uint64_t)(x & 0x1fffff) << 42) | ((uint64_t)(y & 0x1fffff) << 21) | (uint64_t)(z & 0x1fffff);
        };
        for (uint32_t i = 0; i < C; ++i) {
            const int64_t zs = scene_bits ? (int64_t)col_scene[i] * 4096 : 0;   // one grid per scene
            int64_t x0 = cidx(aabb_min[i].x, 0), x1 = cidx(aabb_max[i].x, 0);
            int64_t y0 = cidx(aabb_min[i].y, 1), y1 = cidx(aabb_max[i].y, 1);
            int64_t z0 = cidx(aabb_min[i].z, 2), z1 = cidx(aabb_max[i].z, 2);
            for (int64_t x = x0; x <= x1; ++x)
                for (int64_t y = y0; y <= y1; ++y)
                    for (int64_t z = z0; z <= z1; ++z) grid[key3(x, y, z + zs)].push_back(i);
        }
        std::vector<const std::vector<uint32_t>*> cells;
        std::vector<uint64_t> cell_keys;
        cells.reserve(grid.size());
        for (auto& kv : grid) { cells.push_back(&kv.second); cell_keys.push_back(kv.first); }
        int nt = 1;
#ifdef _OPENMP
        nt = omp_get_max_threads();
#endif
        std::vector<std::vector<uint32_t>> local(nt);
#pragma omp parallel
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            std::vector<uint32_t>& out = local[t];
#pragma omp for schedule(dynamic, 64)
            for (int64_t ci = 0; ci < (int64_t)cells.size(); ++ci) {
                const std::vector<uint32_t>& v = *cells[ci];
                uint64_t k = cell_keys[ci];
                for (size_t a = 0; a < v.size(); ++a)
                    for (size_t b = a + 1; b < v.size(); ++b) {
                        uint32_t i = v[a], j = v[b];
                        // owning cell = cell of the componentwise max of minima
                        double mxv[3] = {std::max(double(aabb_min[i].x), double(aabb_min[j].x)),
                                         std::max(double(aabb_min[i].y), double(aabb_min[j].y)),
                                         std::max(double(aabb_min[i].z), double(aabb_min[j].z))};
                        const int64_t zs = scene_bits ? (int64_t)col_scene[i] * 4096 : 0;
                        if (key3(cidx(mxv[0], 0), cidx(mxv[1], 1), cidx(mxv[2], 2) + zs) != k) continue;
                        uint32_t lo_i = std::min(i, j), hi_i = std::max(i, j);
                        consider_pair(lo_i, hi_i, out);
                    }
            }
        }
        std::vector<uint64_t> all;
        for (auto& l : local)
            for (size_t p = 0; p < l.size(); p += 2) all.push_back(((uint64_t)l[p] << 32) | l[p + 1]);
        std::sort(all.begin(), all.end());
        pairs.resize(all.size() * 2);
        for (size_t p = 0; p < all.size(); ++p) {
            pairs[2 * p] = (uint32_t)(all[p] >> 32);
            pairs[2 * p + 1] = (uint32_t)all[p];
        }
    }

    // ----------------------------------------- collision.wgsl:175-287
    V3<T> support_point(const Obb<T>& o, V3<T> dir) const {
        V3<T> p = o.c;
        const T he[3] = {o.h.x, o.h.y, o.h.z};
        for (int a = 0; a < 3; ++a) {
            T proj = dot(o.ax[a], dir);
            if (std::fabs(proj) > T(1.0e-5f)) p = p + o.ax[a] * he[a] * sgn(proj);
        }
        return p;
    }
    static V3<T> vertex(const Obb<T>& o, uint32_t v) {
        V3<T> p = o.c;
        const T he[3] = {o.h.x, o.h.y, o.h.z};
        for (uint32_t a = 0; a < 3; ++a) {
            T d = (v & (1u << a)) ? T(1) : T(-1);
            p = p + o.ax[a] * he[a] * d;
        }
        return p;
    }
    static bool contains(const Obb<T>& o, V4<T> r, V3<T> p) {
        V3<T> local = quat_rotate(conj(r), p - o.c);
        return std::fabs(local.x) <= o.h.x + T(1.0e-5f) && std::fabs(local.y) <= o.h.y + T(1.0e-5f) &&
               std::fabs(local.z) <= o.h.z + T(1.0e-5f);
    }
    // contains() in collision.wgsl:256-264 rotates by the conjugate collider
    // rotation; boxes given only by axes use the transposed basis instead.
    static bool contains_axes(const Obb<T>& o, V3<T> p) {
        V3<T> d = p - o.c;
        V3<T> local = v3<T>(dot(o.ax[0], d), dot(o.ax[1], d), dot(o.ax[2], d));
        return std::fabs(local.x) <= o.h.x + T(1.0e-5f) && std::fabs(local.y) <= o.h.y + T(1.0e-5f) &&
               std::fabs(local.z) <= o.h.z + T(1.0e-5f);
    }
    V3<T> contact_point(const Obb<T>& a, V4<T> ra, const Obb<T>& b, V4<T> rb, V3<T> n, bool by_axes) const {
        V3<T> sum = v3<T>(0, 0, 0);
        T count = T(0);
        for (uint32_t v = 0; v < 8; ++v) {
            V3<T> pa = vertex(a, v);
            if (by_axes ? contains_axes(b, pa) : contains(b, rb, pa)) { sum = sum + pa; count += T(1); }
            V3<T> pb = vertex(b, v);
            if (by_axes ? contains_axes(a, pb) : contains(a, ra, pb)) { sum = sum + pb; count += T(1); }
        }
        if (count > T(0)) return sum / count;
        V3<T> pa = support_point(a, n), pb = support_point(b, -n);
        return (pa + pb) * T(0.5);
    }

    // ----------------------------------------- collision.wgsl:393-486
    static T projection_radius(const V3<T>* ax, V3<T> e, V3<T> axis) {
        return std::fabs(dot(ax[0], axis)) * e.x + std::fabs(dot(ax[1], axis)) * e.y + std::fabs(dot(ax[2], axis)) * e.z;
    }
    static Sat<T> test_axis(V3<T> delta, const Obb<T>& a, const Obb<T>& b, V3<T> raw, uint32_t idx) {
        T l2 = dot(raw, raw);
        if (l2 < T(1.0e-10f)) return {v3<T>(1, 0, 0), T(3.402823e+38f), 0, idx, 0};
        V3<T> axis = raw * (T(1) / std::sqrt(l2));
        T sd = dot(delta, axis);
        T pen = projection_radius(a.ax, a.h, axis) + projection_radius(b.ax, b.h, axis) - std::fabs(sd);
        if (sd < T(0)) axis = -axis;
        return {axis, pen, 0, idx, 0};
    }
    static Sat<T> obb_sat(const Obb<T>& a, const Obb<T>& b) {
        V3<T> delta = b.c - a.c;
        Sat<T> mn_r = {v3<T>(1, 0, 0), T(3.402823e+38f), 0, 0, 0};
        uint32_t near = 0;
        for (uint32_t i = 0; i < 3; ++i) {
            Sat<T> ra = test_axis(delta, a, b, a.ax[i], 2 * i);
            if (ra.pen < T(0)) { ra.early = 1; return ra; }
            if (ra.pen <= T(1.0e-4f)) near += 1;
            if (ra.pen < mn_r.pen) mn_r = ra;
            Sat<T> rb = test_axis(delta, a, b, b.ax[i], 2 * i + 1);
            if (rb.pen < T(0)) { rb.early = 1; return rb; }
            if (rb.pen <= T(1.0e-4f)) near += 1;
            if (rb.pen < mn_r.pen) mn_r = rb;
        }
        for (uint32_t i = 0; i < 3; ++i)
            for (uint32_t j = 0; j < 3; ++j) {
                Sat<T> r = test_axis(delta, a, b, cross(a.ax[i], b.ax[j]), 6 + 3 * i + j);
                if (r.pen < T(0)) { r.early = 1; return r; }
                if (r.pen < mn_r.pen) mn_r = r;
            }
        mn_r.near = near;
        return mn_r;
    }

    // ----------------------------------------- collision.wgsl:570-603
    void narrowphase() {
        uint64_t np = pairs.size() / 2;
        std::vector<Contact<T>> out4(4 * np);
        std::vector<uint32_t> feat(np);
        std::vector<uint8_t> emit(np);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t pp = 0; pp < (int64_t)np; ++pp) {
            uint32_t ia = pairs[2 * pp], ib = pairs[2 * pp + 1];
            emit[pp] = 0;
            if (!self_collisions && components[col[ia].meta[0]] == components[col[ib].meta[0]]) continue;
            Obb<T> a = obb(ia), b = obb(ib);
            Sat<T> s = obb_sat(a, b);
            emit[pp] = 0;
            if (s.pen < T(-1.0e-5f)) continue;
            V3<T> pts[4];
            uint32_t cnt = 1;
            if (clipped) cnt = manifold_points(a, collider_rotation(ia), b, collider_rotation(ib), s.normal, pts);
            else pts[0] = contact_point(a, collider_rotation(ia), b, collider_rotation(ib), s.normal, false);
            uint32_t ba = col[ia].meta[0], bb = col[ib].meta[0];
            for (uint32_t q = 0; q < cnt; ++q) {
                Contact<T>& c = out4[4 * pp + q];
                c.meta[0] = ba; c.meta[1] = bb; c.meta[2] = ia; c.meta[3] = ib;
                c.np = v4(s.normal, mx(s.pen, T(0)));
                c.aa = v4(pts[q] - xyz(pos[ba]), T(0));
                c.ab = v4(pts[q] - xyz(pos[bb]), T(s.near));
            }
            feat[pp] = s.axis | (s.near << 8) | (s.early << 16);
            emit[pp] = (uint8_t)cnt;
        }
        contacts.clear(); contact_keys.clear(); features.clear();
        for (uint64_t pp = 0; pp < np; ++pp)
            for (uint32_t q = 0; q < emit[pp]; ++q) {
                contacts.push_back(out4[4 * pp + q]);
                contact_keys.push_back(((uint64_t)pairs[2 * pp] << 32) | pairs[2 * pp + 1]);
                features.push_back(feat[pp]);
            }
    }
    // collision.rs:68-103 on the GPU boxes (vertex order and containment of contact_point)
    uint32_t manifold_points(const Obb<T>& a, V4<T> ra, const Obb<T>& b, V4<T> rb, V3<T> n, V3<T>* out) const {
        V3<T> cand[16];
        uint32_t c = 0;
        for (uint32_t side = 0; side < 2; ++side) {
            const Obb<T>& src = side == 0 ? a : b;
            const Obb<T>& dst = side == 0 ? b : a;
            const V4<T> rdst = side == 0 ? rb : ra;
            for (uint32_t v = 0; v < 8; ++v) {
                V3<T> pt = vertex(src, v);
                if (!contains(dst, rdst, pt)) continue;
                bool dup = false;
                for (uint32_t q = 0; q < c; ++q) {
                    V3<T> d = cand[q] - pt;
                    if (!(dot(d, d) > T(1.0e-10f))) { dup = true; break; }
                }
                if (!dup) cand[c++] = pt;
            }
        }
        if (c == 0) {
            out[0] = (support_point(a, n) + support_point(b, -n)) * T(0.5);
            return 1;
        }
        for (uint32_t i = 1; i < c; ++i) {
            V3<T> key = cand[i];
            uint32_t j = i;
            while (j > 0) {
                V3<T> prv = cand[j - 1];
                bool greater = prv.x != key.x ? prv.x > key.x : (prv.y != key.y ? prv.y > key.y : prv.z > key.z);
                if (!greater) break;
                cand[j] = prv;
                --j;
            }
            cand[j] = key;
        }
        const uint32_t m = c < 4 ? c : 4;
        for (uint32_t i = 0; i < m; ++i) out[i] = cand[i];
        return m;
    }

    // ----------------------------------------- collision.wgsl:193-238, 622-664
    void ground_contacts() {
        std::vector<Contact<T>> out(C);
        std::vector<uint8_t> emit(C);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)C; ++ii) {
            uint32_t i = (uint32_t)ii;
            emit[i] = 0;
            const Collider<T>& c = col[i];
            Obb<T> o = obb(i);
            V3<T> down = v3<T>(0, -1, 0);
            V3<T> sp = support_point(o, down);
            uint32_t role = c.meta[3];
            if (role != 0) {
                V3<T> caxis = o.ax[1];
                T ap = dot(caxis, down);
                V3<T> radial = down - caxis * ap;
                T rl = length(radial);
                uint32_t cc = rl < T(0.05f) ? 4u : 1u;
                if (role > cc) continue;
                V3<T> p = o.c - o.ax[0] * c.center.w;
                if (rl < T(0.05f)) {
                    p = p + caxis * sgn(ap) * c.half.y;
                    V3<T> ta = normalize(v3<T>(1, 0, 0) - caxis * caxis.x);
                    V3<T> tb = normalize(cross(caxis, ta));
                    if (role == 1) p = p + ta * c.half.w;
                    else if (role == 2) p = p - ta * c.half.w;
                    else if (role == 3) p = p + tb * c.half.w;
                    else p = p - tb * c.half.w;
                } else {
                    p = p + radial * (c.half.w / rl);
                    if (std::fabs(ap) >= T(0.05f)) p = p + caxis * sgn(ap) * c.half.y;
                }
                sp = p;
            }
            T bottom = sp.y;
            if (bottom > T(1.0e-5f)) continue;
            uint32_t b = c.meta[0];
            Contact<T>& k = out[i];
            k.meta[0] = b; k.meta[1] = INVALID; k.meta[2] = i; k.meta[3] = INVALID;
            k.np = {T(0), T(-1), T(0), mx(-bottom, T(0))};
            k.aa = v4(sp - xyz(pos[b]), T(0));
            k.ab = {T(0), T(0), T(0), role != 0 ? T(-1) : T(0)};
            emit[i] = 1;
        }
        for (uint32_t i = 0; i < C; ++i) {
            if (!emit[i]) continue;
            contacts.push_back(out[i]);
            contact_keys.push_back(((uint64_t)i << 32) | INVALID);
            features.push_back(0xffffu);
        }
    }

    // ----------------------------------------- collision.wgsl:674-736, 752
    V3<T> contact_velocity(uint32_t b, V3<T> arm) const { return xyz(lin[b]) + cross(xyz(ang[b]), arm); }

    void prepare_contacts() {
        uint64_t K = contacts.size();
        diag.contact_count = (uint32_t)std::min<uint64_t>(K, 0xffffffffull);
        if (K > pair_capacity) {
            diag.error_flags |= MK_PAIR_OVERFLOW_FLAG;
            contacts.resize(pair_capacity); contact_keys.resize(pair_capacity); features.resize(pair_capacity);
            K = pair_capacity;
        }
        std::vector<uint8_t> act(K);
        std::vector<uint8_t> acq(K);
#pragma omp parallel for schedule(static)
        for (int64_t kk = 0; kk < (int64_t)K; ++kk) {
            Contact<T>& c = contacts[kk];
            act[kk] = 0; acq[kk] = 0;
            uint32_t a = c.meta[0], b = c.meta[1];
            V3<T> arm_a = xyz(c.aa), arm_b = xyz(c.ab);
            T inv_b = T(0);
            V3<T> vb = v3<T>(0, 0, 0);
            if (b != INVALID) { inv_b = wm[b].x.w; vb = contact_velocity(b, arm_b); }
            if (wm[a].x.w + inv_b <= T(0)) continue;
            V3<T> rel = vb - contact_velocity(a, arm_a);
            V3<T> n = xyz(c.np);
            T vn = dot(rel, n);
            if (c.np.w <= T(1.0e-6f) && vn >= T(0)) { c.meta[2] = INVALID; c.meta[3] = 0; continue; }
            // acquire_manifold (collision.wgsl:499-538) as a map keyed by the
            // ordered collider pair; the hash slot is not part of parity.
            uint64_t key = contact_keys[kk];
            T cached_impulse = T(0);
            if (clipped) {   // the first of the pair's previous rows whose normal and arm match
                auto it = manifold_rows.find(key);
                if (it != manifold_rows.end())
                    for (const Manifold<T>& m : it->second)
                        if (m.tick == tick32 - 1u && dot(xyz(m.np), n) >= T(0.98f) &&
                            length(xyz(m.pi) - arm_a) <= T(0.02f)) {
                            cached_impulse = m.pi.w;
                            break;
                        }
            } else {
                auto it = manifold.find(key);
                if (it != manifold.end()) {
                    const Manifold<T>& m = it->second;
                    bool match = m.tick == tick32 - 1u && dot(xyz(m.np), n) >= T(0.98f) &&
                                 length(xyz(m.pi) - arm_a) <= T(0.02f);
                    if (match) cached_impulse = m.pi.w;
                }
            }
            c.meta[2] = (uint32_t)kk;
            c.meta[3] = 1;
            c.aa.w = cached_impulse;
            acq[kk] = 1;
            if (c.np.w > T(1.0e-5f) || vn < T(-1.0e-5f) || cached_impulse > T(1.0e-6f)) act[kk] = 1;
        }
        active.clear();
        for (uint64_t kk = 0; kk < K; ++kk)
            if (act[kk]) active.push_back((uint32_t)kk);
        acquired_flags.swap(acq);
        diag.active_contact_count = (uint32_t)active.size();
    }
    std::vector<uint8_t> acquired_flags;

    // ----------------------------------------- collision.wgsl:109-132
    V3<T> inverse_inertia(uint32_t b, V3<T> v) const {
        const WorldMass<T>& m = wm[b];
        return xyz(m.x) * v.x + xyz(m.y) * v.y + xyz(m.z) * v.z;
    }
    T impulse_denominator(uint32_t a, uint32_t b, V3<T> arm_a, V3<T> arm_b, V3<T> d) const {
        T r = wm[a].x.w;
        V3<T> ang_a = cross(inverse_inertia(a, cross(arm_a, d)), arm_a);
        r += dot(ang_a, d);
        if (b != INVALID) {
            r += wm[b].x.w;
            V3<T> ang_b = cross(inverse_inertia(b, cross(arm_b, d)), arm_b);
            r += dot(ang_b, d);
        }
        return r;
    }
    T penetration_bias(T pen, bool cyl) const {
        T recovery = cyl ? T(1) : T(0.2f);
        return mn(mx(pen - T(0.001f), T(0)) * recovery / dt, T(1));
    }
    void add_delta(uint32_t b, V3<T> l, V3<T> a) {
        const T s = T(1048576.0f);
        uint32_t* d = &deltas[6 * (size_t)b];
        int32_t v[6] = {fixed_i32(l.x * s), fixed_i32(l.y * s), fixed_i32(l.z * s),
                        fixed_i32(a.x * s), fixed_i32(a.y * s), fixed_i32(a.z * s)};
        for (int k = 0; k < 6; ++k) {
            std::atomic_ref<uint32_t> r(d[k]);
            r.fetch_add((uint32_t)v[k], std::memory_order_relaxed);
        }
    }
    // warm_start (collision.wgsl:774-839) when warm, solve_accumulate (:841-906) otherwise.
    void solve_contact(uint32_t ci, bool warm) {
        Contact<T>& c = contacts[ci];
        uint32_t a = c.meta[0], b = c.meta[1];
        V3<T> arm_a = xyz(c.aa), arm_b = xyz(c.ab);
        V3<T> vb = v3<T>(0, 0, 0);
        if (b != INVALID) vb = contact_velocity(b, arm_b);
        V3<T> n = xyz(c.np);
        T den = impulse_denominator(a, b, arm_a, arm_b, n);
        if (den <= T(0)) return;
        V3<T> rel = vb - contact_velocity(a, arm_a);
        T vn = dot(rel, n);
        if (c.np.w <= T(1.0e-5f) && vn >= T(-1.0e-5f) && c.aa.w <= T(1.0e-6f)) { c.aa.w = T(0); return; }
        bool cyl = c.ab.w < T(0);
        T bias = penetration_bias(c.np.w, cyl);
        T acc, delta;
        if (warm) {
            T ws = cyl ? T(1) : T(0.5f);
            T warmed = c.aa.w * ws;
            acc = mx(warmed + T(0.125f) * (-vn + bias) / den, T(0));
            delta = acc;
        } else {
            T prev = mx(c.aa.w, T(0));
            acc = mx(prev + T(0.125f) * (-vn + bias) / den, T(0));
            delta = acc - prev;
        }
        c.aa.w = acc;
        V3<T> imp = n * delta;
        V3<T> tv = rel - n * vn;
        T ts = length(tv);
        if (ts > T(1.0e-6f)) {
            V3<T> t = tv / ts;
            T dt_den = impulse_denominator(a, b, arm_a, arm_b, t);
            T fr = mn(ts / dt_den, (warm ? acc : std::fabs(delta)) * T(0.05f));
            imp = imp - t * fr;
        }
        add_delta(a, -imp * wm[a].x.w, inverse_inertia(a, cross(arm_a, -imp)));
        if (b != INVALID) add_delta(b, imp * wm[b].x.w, inverse_inertia(b, cross(arm_b, imp)));
    }
    // solve_apply (collision.wgsl:1050-1069)
    void solve_apply() {
        const T s = T(1048576.0f);
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t* d = &deltas[6 * bb];
            V3<T> ld = v3<T>(T((int32_t)d[0]), T((int32_t)d[1]), T((int32_t)d[2])) / s;
            V3<T> ad = v3<T>(T((int32_t)d[3]), T((int32_t)d[4]), T((int32_t)d[5])) / s;
            for (int k = 0; k < 6; ++k) d[k] = 0;
            lin[bb] = v4(xyz(lin[bb]) + ld, T(0));
            ang[bb] = v4(xyz(ang[bb]) + ad, T(0));
        }
    }
    void solve() {
        uint32_t A = (uint32_t)active.size();
        for (uint32_t it = 0; it < std::max(1u, iterations); ++it) {
#pragma omp parallel for schedule(static)
            for (int64_t k = 0; k < (int64_t)A; ++k) solve_contact(active[k], it == 0);
            if (A > 0) solve_apply();
        }
    }
    // ------------------------------------------- contact solve to a residual
    // The fixed passes of solve() repeated until ||r_k|| <= tol * ||r_cold||
    // (or max passes), with r the unrelaxed projected step of the normal row
    // at the state entering a pass, FP64 norms summed in one fixed order
    // (stride-halving trees of 1024 over chunks, then over chunk sums), and
    // 64-bit fixed-point deltas (x 2^32).  With learned predictions two
    // candidates (cached start, predicted start) run the first two passes;
    // the smaller residual after the first pass continues.
    float contact_tol = 0.0f;
    uint32_t contact_max_it = 512;
    std::vector<float> warm_predictions;   // by active position, consumed by the next solve
    bool learned_pending = false;
    struct SolveStats { uint32_t iterations = 0, chosen = 0, converged = 0; double s0 = 0, sk = 0; } stats;

    static double tree1024(const double* v, size_t n) {
        double t[1024];
        for (size_t i = 0; i < 1024; ++i) t[i] = i < n ? v[i] : 0.0;
        for (size_t stride = 512; stride >= 1; stride >>= 1)
            for (size_t i = 0; i < stride; ++i) t[i] += t[i + stride];
        return t[0];
    }
    static double canonical_norm2(const std::vector<double>& r2) {
        std::vector<double> v;
        for (size_t c = 0; c < r2.size(); c += 1024) v.push_back(tree1024(&r2[c], std::min<size_t>(1024, r2.size() - c)));
        while (v.size() > 1) {
            std::vector<double> u;
            for (size_t c = 0; c < v.size(); c += 1024) u.push_back(tree1024(&v[c], std::min<size_t>(1024, v.size() - c)));
            v.swap(u);
        }
        return v.empty() ? 0.0 : v[0];
    }
    void add_delta64(std::vector<uint64_t>& d64, uint32_t b, V3<T> l, V3<T> a) {
        const T s = T(4294967296.0f);
        uint64_t* d = &d64[6 * (size_t)b];
        int64_t v[6] = {fixed_i64(l.x * s), fixed_i64(l.y * s), fixed_i64(l.z * s),
                        fixed_i64(a.x * s), fixed_i64(a.y * s), fixed_i64(a.z * s)};
        for (int k = 0; k < 6; ++k) {
            std::atomic_ref<uint64_t> r(d[k]);
            r.fetch_add((uint64_t)v[k], std::memory_order_relaxed);
        }
    }
    // One contact of one candidate; returns the residual (0 when skipped).
    T solve_contact_res(uint32_t t, bool warm, uint32_t cand, const std::vector<V4<T>>& vl,
                        const std::vector<V4<T>>& va, std::vector<T>& lam_alt, std::vector<uint64_t>& d64) {
        Contact<T>& c = contacts[active[t]];
        uint32_t a = c.meta[0], b = c.meta[1];
        V3<T> arm_a = xyz(c.aa), arm_b = xyz(c.ab);
        auto vel = [&](uint32_t body, V3<T> arm) { return xyz(vl[body]) + cross(xyz(va[body]), arm); };
        V3<T> vb = v3<T>(0, 0, 0);
        if (b != INVALID) vb = vel(b, arm_b);
        V3<T> n = xyz(c.np);
        T den = impulse_denominator(a, b, arm_a, arm_b, n);
        T& lam = cand == 0 ? c.aa.w : lam_alt[t];
        if (warm && cand == 1) lam = T(warm_predictions[t]);
        if (den <= T(0)) return T(0);
        V3<T> rel = vb - vel(a, arm_a);
        T vn = dot(rel, n);
        if (c.np.w <= T(1.0e-5f) && vn >= T(-1.0e-5f) && lam <= T(1.0e-6f)) { lam = T(0); return T(0); }
        bool cyl = c.ab.w < T(0);
        T bias = penetration_bias(c.np.w, cyl);
        T acc, delta, r;
        if (warm) {
            T start = cand == 0 ? c.aa.w * (cyl ? T(1) : T(0.5f)) : lam;
            acc = mx(start + T(0.125f) * (-vn + bias) / den, T(0));
            delta = acc;
            r = mx((-vn + bias) / den, T(0));
        } else {
            T prev = mx(lam, T(0));
            acc = mx(prev + T(0.125f) * (-vn + bias) / den, T(0));
            delta = acc - prev;
            r = mx(prev + (-vn + bias) / den, T(0)) - prev;
        }
        lam = acc;
        V3<T> imp = n * delta;
        V3<T> tv = rel - n * vn;
        T ts = length(tv);
        if (ts > T(1.0e-6f)) {
            V3<T> tg = tv / ts;
            T tden = impulse_denominator(a, b, arm_a, arm_b, tg);
            T fr = mn(ts / tden, (warm ? acc : std::fabs(delta)) * T(0.05f));
            imp = imp - tg * fr;
        }
        add_delta64(d64, a, -imp * wm[a].x.w, inverse_inertia(a, cross(arm_a, -imp)));
        if (b != INVALID) add_delta64(d64, b, imp * wm[b].x.w, inverse_inertia(b, cross(arm_b, imp)));
        return r;
    }
    void solve_residual() {
        const uint32_t A = (uint32_t)active.size();
        stats = SolveStats{};
        const bool learned = learned_pending;
        learned_pending = false;
        if (A == 0) { stats.converged = 1; return; }
        if (learned && warm_predictions.size() < A) warm_predictions.resize(A, 0.0f);
        std::vector<V4<T>> vl[2] = {lin, lin}, va[2] = {ang, ang};
        std::vector<T> lam_alt(A, T(0));
        std::vector<uint64_t> d64[2] = {std::vector<uint64_t>(6ull * B, 0), std::vector<uint64_t>(6ull * B, 0)};
        std::vector<double> r2[2] = {std::vector<double>(A, 0.0), std::vector<double>(A, 0.0)};
        const double tol2 = (double)contact_tol * (double)contact_tol;
        bool dual = learned;
        uint32_t chosen = 0, it = 0;
        double s0 = 0.0, sk = 0.0;
        while (it < contact_max_it) {
            const uint32_t c_first = dual ? 0u : chosen, c_last = dual ? 1u : chosen;
            for (uint32_t c = c_first; c <= c_last; ++c) {
                const bool warm = it == 0;
#pragma omp parallel for schedule(static)
                for (int64_t t = 0; t < (int64_t)A; ++t) {
                    T r = solve_contact_res((uint32_t)t, warm, c, vl[c], va[c], lam_alt, d64[c]);
                    if (!(warm && c == 1)) r2[c][t] = double(r) * double(r);
                }
                const T s = T(2.3283064365386963e-10f);
#pragma omp parallel for schedule(static)
                for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
                    uint64_t* d = &d64[c][6 * bb];
                    V3<T> ld = v3<T>(T((int64_t)d[0]), T((int64_t)d[1]), T((int64_t)d[2])) * s;
                    V3<T> ad = v3<T>(T((int64_t)d[3]), T((int64_t)d[4]), T((int64_t)d[5])) * s;
                    for (int k = 0; k < 6; ++k) d[k] = 0;
                    vl[c][bb] = v4(xyz(vl[c][bb]) + ld, T(0));
                    va[c][bb] = v4(xyz(va[c][bb]) + ad, T(0));
                }
            }
            double S[2] = {0.0, 0.0};
            if (it == 0) S[c_first] = canonical_norm2(r2[c_first]);
            else for (uint32_t c = c_first; c <= c_last; ++c) S[c] = canonical_norm2(r2[c]);
            ++it;
            if (it == 1) { s0 = S[c_first]; sk = s0; continue; }
            if (dual) { chosen = S[1] <= S[0] ? 1u : 0u; dual = false; }
            sk = S[chosen];
            if (sk <= tol2 * s0) { stats.converged = 1; break; }
        }
        lin = vl[chosen]; ang = va[chosen];
        if (chosen == 1)
            for (uint32_t t = 0; t < A; ++t) contacts[active[t]].aa.w = lam_alt[t];
        stats.iterations = it; stats.chosen = chosen; stats.s0 = s0; stats.sk = sk;
    }

    // persist_contacts (collision.wgsl:1071-1088) + the prepare-time writes:
    // every acquired contact's manifold entry holds this tick's values.
    void persist() {
        if (clipped) manifold_rows.clear();
        for (size_t k = 0; k < contacts.size(); ++k) {
            if (acquired_flags.size() <= k || !acquired_flags[k]) continue;
            const Contact<T>& c = contacts[k];
            Manifold<T> m;
            m.tick = tick32;
            m.count = 1;
            m.np = c.np;
            m.pi = c.aa;
            if (clipped) manifold_rows[contact_keys[k]].push_back(m);
            else manifold[contact_keys[k]] = m;
        }
        last_tick = tick32;
    }
    uint32_t last_tick = 0;

    // ----------------------------------------------- snapshot.wgsl:6-14
    void snapshot(uint32_t slot) {
        snap_pos[slot] = pos;
        snap_rot[slot] = rot;
    }


    // ================================================= articulated passes
    // mechanism.wgsl:67-185, articulated.wgsl:94-484, closure.wgsl:94-427,
    // bearings.wgsl:48-102, in the dispatch order of device.rs:963-1155.
    std::vector<Link<T>> links_a, links_b;
    std::vector<uint32_t> mdeltas;     // bearing-projection fixed-point deltas (6 per body)
    std::vector<T> grad, dgl;          // closure accumulators
    uint32_t closure_state[2] = {0, 0};
    struct Pcg { T sol, res, pre, dir, op; };
    std::vector<Pcg> pcg;
    uint32_t jump_rounds = 0;
    bool final_is_a = true;
    std::vector<Link<T>>& final_links() { return final_is_a ? links_a : links_b; }

    V3<T> wii(uint32_t b, V3<T> v) const {   // articulated.wgsl:94-102 (body-frame mass rows)
        V4<T> r = rot[b];
        V3<T> l = quat_rotate(conj(r), v);
        const Mass<T>& m = mass[b];
        V3<T> lr = m.ix * l.x + m.iy * l.y + m.iz * l.z;
        return quat_rotate(r, lr);
    }
    void add_mdelta(uint32_t b, V3<T> l, V3<T> a) {   // articulated.wgsl:104-112
        const T s = T(1048576.0f);
        uint32_t* d = &mdeltas[6 * (size_t)b];
        int32_t v[6] = {fixed_i32(l.x * s), fixed_i32(l.y * s), fixed_i32(l.z * s),
                        fixed_i32(a.x * s), fixed_i32(a.y * s), fixed_i32(a.z * s)};
        for (int k = 0; k < 6; ++k) {
            std::atomic_ref<uint32_t> r(d[k]);
            r.fetch_add((uint32_t)v[k], std::memory_order_relaxed);
        }
    }
    void solve_linear_axis(uint32_t a, uint32_t b, V3<T> arm_a, V3<T> arm_b, V3<T> rel, V3<T> d) {   // :114-143
        V3<T> ang_a = cross(arm_a, d), ang_b = cross(arm_b, d);
        T den = mass[a].inv_mass + mass[b].inv_mass + dot(ang_a, wii(a, ang_a)) + dot(ang_b, wii(b, ang_b));
        if (den <= T(1.0e-12f)) return;
        V3<T> imp = d * (T(0.5f) * dot(rel, d) / den);
        add_mdelta(a, imp * mass[a].inv_mass, wii(a, cross(arm_a, imp)));
        add_mdelta(b, -imp * mass[b].inv_mass, wii(b, cross(arm_b, -imp)));
    }
    void solve_angular_axis(uint32_t a, uint32_t b, V3<T> rel, V3<T> axis) {   // :145-155
        V3<T> ia = wii(a, axis), ib = wii(b, axis);
        T den = dot(axis, ia + ib);
        if (den <= T(1.0e-12f)) return;
        T imp = T(0.5f) * dot(rel, axis) / den;
        add_mdelta(a, v3<T>(0, 0, 0), ia * imp);
        add_mdelta(b, v3<T>(0, 0, 0), -ib * imp);
    }
    void hinge_tangents(uint32_t a, uint32_t b, const Bearing<T>& br, V3<T>& ta, V3<T>& tb) const {
        V3<T> axa = normalize(quat_rotate(rot[a], xyz(br.xa)));
        V3<T> axb = normalize(quat_rotate(rot[b], xyz(br.xb)));
        V3<T> hinge = normalize(axa + axb);
        V3<T> helper = std::fabs(hinge.x) > T(0.8f) ? v3<T>(0, 1, 0) : v3<T>(1, 0, 0);
        ta = normalize(cross(hinge, helper));
        tb = cross(hinge, ta);
    }
    void project_bearing_velocities() {   // articulated.wgsl:287-316 (relaxed Jacobi)
#pragma omp parallel for schedule(static)
        for (int64_t jj = 0; jj < (int64_t)J; ++jj) {
            const Bearing<T>& br = bear[jj];
            uint32_t a = br.meta[0], b = br.meta[1];
            V3<T> arm_a = quat_rotate(rot[a], xyz(br.aa)), arm_b = quat_rotate(rot[b], xyz(br.ab));
            V3<T> va = xyz(lin[a]) + cross(xyz(ang[a]), arm_a);
            V3<T> vb = xyz(lin[b]) + cross(xyz(ang[b]), arm_b);
            V3<T> rel = vb - va;
            solve_linear_axis(a, b, arm_a, arm_b, rel, v3<T>(1, 0, 0));
            solve_linear_axis(a, b, arm_a, arm_b, rel, v3<T>(0, 1, 0));
            solve_linear_axis(a, b, arm_a, arm_b, rel, v3<T>(0, 0, 1));
            V3<T> ta, tb;
            hinge_tangents(a, b, br, ta, tb);
            V3<T> rang = xyz(ang[b]) - xyz(ang[a]);
            solve_angular_axis(a, b, rang, ta);
            solve_angular_axis(a, b, rang, tb);
        }
    }
    void apply_mdeltas() {   // articulated.wgsl:318-337
        const T s = T(1048576.0f);
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t* d = &mdeltas[6 * bb];
            V3<T> ld = v3<T>(T((int32_t)d[0]), T((int32_t)d[1]), T((int32_t)d[2])) / s;
            V3<T> ad = v3<T>(T((int32_t)d[3]), T((int32_t)d[4]), T((int32_t)d[5])) / s;
            for (int k = 0; k < 6; ++k) d[k] = 0;
            lin[bb] = v4(xyz(lin[bb]) + ld, T(0));
            ang[bb] = v4(xyz(ang[bb]) + ad, T(0));
        }
    }
    void bearing_projection_iteration() { project_bearing_velocities(); apply_mdeltas(); }

    // serial Gauss-Seidel variants (articulated.wgsl:157-285)
    void linear_axis_immediate(uint32_t a, uint32_t b, V3<T> arm_a, V3<T> arm_b, V3<T> rel, V3<T> d) {
        V3<T> ang_a = cross(arm_a, d), ang_b = cross(arm_b, d);
        T den = mass[a].inv_mass + mass[b].inv_mass + dot(ang_a, wii(a, ang_a)) + dot(ang_b, wii(b, ang_b));
        if (den <= T(1.0e-12f)) return;
        V3<T> imp = d * (dot(rel, d) / den);
        lin[a] = v4(xyz(lin[a]) + imp * mass[a].inv_mass, T(0));
        ang[a] = v4(xyz(ang[a]) + wii(a, cross(arm_a, imp)), T(0));
        lin[b] = v4(xyz(lin[b]) - imp * mass[b].inv_mass, T(0));
        ang[b] = v4(xyz(ang[b]) + wii(b, cross(arm_b, -imp)), T(0));
    }
    void angular_axis_immediate(uint32_t a, uint32_t b, V3<T> rel, V3<T> axis) {
        V3<T> ia = wii(a, axis), ib = wii(b, axis);
        T den = dot(axis, ia + ib);
        if (den <= T(1.0e-12f)) return;
        T imp = dot(rel, axis) / den;
        ang[a] = v4(xyz(ang[a]) + ia * imp, T(0));
        ang[b] = v4(xyz(ang[b]) - ib * imp, T(0));
    }
    void project_bearing_row_immediate(uint32_t j) {
        const Bearing<T>& br = bear[j];
        uint32_t a = br.meta[0], b = br.meta[1];
        V3<T> arm_a = quat_rotate(rot[a], xyz(br.aa)), arm_b = quat_rotate(rot[b], xyz(br.ab));
        const V3<T> dirs[3] = {v3<T>(1, 0, 0), v3<T>(0, 1, 0), v3<T>(0, 0, 1)};
        for (int k = 0; k < 3; ++k) {
            V3<T> va = xyz(lin[a]) + cross(xyz(ang[a]), arm_a);
            V3<T> vb = xyz(lin[b]) + cross(xyz(ang[b]), arm_b);
            linear_axis_immediate(a, b, arm_a, arm_b, vb - va, dirs[k]);
        }
        V3<T> ta, tb;
        hinge_tangents(a, b, br, ta, tb);
        V3<T> rang = xyz(ang[b]) - xyz(ang[a]);
        angular_axis_immediate(a, b, rang, ta);
        rang = xyz(ang[b]) - xyz(ang[a]);
        angular_axis_immediate(a, b, rang, tb);
    }
    void project_bearing_velocities_serial() {
        for (uint32_t j = 0; j < J; ++j) project_bearing_row_immediate(j);
        for (uint32_t j = J; j > 0; --j) project_bearing_row_immediate(j - 1);
    }

    V3<T> permitted_axis(uint32_t body) const {   // articulated.wgsl:339-348
        const MechBody<T>& m = mech[body];
        uint32_t parent = m.meta[0];
        const Bearing<T>& br = bear[m.meta[1]];
        V3<T> axis = normalize(quat_rotate(rot[parent], xyz(br.xa)));
        if (m.meta[2] != 0) axis = -normalize(quat_rotate(rot[parent], xyz(br.xb)));
        return axis;
    }
    T permitted_speed(uint32_t body) const {
        uint32_t parent = mech[body].meta[0];
        return dot(xyz(ang[body]) - xyz(ang[parent]), permitted_axis(body));
    }
    T stabilized_speed(uint32_t body, T speed) const {
        bool aligned = std::fabs(permitted_axis(body).y) > T(0.999f);
        return (aligned && std::fabs(speed) < T(0.005f)) ? T(0) : speed;
    }
    void advance_coordinates() {   // articulated.wgsl:366-415
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t body = (uint32_t)bb;
            if (mech[body].meta[3] != 0) continue;
            const Bearing<T>& br = bear[mech[body].meta[1]];
            uint32_t c = br.meta[2];
            if (c == INVALID) continue;
            T measured = permitted_speed(body) * ang_damp;
            const Drive& dr = drives[c];
            T speed = T(0);
            if (dr.mode == MK_DRIVE_MODE_PASSIVE) {
                speed = stabilized_speed(body, measured);
            } else {
                T desired = clampv(T(dr.target_speed), T(-dr.max_speed), T(dr.max_speed));
                if (dr.mode == MK_DRIVE_MODE_ANGLE) {
                    T err = T(dr.target_angle) - coords[c].x;
                    T brake = std::sqrt(T(2) * T(dr.max_acc) * std::fabs(err));
                    desired = sgn(err) * mn(brake, T(dr.max_speed));
                    if (std::fabs(err) < T(0.0005f)) desired = T(0);
                }
                T budget = T(dr.max_acc) * dt;
                speed = measured + clampv(desired - measured, -budget, budget);
            }
            T angle = coords[c].x + speed * dt;
            if (angle < T(dr.min_angle)) { angle = T(dr.min_angle); speed = T(0); }
            else if (angle > T(dr.max_angle)) { angle = T(dr.max_angle); speed = T(0); }
            coords[c].y = speed;
            coords[c].x = angle;
        }
    }
    void capture_coordinates() {   // articulated.wgsl:417-429
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t body = (uint32_t)bb;
            if (mech[body].meta[3] != 0) continue;
            uint32_t c = bear[mech[body].meta[1]].meta[2];
            if (c != INVALID) coords[c].y = stabilized_speed(body, permitted_speed(body));
        }
    }
    void reconstruct_body_velocities() {   // articulated.wgsl:431-456 (serial preorder)
        for (uint32_t t = 0; t < B; ++t) {
            uint32_t body = preorder[t];
            const MechBody<T>& m = mech[body];
            if (m.meta[3] != 0) continue;
            uint32_t parent = m.meta[0];
            const Bearing<T>& br = bear[m.meta[1]];
            V3<T> axis = normalize(quat_rotate(rot[parent], xyz(br.xa)));
            V3<T> pa = quat_rotate(rot[parent], xyz(br.aa));
            V3<T> ca = quat_rotate(rot[body], xyz(br.ab));
            if (m.meta[2] != 0) {
                axis = -normalize(quat_rotate(rot[parent], xyz(br.xb)));
                pa = quat_rotate(rot[parent], xyz(br.ab));
                ca = quat_rotate(rot[body], xyz(br.aa));
            }
            T speed = coords[br.meta[2]].y;
            V3<T> angular = xyz(ang[parent]) + axis * speed;
            V3<T> av = xyz(lin[parent]) + cross(xyz(ang[parent]), pa);
            lin[body] = v4(av - cross(angular, ca), T(0));
            ang[body] = v4(angular, T(0));
        }
    }
    void validate_articulated_state() {   // articulated.wgsl:458-484
        std::atomic<uint32_t> bad{0};
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t body = (uint32_t)bb;
            T rl = dot4(rot[body], rot[body]);
            bool valid = finite4(pos[body]) && finite4(rot[body]) && finite4(lin[body]) && finite4(ang[body]) &&
                         rl > T(0.5f) && rl < T(1.5f);
            const MechBody<T>& m = mech[body];
            if (m.meta[3] == 0) {
                uint32_t c = bear[m.meta[1]].meta[2];
                const V4<T>& st = coords[c];
                const T lim = T(3.402823e+38f);
                valid = valid && st.x == st.x && std::fabs(st.x) < lim && st.y == st.y && std::fabs(st.y) < lim;
            }
            if (!valid) bad = 1;
        }
        if (bad.load()) diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
    }

    // ---------------------------------------------- forward kinematics
    static V4<T> axis_rotation(V3<T> axis, T angle) {   // mechanism.wgsl:67-70
        T h = angle * T(0.5f);
        V3<T> v = normalize(axis) * tsin(h);
        return {v.x, v.y, v.z, tcos(h)};
    }
    void prepare_links() {   // mechanism.wgsl:72-108
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t body = (uint32_t)bb;
            const MechBody<T>& m = mech[body];
            Link<T>& L = links_a[body];
            if (m.meta[3] != 0) {
                L.pos = {0, 0, 0, 0}; L.rot = {0, 0, 0, 1};
                L.meta[0] = body; L.meta[1] = 1; L.meta[2] = 0; L.meta[3] = 0;
                continue;
            }
            const Bearing<T>& br = bear[m.meta[1]];
            T angle = coords[br.meta[2]].x;
            V4<T> rr;
            V3<T> rp;
            if (m.meta[2] == 0) {
                rr = quat_multiply(axis_rotation(xyz(br.xa), angle), m.brot);
                rp = xyz(br.aa) - quat_rotate(rr, xyz(br.ab));
            } else {
                rr = quat_multiply(axis_rotation(xyz(br.xb), -angle), m.brot);
                rp = xyz(br.ab) - quat_rotate(rr, xyz(br.aa));
            }
            L.pos = v4(rp, T(0)); L.rot = rr;
            L.meta[0] = m.meta[0]; L.meta[1] = 0; L.meta[2] = 0; L.meta[3] = 0;
        }
    }
    static Link<T> compose(const Link<T>& child, const Link<T>& parent) {   // mechanism.wgsl:110-119
        Link<T> r;
        r.pos = v4(xyz(parent.pos) + quat_rotate(parent.rot, xyz(child.pos)), T(0));
        r.rot = normalize4(quat_multiply(parent.rot, child.rot));
        r.meta[0] = parent.meta[0]; r.meta[1] = 0; r.meta[2] = 0; r.meta[3] = 0;
        return r;
    }
    void jump(const std::vector<Link<T>>& src, std::vector<Link<T>>& dst) {   // mechanism.wgsl:121-149
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            const Link<T>& child = src[bb];
            if (child.meta[1] != 0) { dst[bb] = child; continue; }
            const Link<T>& par = src[child.meta[0]];
            dst[bb] = compose(child, par);
            dst[bb].meta[1] = par.meta[1];
        }
    }
    void forward_kinematics() {
        prepare_links();
        bool a_final = true;
        for (uint32_t r = 0; r < jump_rounds; ++r) {
            if (a_final) jump(links_a, links_b); else jump(links_b, links_a);
            a_final = !a_final;
        }
    }
    void publish() {   // mechanism.wgsl:151-185
        const std::vector<Link<T>>& L = final_links();
#pragma omp parallel for schedule(static)
        for (int64_t bb = 0; bb < (int64_t)B; ++bb) {
            uint32_t root_body = L[bb].meta[0];
            if ((uint32_t)bb == root_body) continue;
            pos[bb] = v4(xyz(pos[root_body]) + quat_rotate(rot[root_body], xyz(L[bb].pos)), T(0));
            rot[bb] = normalize4(quat_multiply(rot[root_body], L[bb].rot));
        }
    }

    // ------------------------------------------------------ closures
    struct Vec2 { V3<T> p, a; };
    void joint_frame(uint32_t body, V3<T>& axis, V3<T>& anchor, uint32_t& coord, uint32_t& parent) const {
        const MechBody<T>& m = mech[body];
        parent = m.meta[0];
        const Bearing<T>& tb = bear[m.meta[1]];
        const Link<T>& pp = links_final_const()[parent];
        if (m.meta[2] == 0) {
            axis = normalize(quat_rotate(pp.rot, xyz(tb.xa)));
            anchor = xyz(pp.pos) + quat_rotate(pp.rot, xyz(tb.aa));
        } else {
            axis = -normalize(quat_rotate(pp.rot, xyz(tb.xb)));
            anchor = xyz(pp.pos) + quat_rotate(pp.rot, xyz(tb.ab));
        }
        coord = tb.meta[2];
    }
    const std::vector<Link<T>>& links_final_const() const { return final_is_a ? links_a : links_b; }
    void closure_frames(const Bearing<T>& br, V3<T>& anc_a, V3<T>& anc_b, V3<T>& ax_a, V3<T>& ax_b) const {
        const std::vector<Link<T>>& L = links_final_const();
        const Link<T>& pa = L[br.meta[0]];
        const Link<T>& pb = L[br.meta[1]];
        anc_a = xyz(pa.pos) + quat_rotate(pa.rot, xyz(br.aa));
        anc_b = xyz(pb.pos) + quat_rotate(pb.rot, xyz(br.ab));
        ax_a = normalize(quat_rotate(pa.rot, xyz(br.xa)));
        ax_b = normalize(quat_rotate(pb.rot, xyz(br.xb)));
    }
    // Reference-loop slot values, kept only when a coordinate's run is long enough for
    // the GPU's two-level sum (gather_run): rec_g/rec_d per slot (NaN: no contribution).
    bool rec_long = false;
    std::vector<T> rec_g, rec_d;
    void accumulate_branch(uint32_t start, V3<T> ea, V3<T> ex, V3<T> rp, V3<T> ra, T sign,
                           uint32_t* slot = nullptr) {   // closure.wgsl:128-192
        uint32_t body = start;
        for (uint32_t guard = 0; guard <= B; ++guard) {
            if (mech[body].meta[3] != 0) break;
            V3<T> axis, anchor; uint32_t c, parent;
            joint_frame(body, axis, anchor, c, parent);
            if (c >= Q) { diag.error_flags |= MK_INVALID_NUMERIC_FLAG; }
            else {
                V3<T> pd = cross(axis, ea - anchor) * sign;
                V3<T> ad = cross(axis, ex) * sign;
                T g = dot(rp, pd) + T(1) * dot(ra, ad);
                T d = dot(pd, pd) + T(1) * dot(ad, ad);
                if (g == g && d == d) {
                    grad[c] += g; dgl[c] += d;
                    if (slot) { rec_g[*slot] = g; rec_d[*slot] = d; }
                }
                else diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
            }
            if (slot) ++*slot;
            body = parent;
        }
    }
    // After the serial accumulation: the long runs summed in the GPU's two levels instead.
    void regather_long(std::vector<T>& out_g, std::vector<T>* out_d) const {
        for (size_t q = 0; q + 1 < ct.cq_off.size(); ++q) {
            if (ct.cq_off[q + 1] - ct.cq_off[q] <= kLongList) continue;
            T g, d;
            if (out_d) gather_run<true>((uint32_t)q, rec_g, rec_d, g, d);
            else gather_run<false>((uint32_t)q, rec_g, rec_g, g, d);
            out_g[ct.cq_coords[q]] = g;
            if (out_d) (*out_d)[ct.cq_coords[q]] = d;
        }
    }
    void evaluate_closures() {   // closure.wgsl:268-319 (sequential in bearing order)
        if (rec_long) {
            rec_g.assign(ct.slot_body.size(), std::numeric_limits<T>::quiet_NaN());
            rec_d.assign(ct.slot_body.size(), T(0));
        }
        uint32_t k = 0;
        for (uint32_t j = 0; j < J; ++j) {
            const Bearing<T>& br = bear[j];
            if (br.meta[3] == 0) continue;
            uint32_t slot = rec_long ? ct.cl_slot_off[k] : 0u;
            ++k;
            V3<T> aa, ab, xa, xb;
            closure_frames(br, aa, ab, xa, xb);
            V3<T> rp = aa - ab, ra = xa - xb;
            auto finite3 = [](V3<T> v) {
                const T lim = T(3.402823e+38f);
                return v.x == v.x && v.y == v.y && v.z == v.z && std::fabs(v.x) < lim && std::fabs(v.y) < lim &&
                       std::fabs(v.z) < lim;
            };
            if (!finite3(rp) || !finite3(ra)) {   // per-bearing return in the kernel
                diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
                closure_state[0] = closure_state[1] = 0xffffffffu;
                continue;
            }
            uint32_t um = round_u32(length(rp) * T(1000000.0f));
            // closure.wgsl:295 measures the axis error as acos(dot); in FP32 that
            // reads 0 below ~3.5e-4 rad (dot rounds to 1), blind to its own
            // 1000 micro-degree tolerance.  The angle is taken as
            // atan2(|a x b|, a . b), the form bearings.wgsl:56-59 validates with.
            T deg = tatan2(length(cross(xa, xb)), clampv(dot(xa, xb), T(-1), T(1))) * T(57.295779513f);
            uint32_t ud = round_u32(deg * T(1000000.0f));
            closure_state[0] = std::max(closure_state[0], um);
            closure_state[1] = std::max(closure_state[1], ud);
            if (um <= 10u && ud <= 1000u) continue;
            accumulate_branch(br.meta[0], aa, xa, rp, ra, T(1), rec_long ? &slot : nullptr);
            accumulate_branch(br.meta[1], ab, xb, rp, ra, T(-1), rec_long ? &slot : nullptr);
        }
        if (rec_long) regather_long(grad, &dgl);
    }
    Vec2 branch_product(uint32_t start, V3<T> ea, V3<T> ex, T sign) const {   // closure.wgsl:194-230
        Vec2 prod{v3<T>(0, 0, 0), v3<T>(0, 0, 0)};
        uint32_t body = start;
        for (uint32_t guard = 0; guard <= B; ++guard) {
            if (mech[body].meta[3] != 0) break;
            V3<T> axis, anchor; uint32_t c, parent;
            joint_frame(body, axis, anchor, c, parent);
            T d = pcg[c].dir;
            prod.p = prod.p + sign * cross(axis, ea - anchor) * d;
            prod.a = prod.a + sign * cross(axis, ex) * d;
            body = parent;
        }
        return prod;
    }
    void branch_transpose(uint32_t start, V3<T> ea, V3<T> ex, const Vec2& prod, T sign,
                          uint32_t* slot = nullptr) {   // closure.wgsl:232-266
        uint32_t body = start;
        for (uint32_t guard = 0; guard <= B; ++guard) {
            if (mech[body].meta[3] != 0) break;
            V3<T> axis, anchor; uint32_t c, parent;
            joint_frame(body, axis, anchor, c, parent);
            V3<T> pd = sign * cross(axis, ea - anchor);
            V3<T> ad = sign * cross(axis, ex);
            const T v = dot(pd, prod.p) + T(1) * dot(ad, prod.a);
            pcg[c].op += v;
            if (slot) rec_g[(*slot)++] = v;
            body = parent;
        }
    }
    uint32_t closure_pcg_rounds = 8;
    void solve_closure_pcg() {   // closure.wgsl:333-427 (one Newton step, 8 diagonal-PCG rounds)
        const bool chunked = ct.cq_coords.size() > kSerialDot;
        T rz = T(0);
        for (uint32_t c = 0; c < Q; ++c) {
            T g = grad[c], d = dgl[c], r = T(0), z = T(0);
            if (d > T(1.0e-12f)) { r = -g; z = r / d; }
            pcg[c] = {T(0), r, z, z, T(0)};
            rz += r * z;
        }
        if (chunked) rz = closure_dot_chunked([&](uint32_t c) { return pcg[c].res * pcg[c].pre; });
        for (uint32_t it = 0; it < closure_pcg_rounds; ++it) {
            for (uint32_t c = 0; c < Q; ++c) pcg[c].op = T(0);
            uint32_t slot = 0;
            for (uint32_t j = 0; j < J; ++j) {
                const Bearing<T>& br = bear[j];
                if (br.meta[3] == 0) continue;
                V3<T> aa, ab, xa, xb;
                closure_frames(br, aa, ab, xa, xb);
                Vec2 pa = branch_product(br.meta[0], aa, xa, T(1));
                Vec2 pb = branch_product(br.meta[1], ab, xb, T(-1));
                Vec2 prod{pa.p + pb.p, pa.a + pb.a};
                branch_transpose(br.meta[0], aa, xa, prod, T(1), rec_long ? &slot : nullptr);
                branch_transpose(br.meta[1], ab, xb, prod, T(-1), rec_long ? &slot : nullptr);
            }
            if (rec_long) {
                std::vector<T> op_long(Q, T(0));
                regather_long(op_long, nullptr);
                for (size_t q = 0; q + 1 < ct.cq_off.size(); ++q)
                    if (ct.cq_off[q + 1] - ct.cq_off[q] > kLongList) pcg[ct.cq_coords[q]].op = op_long[ct.cq_coords[q]];
            }
            T dop = T(0);
            for (uint32_t c = 0; c < Q; ++c) dop += pcg[c].dir * pcg[c].op;
            if (chunked) dop = closure_dot_chunked([&](uint32_t c) { return pcg[c].dir * pcg[c].op; });
            T alpha = std::fabs(dop) > T(1.0e-20f) ? rz / dop : T(0);
            T nrz = T(0);
            for (uint32_t c = 0; c < Q; ++c) {
                pcg[c].sol += alpha * pcg[c].dir;
                pcg[c].res -= alpha * pcg[c].op;
                T d = dgl[c];
                pcg[c].pre = T(0);
                if (d > T(1.0e-12f)) pcg[c].pre = pcg[c].res / d;
                nrz += pcg[c].res * pcg[c].pre;
            }
            if (chunked) nrz = closure_dot_chunked([&](uint32_t c) { return pcg[c].res * pcg[c].pre; });
            T beta = std::fabs(rz) > T(1.0e-20f) ? nrz / rz : T(0);
            for (uint32_t c = 0; c < Q; ++c) pcg[c].dir = pcg[c].pre + beta * pcg[c].dir;
            rz = nrz;
        }
        for (uint32_t c = 0; c < Q; ++c) {
            T st = clampv(T(0.35f) * pcg[c].sol, T(-0.2f), T(0.2f));
            if (st == st) coords[c].x += st;
            else diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
        }
    }
    void closure_loop() {   // device.rs:973-1020
        build_closure_topology();
        rec_long = has_long_runs();
        bool converged_prev = false;
        for (uint32_t step = 0; step < 12; ++step) {
            std::fill(grad.begin(), grad.end(), T(0));
            std::fill(dgl.begin(), dgl.end(), T(0));
            closure_state[0] = closure_state[1] = 0;
            if (step == 0 || !converged_prev) evaluate_closures();
            bool unconverged = closure_state[0] > 10u || closure_state[1] > 1000u;
            if (unconverged) {
                solve_closure_pcg();
                forward_kinematics();
            }
            converged_prev = !unconverged;
        }
    }

    // ------------------------------------------ closure PCG to a residual
    // MK_CLOSURE_PCG_RESIDUAL: per Newton step, PCG on (J^T J) dtheta = -g
    // until ||r|| <= tol ||r0|| with FP64 dot products summed in the order
    // of the GPU's 1024-thread block (strided partials, warp shuffle-down
    // trees, warp 0 over the warp sums); block Jacobi over 2 x 2 blocks of
    // consecutive closure coordinates, optionally replaced per block by the
    // network's output (given from outside, per Newton step).
    uint32_t closure_mode = 0, closure_max_it = 256, learned_precond = 0, precond = 0;
    std::vector<uint32_t> loop_off, loop_q;
    std::vector<T> loop_l;   // 36 per loop
    float closure_tol = 1.0e-5f;
    struct ClosureTopo {
        std::vector<uint32_t> cl_bearings, cl_slot_off, cl_split, slot_body, slot_closure, cq_coords, cq_off, cq_slots;
        bool built = false;
    } ct;
    std::vector<V3<T>> slot_pd, slot_ad;
    std::vector<uint32_t> slot_coord;
    std::vector<T> slot_g, slot_d, probe1, probe2;
    struct Blk { T m11, m12, m22; };
    std::vector<Blk> blk_m;
    std::vector<float> blk_feat;        // 16 per block
    std::vector<float> precond_outputs; // 12 x blocks x 3 (learned)
    struct ClosureStats { uint32_t newton_steps = 0, pcg_iterations = 0, learned = 0, rejected = 0; double max_rel = 0; } cstats;

    void build_closure_topology() {
        if (ct.built) return;
        ct.built = true;
        std::map<uint32_t, std::vector<uint32_t>> coord_slots;
        ct.cl_slot_off.push_back(0);
        for (uint32_t j = 0; j < J; ++j) {
            const Bearing<T>& br = bear[j];
            if (br.meta[3] == 0) continue;
            const uint32_t k = (uint32_t)ct.cl_bearings.size();
            ct.cl_bearings.push_back(j);
            for (int side = 0; side < 2; ++side) {
                if (side == 1) ct.cl_split.push_back((uint32_t)ct.slot_body.size());
                uint32_t body = br.meta[side];
                for (uint32_t guard = 0; guard <= B && body < B; ++guard) {
                    if (mech[body].meta[3] != 0) break;
                    const uint32_t coord = bear[mech[body].meta[1]].meta[2];
                    coord_slots[coord].push_back((uint32_t)ct.slot_body.size());
                    ct.slot_body.push_back(body);
                    ct.slot_closure.push_back(k);
                    body = mech[body].meta[0];
                }
            }
            ct.cl_slot_off.push_back((uint32_t)ct.slot_body.size());
        }
        ct.cq_off.push_back(0);
        for (auto& kv : coord_slots) {
            ct.cq_coords.push_back(kv.first);
            for (uint32_t sl : kv.second) ct.cq_slots.push_back(sl);
            ct.cq_off.push_back((uint32_t)ct.cq_slots.size());
        }
        // per-loop blocks (first closure containing a coordinate; pieces of at most 8)
        std::map<uint32_t, uint32_t> position;
        for (uint32_t q = 0; q < ct.cq_coords.size(); ++q) position[ct.cq_coords[q]] = q;
        std::vector<uint8_t> taken(ct.cq_coords.size(), 0);
        loop_off.assign(1, 0);
        loop_q.clear();
        for (size_t k = 0; k + 1 < ct.cl_slot_off.size(); ++k) {
            std::vector<uint32_t> qs;
            for (uint32_t sl = ct.cl_slot_off[k]; sl < ct.cl_slot_off[k + 1]; ++sl) {
                const uint32_t coord = bear[mech[ct.slot_body[sl]].meta[1]].meta[2];
                auto it = position.find(coord);
                if (it == position.end() || taken[it->second]) continue;
                taken[it->second] = 1;
                qs.push_back(it->second);
            }
            std::sort(qs.begin(), qs.end());
            for (size_t i = 0; i < qs.size(); i += 5) {   // pieces of 5: a closure's J^T J has rank <= 5
                for (size_t j = i; j < std::min<size_t>(qs.size(), i + 5); ++j) loop_q.push_back(qs[j]);
                loop_off.push_back((uint32_t)loop_q.size());
            }
        }
    }
    template <class S>
    static S block_sum_1024(const std::vector<S>& part) {   // part: 1024 per-thread partials
        S warp[32];
        for (int w = 0; w < 32; ++w) {
            S v[32];
            for (int l = 0; l < 32; ++l) v[l] = part[32 * w + l];
            for (int o = 16; o > 0; o >>= 1) {
                S nv[32];
                for (int l = 0; l < 32; ++l) nv[l] = v[l] + (l + o < 32 ? v[l + o] : v[l]);
                std::memcpy(v, nv, sizeof(v));
            }
            warp[w] = v[0];
        }
        S v[32];
        std::memcpy(v, warp, sizeof(v));
        for (int o = 16; o > 0; o >>= 1) {
            S nv[32];
            for (int l = 0; l < 32; ++l) nv[l] = v[l] + (l + o < 32 ? v[l + o] : v[l]);
            std::memcpy(v, nv, sizeof(v));
        }
        return v[0];
    }
    // The reference loop's dot products above 512 closure coordinates, in the GPU's
    // order: per chunk of 1,024 closure coordinates the block tree of the per-thread
    // terms (in T), the chunk sums added in chunk order.  Up to 512 the reference's
    // serial sum over the coordinates is kept.
    static constexpr uint32_t kSerialDot = 512;
    template <class F> T closure_dot_chunked(F term) const {   // term(c) -> T for coordinate c
        const uint32_t NQ = (uint32_t)ct.cq_coords.size();
        T acc = T(0);
        for (uint32_t c0 = 0; c0 < NQ; c0 += 1024) {
            std::vector<T> part(1024, T(0));
            for (uint32_t t = 0; t < 1024 && c0 + t < NQ; ++t) part[t] = term(ct.cq_coords[c0 + t]);
            acc += block_sum_1024(part);
        }
        return acc;
    }
    // The GPU's order: chunks of 1,024 coordinates (one per thread), the block
    // tree per chunk, the chunk sums added in chunk order.
    template <class F> double closure_dot_d(F term) const {   // term(q) -> double
        const uint32_t NQ = (uint32_t)ct.cq_coords.size();
        double acc = 0.0;
        for (uint32_t c0 = 0; c0 < NQ; c0 += 1024) {
            std::vector<double> part(1024, 0.0);
            for (uint32_t t = 0; t < 1024 && c0 + t < NQ; ++t) part[t] = term(c0 + t);
            acc += block_sum_1024(part);
        }
        return acc;
    }
    // The GPU's summation order of a closure coordinate's slot values: its run
    // serially when it has at most kLongList slots, else each chunk of kLongList
    // consecutive slots serially, then the chunk sums serially in chunk order.
    // kEval: a NaN gradient marks a slot without contribution (diagonal beside it).
    static constexpr uint32_t kLongList = 256;
    template <bool kEval>
    void gather_run(uint32_t q, const std::vector<T>& vg, const std::vector<T>& vd, T& g, T& d) const {
        const uint32_t i0 = ct.cq_off[q], i1 = ct.cq_off[q + 1];
        auto part = [&](uint32_t a, uint32_t b, T& pg, T& pd) {
            pg = T(0);
            pd = T(0);
            for (uint32_t i = a; i < b; ++i) {
                const uint32_t sl = ct.cq_slots[i];
                const T sg = vg[sl];
                if (kEval) {
                    if (sg == sg) { pg += sg; pd += vd[sl]; }
                } else {
                    pg += sg;
                }
            }
        };
        if (i1 - i0 <= kLongList) { part(i0, i1, g, d); return; }
        g = T(0);
        d = T(0);
        for (uint32_t a = i0; a < i1; a += kLongList) {
            T pg, pd;
            part(a, std::min(a + kLongList, i1), pg, pd);
            g += pg;
            if (kEval) d += pd;
        }
    }
    bool has_long_runs() const {
        for (size_t q = 0; q + 1 < ct.cq_off.size(); ++q)
            if (ct.cq_off[q + 1] - ct.cq_off[q] > kLongList) return true;
        return false;
    }
    void closure_apply(const std::vector<T>& x, std::vector<T>& out) {
        const uint32_t NC = (uint32_t)ct.cl_bearings.size();
        for (uint32_t k = 0; k < NC; ++k) {
            const uint32_t s0 = ct.cl_slot_off[k], s1 = ct.cl_slot_off[k + 1], split = ct.cl_split[k];
            V3<T> pp[2] = {v3<T>(0, 0, 0), v3<T>(0, 0, 0)}, pa[2] = {v3<T>(0, 0, 0), v3<T>(0, 0, 0)};
            for (uint32_t sl = s0; sl < s1; ++sl) {
                const int side = sl < split ? 0 : 1;
                const T dv = x[slot_coord[sl]];
                pp[side] = pp[side] + slot_pd[sl] * dv;
                pa[side] = pa[side] + slot_ad[sl] * dv;
            }
            const V3<T> P = pp[0] + pp[1], A = pa[0] + pa[1];
            for (uint32_t sl = s0; sl < s1; ++sl) slot_g[sl] = dot(slot_pd[sl], P) + T(1) * dot(slot_ad[sl], A);
        }
        for (size_t q = 0; q < ct.cq_coords.size(); ++q) {
            T o, unused;
            gather_run<false>((uint32_t)q, slot_g, slot_g, o, unused);
            out[ct.cq_coords[q]] = o;
        }
    }
    T closure_coupling(uint32_t qi, uint32_t qj) const {
        T r = T(0);
        for (uint32_t a = ct.cq_off[qi]; a < ct.cq_off[qi + 1]; ++a) {
            const uint32_t sa = ct.cq_slots[a];
            for (uint32_t b = ct.cq_off[qj]; b < ct.cq_off[qj + 1]; ++b) {
                const uint32_t sb = ct.cq_slots[b];
                if (ct.slot_closure[sa] != ct.slot_closure[sb]) continue;
                r += dot(slot_pd[sa], slot_pd[sb]) + T(1) * dot(slot_ad[sa], slot_ad[sb]);
            }
        }
        return r;
    }
    // returns false once converged
    bool closure_eval_step() {
        const uint32_t NC = (uint32_t)ct.cl_bearings.size(), NS = (uint32_t)ct.slot_body.size();
        const uint32_t NQ = (uint32_t)ct.cq_coords.size(), NBK = (NQ + 1) / 2;
        slot_pd.assign(NS, v3<T>(0, 0, 0)); slot_ad.assign(NS, v3<T>(0, 0, 0)); slot_coord.assign(NS, 0);
        slot_g.assign(NS, T(0)); slot_d.assign(NS, T(0));
        closure_state[0] = closure_state[1] = 0;
        auto finite3 = [](V3<T> v) {
            const T lim = T(3.402823e+38f);
            return v.x == v.x && v.y == v.y && v.z == v.z && std::fabs(v.x) < lim && std::fabs(v.y) < lim &&
                   std::fabs(v.z) < lim;
        };
        for (uint32_t k = 0; k < NC; ++k) {
            const Bearing<T>& br = bear[ct.cl_bearings[k]];
            V3<T> aa, ab, xa, xb;
            closure_frames(br, aa, ab, xa, xb);
            V3<T> rp = aa - ab, ra = xa - xb;
            bool active = true;
            if (!finite3(rp) || !finite3(ra)) {
                diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
                closure_state[0] = closure_state[1] = 0xffffffffu;
                active = false;
            } else {
                uint32_t um = round_u32(length(rp) * T(1000000.0f));
                T deg = tatan2(length(cross(xa, xb)), clampv(dot(xa, xb), T(-1), T(1))) * T(57.295779513f);
                uint32_t ud = round_u32(deg * T(1000000.0f));
                closure_state[0] = std::max(closure_state[0], um);
                closure_state[1] = std::max(closure_state[1], ud);
                active = !(um <= 10u && ud <= 1000u);
            }
            const uint32_t s0 = ct.cl_slot_off[k], s1 = ct.cl_slot_off[k + 1], split = ct.cl_split[k];
            for (uint32_t sl = s0; sl < s1; ++sl) {
                const bool side_a = sl < split;
                const V3<T> ea = side_a ? aa : ab, ex = side_a ? xa : xb;
                const T sign = side_a ? T(1) : T(-1);
                V3<T> axis, anchor; uint32_t coord, parent;
                joint_frame(ct.slot_body[sl], axis, anchor, coord, parent);
                bool valid = false;
                T g = T(0), d = T(0);
                if (coord >= Q) { diag.error_flags |= MK_INVALID_NUMERIC_FLAG; coord = 0; }
                else {
                    slot_pd[sl] = cross(axis, ea - anchor) * sign;
                    slot_ad[sl] = cross(axis, ex) * sign;
                    if (active) {
                        g = dot(rp, slot_pd[sl]) + T(1) * dot(ra, slot_ad[sl]);
                        d = dot(slot_pd[sl], slot_pd[sl]) + T(1) * dot(slot_ad[sl], slot_ad[sl]);
                        if (g == g && d == d) valid = true;
                        else diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
                    }
                }
                slot_coord[sl] = coord;
                slot_g[sl] = valid ? g : std::numeric_limits<T>::quiet_NaN();
                slot_d[sl] = valid ? d : T(0);
            }
        }
        for (uint32_t q = 0; q < NQ; ++q) {
            T g, d;
            gather_run<true>(q, slot_g, slot_d, g, d);
            grad[ct.cq_coords[q]] = g;
            dgl[ct.cq_coords[q]] = d;
        }
        const bool unconverged = closure_state[0] > 10u || closure_state[1] > 1000u;
        // the 2 x 2 blocks and the network's inputs, for the preconditioners that use them
        const bool pair_blocks = this->precond == MK_PRECOND_LEARNED || this->precond == MK_PRECOND_PAIR_BLOCKS;
        std::vector<T> ones(Q, T(0)), alt(Q, T(0));
        for (uint32_t q = 0; q < NQ; ++q) { ones[ct.cq_coords[q]] = T(1); alt[ct.cq_coords[q]] = (q & 1u) ? T(-1) : T(1); }
        probe1.assign(Q, T(0)); probe2.assign(Q, T(0));
        if (pair_blocks) closure_apply(ones, probe1);
        if (pair_blocks) closure_apply(alt, probe2);
        blk_m.assign(NBK, Blk{T(0), T(0), T(0)});
        blk_feat.assign(pair_blocks ? 16ull * NBK : 0ull, 0.0f);
        std::vector<T> blk_b(NBK, T(0));
        for (uint32_t blk = 0; pair_blocks && blk < NBK; ++blk) {
            const uint32_t qi = 2 * blk, qj = qi + 1;
            const bool pair = qj < NQ;
            const T a = dgl[ct.cq_coords[qi]], d = pair ? dgl[ct.cq_coords[qj]] : T(0);
            const T bij = pair ? closure_coupling(qi, qj) : T(0);
            Blk inv{a > T(1.0e-12f) ? T(1) / a : T(0), T(0), d > T(1.0e-12f) ? T(1) / d : T(0)};
            if (pair && a > T(1.0e-12f) && d > T(1.0e-12f)) {
                const T det = a * d - bij * bij;
                if (det > T(1.0e-6f) * (a * d)) inv = Blk{d / det, -bij / det, a / det};
            }
            blk_m[blk] = inv;
            blk_b[blk] = bij;
        }
        for (uint32_t blk = 0; pair_blocks && blk < NBK; ++blk) {
            float* f = &blk_feat[16ull * blk];
            f[15] = 1.0f;
            const uint32_t qi = 2 * blk, qj = qi + 1;
            const uint32_t ci = ct.cq_coords[qi];
            const bool pair = qj < NQ;
            const uint32_t cj = pair ? ct.cq_coords[qj] : ci;
            const T a = dgl[ci], d = pair ? dgl[cj] : T(0), bij = blk_b[blk];
            const uint32_t pb = blk ^ 1u;
            const bool partner = pb < NBK && 2 * pb + 1 < NQ;
            if (pair && partner && a > T(1.0e-12f) && d > T(1.0e-12f)) {
                const T pa = dgl[ct.cq_coords[2 * pb]], pd = dgl[ct.cq_coords[2 * pb + 1]];
                if (pa > T(1.0e-12f) && pd > T(1.0e-12f)) {
                    const T s1i = probe1[ci] - a - bij, ssi = probe2[ci] - a + bij;
                    const T s1j = probe1[cj] - bij - d, ssj = probe2[cj] - bij + d;
                    const T sa = std::sqrt(a), sd = std::sqrt(d), spa = std::sqrt(pa), spd = std::sqrt(pd);
                    f[0] = (float)(bij / (sa * sd)); f[1] = (float)(blk_b[pb] / (spa * spd));
                    f[2] = (float)(T(0.5f) * (s1i + ssi) / (sa * spa)); f[3] = (float)(T(0.5f) * (s1i - ssi) / (sa * spd));
                    f[4] = (float)(T(0.5f) * (s1j + ssj) / (sd * spa)); f[5] = (float)(T(0.5f) * (s1j - ssj) / (sd * spd));
                    f[6] = (float)tlog(a / d); f[7] = 1.0f;
                }
            }
        }
        if (precond == MK_PRECOND_BLOCK_JACOBI) {
            const uint32_t NL = (uint32_t)loop_off.size() - 1;
            loop_l.assign(36ull * NL, T(0));
            for (uint32_t lp = 0; lp < NL; ++lp) {
                const uint32_t o = loop_off[lp], n = loop_off[lp + 1] - o;
                T a[36];
                T mean = T(0);
                for (uint32_t i = 0; i < n; ++i) mean += dgl[ct.cq_coords[loop_q[o + i]]];
                mean = n ? mean / T(n) : T(0);
                for (uint32_t i = 0; i < n; ++i)
                    for (uint32_t j = 0; j <= i; ++j)
                        a[i * (i + 1) / 2 + j] = i == j ? dgl[ct.cq_coords[loop_q[o + i]]] + T(1.0e-6f) * mean
                                                        : closure_coupling(loop_q[o + i], loop_q[o + j]);
                bool ok = mean > T(1.0e-12f);
                for (uint32_t j = 0; j < n && ok; ++j) {
                    T dj = a[j * (j + 1) / 2 + j];
                    for (uint32_t k = 0; k < j; ++k) dj -= a[j * (j + 1) / 2 + k] * a[j * (j + 1) / 2 + k];
                    if (!(dj > T(0))) { ok = false; break; }
                    const T ljj = std::sqrt(dj);
                    a[j * (j + 1) / 2 + j] = ljj;
                    for (uint32_t i = j + 1; i < n; ++i) {
                        T v = a[i * (i + 1) / 2 + j];
                        for (uint32_t k = 0; k < j; ++k) v -= a[i * (i + 1) / 2 + k] * a[j * (j + 1) / 2 + k];
                        a[i * (i + 1) / 2 + j] = v / ljj;
                    }
                }
                T* l = &loop_l[36ull * lp];
                for (uint32_t i = 0; i < n; ++i)
                    for (uint32_t j = 0; j <= i; ++j) {
                        T v = a[i * (i + 1) / 2 + j];
                        if (!ok) {
                            const T dii = dgl[ct.cq_coords[loop_q[o + i]]];
                            v = (i == j) ? (dii > T(1.0e-12f) ? std::sqrt(dii) : T(0)) : T(0);
                        }
                        l[i * (i + 1) / 2 + j] = v;
                    }
            }
        }
        return unconverged;
    }
    void closure_pcg_step(uint32_t step) {
        const uint32_t NQ = (uint32_t)ct.cq_coords.size(), NBK = (NQ + 1) / 2;
        if (learned_precond) {
            for (uint32_t blk = 0; blk < NBK; ++blk) {
                const size_t o = 3ull * ((size_t)step * NBK + blk);
                const T t11 = o + 2 < precond_outputs.size() ? T(precond_outputs[o]) : T(0);
                const T t12 = o + 2 < precond_outputs.size() ? T(precond_outputs[o + 1]) : T(0);
                const T t22 = o + 2 < precond_outputs.size() ? T(precond_outputs[o + 2]) : T(0);
                const uint32_t qi = 2 * blk, qj = qi + 1;
                const uint32_t ci = ct.cq_coords[qi];
                const bool pair = qj < NQ;
                const T a = dgl[ci], d = pair ? dgl[ct.cq_coords[qj]] : T(0);
                if (pair) {
                    if (a > T(1.0e-12f) && d > T(1.0e-12f) && t11 > T(0) && t22 > T(0) &&
                        t11 * t22 - t12 * t12 > T(1.0e-6f) * (t11 * t22)) {
                        const T sa = std::sqrt(a), sd = std::sqrt(d);
                        blk_m[blk] = Blk{t11 / a, t12 / (sa * sd), t22 / d};
                        ++cstats.learned;
                    } else ++cstats.rejected;
                } else if (a > T(1.0e-12f) && t11 > T(0)) {
                    blk_m[blk] = Blk{t11 / a, T(0), T(0)};
                    ++cstats.learned;
                } else ++cstats.rejected;
            }
        }
        std::vector<T> sol(Q, T(0)), res(Q, T(0)), pre(Q, T(0)), dir(Q, T(0)), op(Q, T(0));
        auto precond = [&]() {
            if (this->precond == MK_PRECOND_DIAGONAL) {   // closure.wgsl:343-346, :396-400
                for (uint32_t q = 0; q < NQ; ++q) {
                    const uint32_t c = ct.cq_coords[q];
                    pre[c] = dgl[c] > T(1.0e-12f) ? res[c] / dgl[c] : T(0);
                }
                return;
            }
            if (this->precond == MK_PRECOND_BLOCK_JACOBI) {
                const uint32_t NL = (uint32_t)loop_off.size() - 1;
                for (uint32_t lp = 0; lp < NL; ++lp) {
                    const uint32_t o = loop_off[lp], n = loop_off[lp + 1] - o;
                    const T* l = &loop_l[36ull * lp];
                    T y[8];
                    for (uint32_t i = 0; i < n; ++i) {
                        T v = res[ct.cq_coords[loop_q[o + i]]];
                        for (uint32_t k = 0; k < i; ++k) v -= l[i * (i + 1) / 2 + k] * y[k];
                        const T lii = l[i * (i + 1) / 2 + i];
                        y[i] = lii > T(0) ? v / lii : T(0);
                    }
                    for (uint32_t ii = n; ii-- > 0;) {
                        T v = y[ii];
                        for (uint32_t k = ii + 1; k < n; ++k) v -= l[k * (k + 1) / 2 + ii] * y[k];
                        const T lii = l[ii * (ii + 1) / 2 + ii];
                        y[ii] = lii > T(0) ? v / lii : T(0);
                    }
                    for (uint32_t i = 0; i < n; ++i) pre[ct.cq_coords[loop_q[o + i]]] = y[i];
                }
                return;
            }
            for (uint32_t blk = 0; blk < NBK; ++blk) {
                const Blk& mi = blk_m[blk];
                const uint32_t qi = 2 * blk, qj = qi + 1;
                const uint32_t ci = ct.cq_coords[qi];
                if (qj < NQ) {
                    const uint32_t cj = ct.cq_coords[qj];
                    const T ri = res[ci], rj = res[cj];
                    pre[ci] = mi.m11 * ri + mi.m12 * rj;
                    pre[cj] = mi.m12 * ri + mi.m22 * rj;
                } else {
                    pre[ci] = mi.m11 * res[ci];
                }
            }
        };
        for (uint32_t q = 0; q < NQ; ++q) { const uint32_t c = ct.cq_coords[q]; sol[c] = T(0); res[c] = -grad[c]; }
        precond();
        for (uint32_t q = 0; q < NQ; ++q) { const uint32_t c = ct.cq_coords[q]; dir[c] = pre[c]; }
        auto cq = [&](uint32_t q) { return ct.cq_coords[q]; };
        double rz = closure_dot_d([&](uint32_t q) { return (double)res[cq(q)] * (double)pre[cq(q)]; });
        const double rr0 = closure_dot_d([&](uint32_t q) { return (double)res[cq(q)] * (double)res[cq(q)]; });
        double rr = rr0;
        const double tol2 = (double)closure_tol * (double)closure_tol;
        uint32_t it = 0;
        while (it < closure_max_it && rr > tol2 * rr0) {
            closure_apply(dir, op);
            const double pq = closure_dot_d([&](uint32_t q) { return (double)dir[cq(q)] * (double)op[cq(q)]; });
            const T alpha = std::fabs(pq) > 1.0e-30 ? T(rz / pq) : T(0);
            for (uint32_t q = 0; q < NQ; ++q) {
                const uint32_t c = cq(q);
                sol[c] += alpha * dir[c];
                res[c] -= alpha * op[c];
            }
            rr = closure_dot_d([&](uint32_t q) { return (double)res[cq(q)] * (double)res[cq(q)]; });
            ++it;
            if (rr <= tol2 * rr0) break;
            precond();
            const double nrz = closure_dot_d([&](uint32_t q) { return (double)res[cq(q)] * (double)pre[cq(q)]; });
            const T beta = std::fabs(rz) > 1.0e-300 ? T(nrz / rz) : T(0);
            for (uint32_t q = 0; q < NQ; ++q) { const uint32_t c = cq(q); dir[c] = pre[c] + beta * dir[c]; }
            rz = nrz;
        }
        cstats.pcg_iterations += it;
        const double rel = rr0 > 0.0 ? std::sqrt(rr / rr0) : 0.0;
        cstats.max_rel = std::max(cstats.max_rel, rel);
        for (uint32_t q = 0; q < NQ; ++q) {
            const uint32_t c = cq(q);
            T st = clampv(T(0.35f) * sol[c], T(-0.2f), T(0.2f));
            if (st == st) coords[c].x += st;
            else diag.error_flags |= MK_INVALID_NUMERIC_FLAG;
        }
    }
    void closure_loop_pcg() {
        build_closure_topology();
        cstats = ClosureStats{};
        for (uint32_t step = 0; step < 12; ++step) {
            std::fill(grad.begin(), grad.end(), T(0));
            std::fill(dgl.begin(), dgl.end(), T(0));
            if (!closure_eval_step()) break;
            ++cstats.newton_steps;
            closure_pcg_step(step);
            forward_kinematics();
        }
    }

    void mechanism_passes() {   // device.rs:963-1048
        for (uint32_t it = 0; it < std::max(1u, iterations); ++it) bearing_projection_iteration();
        advance_coordinates();
        forward_kinematics();
        if (closure_count > 0) {
            if (closure_mode == MK_CLOSURE_PCG_RESIDUAL) closure_loop_pcg();
            else closure_loop();
        }
        publish();
        reconstruct_body_velocities();
    }
    void post_contact_mechanism() {   // device.rs:1128-1155
        if (!has_dynamic_root)
            for (uint32_t it = 0; it < std::max(1u, iterations); ++it) bearing_projection_iteration();
        capture_coordinates();
        if (!has_dynamic_root) reconstruct_body_velocities();
    }
    void validate_bearings(bool use_links) {   // bearings.wgsl:48-102
        for (uint32_t j = 0; j < J; ++j) {
            const Bearing<T>& br = bear[j];
            uint32_t a = br.meta[0], b = br.meta[1];
            V4<T> pa, qa, pb, qb;
            if (use_links) {
                const std::vector<Link<T>>& L = links_final_const();
                pa = L[a].pos; qa = L[a].rot; pb = L[b].pos; qb = L[b].rot;
            } else {
                pa = pos[a]; qa = rot[a]; pb = pos[b]; qb = rot[b];
            }
            V3<T> anc_a = xyz(pa) + quat_rotate(qa, xyz(br.aa));
            V3<T> anc_b = xyz(pb) + quat_rotate(qb, xyz(br.ab));
            V3<T> axa = normalize(quat_rotate(qa, xyz(br.xa)));
            V3<T> axb = normalize(quat_rotate(qb, xyz(br.xb)));
            uint32_t um = round_u32(length(anc_a - anc_b) * T(1000000.0f));
            T deg = tatan2(length(cross(axa, axb)), clampv(dot(axa, axb), T(-1), T(1))) * T(57.295779513f);
            uint32_t ud = round_u32(deg * T(1000000.0f));
            diag.max_anchor_micrometers = std::max(diag.max_anchor_micrometers, um);
            diag.max_axis_microdegrees = std::max(diag.max_axis_microdegrees, ud);
            if (br.meta[3] != 0 && (um > 10u || ud > 1000u)) diag.error_flags |= MK_CONSTRAINT_NON_CONVERGENCE_FLAG;
        }
    }

    // serial contact Gauss-Seidel (collision.wgsl:908-1048), mechanisms with a
    // dynamic root and at most 64 bearings (device.rs:1370-1417)
    void solve_contact_immediate(uint32_t ci) {
        Contact<T>& c = contacts[ci];
        uint32_t a = c.meta[0], b = c.meta[1];
        V3<T> arm_a = xyz(c.aa), arm_b = xyz(c.ab);
        V3<T> vb = v3<T>(0, 0, 0);
        if (b != INVALID) vb = contact_velocity(b, arm_b);
        V3<T> n = xyz(c.np);
        T den = impulse_denominator(a, b, arm_a, arm_b, n);
        if (den <= T(0)) return;
        V3<T> rel = vb - contact_velocity(a, arm_a);
        T vn = dot(rel, n);
        if (c.np.w <= T(1.0e-5f) && vn >= T(-1.0e-5f) && c.aa.w <= T(1.0e-6f)) { c.aa.w = T(0); return; }
        T prev = mx(c.aa.w, T(0));
        T acc = mx(prev + (-vn + penetration_bias(c.np.w, c.ab.w < T(0))) / den, T(0));
        T delta = acc - prev;
        c.aa.w = acc;
        V3<T> imp = n * delta;
        V3<T> tv = rel - n * vn;
        T ts = length(tv);
        if (ts > T(1.0e-6f)) {
            V3<T> t = tv / ts;
            T tden = impulse_denominator(a, b, arm_a, arm_b, t);
            T fr = mn(ts / tden, std::fabs(delta) * T(0.05f));
            imp = imp - t * fr;
        }
        lin[a] = v4(xyz(lin[a]) - imp * wm[a].x.w, T(0));
        ang[a] = v4(xyz(ang[a]) + inverse_inertia(a, cross(arm_a, -imp)), T(0));
        if (b != INVALID) {
            lin[b] = v4(xyz(lin[b]) + imp * wm[b].x.w, T(0));
            ang[b] = v4(xyz(ang[b]) + inverse_inertia(b, cross(arm_b, imp)), T(0));
        }
    }
    void solve_serial_pass() {
        uint32_t A = (uint32_t)active.size();
        if (A > 64) {
            for (uint32_t k = 0; k < A; ++k) solve_contact_immediate(active[k]);
            for (uint32_t k = A; k > 0; --k) solve_contact_immediate(active[k - 1]);
            return;
        }
        std::vector<uint32_t> order(active.begin(), active.end());
        std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
            const Contact<T>& cx = contacts[x]; const Contact<T>& cy = contacts[y];
            if (cx.meta[0] != cy.meta[0]) return cx.meta[0] < cy.meta[0];
            if (cx.meta[1] != cy.meta[1]) return cx.meta[1] < cy.meta[1];
            return cx.meta[2] < cy.meta[2];
        });
        for (uint32_t k = 0; k < A; ++k) solve_contact_immediate(order[k]);
        for (uint32_t k = A; k > 0; --k) solve_contact_immediate(order[k - 1]);
    }

    bool mechanism_active() const { return max_depth > 0; }
    // device.rs:1370-1373; a batch of several scenes keeps the parallel form so that
    // one scene's path does not depend on the batch it is stepped in
    bool serial_mechanism() const { return mechanism_active() && has_dynamic_root && J <= 64 && !scene_bits; }

    // device.rs:1219-1431, with bearing projection interleaved when a
    // mechanism root is dynamic (:1363-1416)
    void collision_passes() {
        update_world_masses();
        compute_bounds();
        broadphase();
        narrowphase();
        ground_contacts();
        prepare_contacts();
        const bool interleave = mechanism_active() && has_dynamic_root;
        const bool serial = serial_mechanism();
        const uint32_t A = (uint32_t)active.size();
        if (contact_tol > 0.0f && !interleave) {
            solve_residual();
            persist();
            return;
        }
        // warm start + apply
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < (int64_t)A; ++k) solve_contact(active[k], true);
        if (A > 0) solve_apply();
        if (interleave) {
            if (serial) { if (A > 0) project_bearing_velocities_serial(); }
            else bearing_projection_iteration();
        }
        const uint32_t iters = serial ? std::max(1u, iterations) * 12u : std::max(1u, iterations);
        for (uint32_t it = 1; it < iters; ++it) {
            if (serial) {
                solve_serial_pass();
            } else {
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < (int64_t)A; ++k) solve_contact(active[k], false);
                if (A > 0) solve_apply();
            }
            if (interleave) {
                if (serial) { if (A > 0) project_bearing_velocities_serial(); }
                else bearing_projection_iteration();
            }
        }
        persist();
    }

    int step(uint64_t tick) override {
        diag = GpuDiagnostics{};
        tick32 = (uint32_t)tick;
        uint32_t slot = (uint32_t)(tick % 3);
        std::fill(deltas.begin(), deltas.end(), 0u);
        std::fill(mdeltas.begin(), mdeltas.end(), 0u);
        integrate();
        if (mechanism_active()) mechanism_passes();
        bool run_collisions = collisions && C > 0;
        if (run_collisions) collision_passes();
        if (mechanism_active() && run_collisions) post_contact_mechanism();
        if (mechanism_active()) validate_articulated_state();
        if (J > 0) validate_bearings(mechanism_active());
        snapshot(slot);
        return 0;
    }
};

}  // namespace orc

using namespace orc;

struct OrWorld {
    WorldBase* w = nullptr;
    World<float>* f = nullptr;
    World<double>* d = nullptr;
};

template <class T>
static World<T>* build_world(const MkCreation* cr, const MkConfig* cfg, uint32_t pair_capacity) {
    World<T>* w = new World<T>();
    w->precision = sizeof(T) == 4 ? 32 : 64;
    w->B = cr->body_count; w->C = cr->collider_count; w->J = cr->bearing_count;
    w->S = cr->suppression_count; w->Q = cr->coordinate_count; w->max_depth = cr->max_depth;
    w->closure_count = cr->closure_count; w->has_dynamic_root = cr->has_dynamic_root;
    MkConfig c;
    if (cfg) c = *cfg; else { std::memset(&c, 0, sizeof(c)); c.collisions_enabled = 1; c.mechanism_self_collisions = 1; c.solver_iterations = 8; }
    w->dt = T(c.delta_seconds != 0.0f ? c.delta_seconds : 1.0f / 60.0f);
    w->gravity = T(c.gravity_y != 0.0f ? c.gravity_y : -9.81f);
    w->lin_damp = T(c.linear_damping != 0.0f ? c.linear_damping : 0.999f);
    w->ang_damp = T(c.angular_damping != 0.0f ? c.angular_damping : 0.98f);
    w->iterations = c.solver_iterations ? c.solver_iterations : 8;
    w->morton_mode = c.morton_mode;
    w->collisions = c.collisions_enabled;
    w->self_collisions = c.mechanism_self_collisions;
    w->pair_capacity = pair_capacity ? pair_capacity : MK_DEFAULT_MAX_CONTACT_PAIRS;
    w->contact_tol = c.contact_tolerance > 0.0f ? c.contact_tolerance : 0.0f;
    w->clipped = c.contact_manifold == MK_MANIFOLD_CLIPPED ? 1u : 0u;
    w->contact_max_it = c.contact_max_iterations ? c.contact_max_iterations : 512u;
    w->closure_mode = c.closure_mode;
    w->closure_tol = c.closure_tolerance > 0.0f ? c.closure_tolerance : 1.0e-5f;
    w->closure_max_it = c.closure_max_iterations ? c.closure_max_iterations : 256u;
    w->learned_precond = (c.closure_mode == MK_CLOSURE_PCG_RESIDUAL && c.preconditioner == MK_PRECOND_LEARNED) ? 1u : 0u;
    w->precond = c.preconditioner;
    uint32_t B = w->B, C = w->C;
    w->pos.resize(B); w->rot.resize(B); w->lin.resize(B); w->ang.resize(B);
    w->inv_mass.resize(B); w->mass.resize(B); w->root.resize(B); w->components.resize(B);
    for (uint32_t i = 0; i < B; ++i) {
        w->pos[i] = load4<T>(cr->transforms[i].position);
        w->rot[i] = load4<T>(cr->transforms[i].rotation);
        if (cr->velocities) {
            w->lin[i] = load4<T>(cr->velocities[i].linear);
            w->ang[i] = load4<T>(cr->velocities[i].angular);
        } else {
            w->lin[i] = {0, 0, 0, 0}; w->ang[i] = {0, 0, 0, 0};
        }
        const GpuMass& m = cr->masses[i];
        w->inv_mass[i] = T(m.inverse_mass[0]);
        w->mass[i].inv_mass = T(m.inverse_mass[0]);
        w->mass[i].ix = xyz(load4<T>(m.inverse_inertia_x));
        w->mass[i].iy = xyz(load4<T>(m.inverse_inertia_y));
        w->mass[i].iz = xyz(load4<T>(m.inverse_inertia_z));
        w->root[i] = cr->root_flags ? cr->root_flags[i] : 1u;
        w->components[i] = cr->body_components ? cr->body_components[i] : i;
    }
    w->col.resize(C);
    for (uint32_t i = 0; i < C; ++i) {
        const GpuCollider& g = cr->colliders[i];
        w->col[i].center = load4<T>(g.local_center);
        w->col[i].rot = load4<T>(g.local_rotation);
        w->col[i].half = load4<T>(g.half_extents);
        for (int k = 0; k < 4; ++k) w->col[i].meta[k] = g.metadata[k];
    }
    w->sup.resize(2 * (size_t)w->S);
    for (uint32_t i = 0; i < w->S; ++i) {
        w->sup[2 * i] = cr->suppressed_pairs[i].collider_a;
        w->sup[2 * i + 1] = cr->suppressed_pairs[i].collider_b;
    }
    w->wm.resize(B);
    w->deltas.assign(6 * (size_t)B, 0u);
    w->aabb_min.resize(C); w->aabb_max.resize(C);
    w->keys.resize(C); w->skeys.resize(C); w->svals.resize(C);
    for (int s = 0; s < 3; ++s) { w->snap_pos[s] = w->pos; w->snap_rot[s] = w->rot; }
    w->coords.assign(w->Q, V4<T>{0, 0, 0, 0});
    uint32_t J = w->J;
    w->bear.resize(J);
    for (uint32_t j = 0; j < J; ++j) {
        const GpuBearing& g = cr->bearings[j];
        w->bear[j].aa = load4<T>(g.local_anchor_a); w->bear[j].ab = load4<T>(g.local_anchor_b);
        w->bear[j].xa = load4<T>(g.local_axis_a); w->bear[j].xb = load4<T>(g.local_axis_b);
        for (int k = 0; k < 4; ++k) w->bear[j].meta[k] = g.metadata[k];
    }
    w->mech.resize(B);
    w->preorder.resize(B);
    for (uint32_t i = 0; i < B; ++i) {
        if (cr->mechanism_bodies) {
            const GpuMechanismBody& g = cr->mechanism_bodies[i];
            for (int k = 0; k < 4; ++k) { w->mech[i].meta[k] = g.metadata[k]; w->mech[i].trav[k] = g.traversal[k]; }
            w->mech[i].bpos = load4<T>(g.bind_relative_position);
            w->mech[i].brot = load4<T>(g.bind_relative_rotation);
        } else {
            w->mech[i].meta[0] = i; w->mech[i].meta[1] = INVALID; w->mech[i].meta[2] = 0; w->mech[i].meta[3] = 1;
            for (int k = 0; k < 4; ++k) w->mech[i].trav[k] = 0;
            w->mech[i].bpos = {0, 0, 0, 0}; w->mech[i].brot = {0, 0, 0, 1};
        }
        w->preorder[i] = cr->preorder ? cr->preorder[i] : i;
    }
    w->drives.resize(w->Q);
    for (uint32_t c = 0; c < w->Q; ++c) {
        Drive d{};
        if (cr->drives) {
            const GpuMechanismDrive& g = cr->drives[c];
            d.mode = g.mode; d.max_acc = g.max_acceleration; d.max_speed = g.max_speed;
            d.target_speed = g.target_speed; d.target_angle = g.target_angle;
            d.min_angle = g.min_angle; d.max_angle = g.max_angle;
        } else {
            d.mode = MK_DRIVE_MODE_PASSIVE; d.min_angle = -INFINITY; d.max_angle = INFINITY;
        }
        w->drives[c] = d;
    }
    uint32_t covered = 1, rounds = 0;
    while (covered < w->max_depth) { covered *= 2; ++rounds; }
    if (w->max_depth > 0 && rounds == 0) rounds = 1;
    w->jump_rounds = rounds;
    w->final_is_a = rounds % 2 == 0;
    w->links_a.assign(B, Link<T>{});
    w->links_b.assign(B, Link<T>{});
    w->mdeltas.assign(6 * (size_t)B, 0u);
    w->grad.assign(w->Q, T(0));
    w->dgl.assign(w->Q, T(0));
    w->pcg.assign(w->Q, typename World<T>::Pcg{});
    return w;
}

template <class T> static void put4(float* d, const V4<T>& v) { d[0] = float(v.x); d[1] = float(v.y); d[2] = float(v.z); d[3] = float(v.w); }
template <class T> static void put4d(double* d, const V4<T>& v) { d[0] = double(v.x); d[1] = double(v.y); d[2] = double(v.z); d[3] = double(v.w); }

extern "C" {

OrWorld* or_create(const MkCreation* creation, const MkConfig* config, int precision, uint32_t pair_capacity) {
    if (!creation) return nullptr;
    OrWorld* o = new OrWorld();
    if (precision == 64) { o->d = build_world<double>(creation, config, pair_capacity); o->w = o->d; }
    else { o->f = build_world<float>(creation, config, pair_capacity); o->w = o->f; }
    return o;
}

void or_destroy(OrWorld* o) {
    if (!o) return;
    delete o->w;
    delete o;
}

void or_set_threads(int threads) {
    g_threads = threads;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int or_step(OrWorld* o, uint64_t tick) { return o->w->step(tick); }

#define DISPATCH(expr_f, expr_d) do { if (o->f) { auto* w = o->f; expr_f; } else { auto* w = o->d; expr_d; } } while (0)
#define BOTH(...) do { if (o->f) { auto* w = o->f; __VA_ARGS__; } else { auto* w = o->d; __VA_ARGS__; } } while (0)

uint64_t or_count(const OrWorld* o, int what) {
    uint64_t r = 0;
    BOTH({
        switch (what) {
            case OR_COUNT_PAIRS: r = w->pairs.size() / 2; break;
            case OR_COUNT_CONTACTS: r = w->contacts.size(); break;
            case OR_COUNT_ACTIVE: r = w->active.size(); break;
            case OR_COUNT_BODIES: r = w->B; break;
            case OR_COUNT_COLLIDERS: r = w->C; break;
            case OR_COUNT_MANIFOLD: {
                uint64_t n = 0;
                for (auto& kv : w->manifold) if (kv.second.tick == w->last_tick) ++n;
                r = n; break;
            }
            case OR_COUNT_COORDINATES: r = w->Q; break;
            case OR_COUNT_BEARINGS: r = w->J; break;
        }
    });
    return r;
}


void or_get_state(const OrWorld* o, GpuTransform* tr, GpuVelocity* vel) {
    BOTH({
        for (uint32_t i = 0; i < w->B; ++i) {
            if (tr) { put4(tr[i].position, w->pos[i]); put4(tr[i].rotation, w->rot[i]); }
            if (vel) { put4(vel[i].linear, w->lin[i]); put4(vel[i].angular, w->ang[i]); }
        }
    });
}

void or_get_state_f64(const OrWorld* o, double* p, double* r, double* l, double* a) {
    BOTH({
        for (uint32_t i = 0; i < w->B; ++i) {
            if (p) put4d(p + 4 * i, w->pos[i]);
            if (r) put4d(r + 4 * i, w->rot[i]);
            if (l) put4d(l + 4 * i, w->lin[i]);
            if (a) put4d(a + 4 * i, w->ang[i]);
        }
    });
}

void or_set_state(OrWorld* o, const GpuTransform* tr, const GpuVelocity* vel) {
    DISPATCH({
        for (uint32_t i = 0; i < w->B; ++i) {
            if (tr) { w->pos[i] = load4<float>(tr[i].position); w->rot[i] = load4<float>(tr[i].rotation); }
            if (vel) { w->lin[i] = load4<float>(vel[i].linear); w->ang[i] = load4<float>(vel[i].angular); }
        }
    }, {
        for (uint32_t i = 0; i < w->B; ++i) {
            if (tr) { w->pos[i] = load4<double>(tr[i].position); w->rot[i] = load4<double>(tr[i].rotation); }
            if (vel) { w->lin[i] = load4<double>(vel[i].linear); w->ang[i] = load4<double>(vel[i].angular); }
        }
    });
}

void or_get_diagnostics(const OrWorld* o, GpuDiagnostics* out) { BOTH(*out = w->diag); }
// Residual-mode solve outcome of the last step: iterations, chosen, converged, s0, sk.
void or_get_solve_stats(const OrWorld* o, uint32_t* u3, double* d2) {
    BOTH((u3[0] = w->stats.iterations, u3[1] = w->stats.chosen, u3[2] = w->stats.converged,
          d2[0] = w->stats.s0, d2[1] = w->stats.sk));
}
// Closure PCG outcome of the last step: newton steps, pcg iterations, learned, rejected blocks; max rel residual.
void or_get_closure_stats(const OrWorld* o, uint32_t* u4, double* d1) {
    BOTH((u4[0] = w->cstats.newton_steps, u4[1] = w->cstats.pcg_iterations, u4[2] = w->cstats.learned,
          u4[3] = w->cstats.rejected, d1[0] = w->cstats.max_rel));
}
// Preconditioner network outputs (12 x blocks x 3) for the next step.
void or_set_precond_outputs(OrWorld* o, const float* out, uint32_t n) {
    BOTH(w->precond_outputs.assign(out, out + n));
}
// Block inputs of the last evaluated Newton step (blocks x 16).
uint32_t or_get_closure_blocks(const OrWorld* o, float* out) {
    uint32_t n = 0;
    BOTH((n = (uint32_t)w->blk_feat.size() / 16, out ? (void)std::copy(w->blk_feat.begin(), w->blk_feat.end(), out) : (void)0));
    return n;
}
// Batched scenes: the scene of each collider (scene indices ascending with the collider index).
void or_set_batch(OrWorld* o, const uint32_t* collider_scene, uint32_t scene_count) {
    uint32_t bits = 0;
    while ((1u << bits) < scene_count) ++bits;
    BOTH((w->col_scene.assign(collider_scene, collider_scene + w->C), w->scene_bits = scene_count > 1 ? bits : 0u));
}
// Learned warm-start impulses (by active position) for the next step's solve.
void or_set_warm_predictions(OrWorld* o, const float* pred, uint32_t n) {
    BOTH((w->warm_predictions.assign(pred, pred + n), w->learned_pending = true));
}

void or_get_pairs(const OrWorld* o, GpuPair* out) {
    BOTH({ for (size_t p = 0; p < w->pairs.size() / 2; ++p) { out[p].collider_a = w->pairs[2 * p]; out[p].collider_b = w->pairs[2 * p + 1]; } });
}

void or_get_contacts(const OrWorld* o, GpuContact* out) {
    BOTH({
        for (size_t k = 0; k < w->contacts.size(); ++k) {
            const auto& c = w->contacts[k];
            for (int j = 0; j < 4; ++j) out[k].metadata[j] = c.meta[j];
            put4(out[k].normal_penetration, c.np); put4(out[k].arm_a_impulse, c.aa); put4(out[k].arm_b, c.ab);
        }
    });
}

void or_get_contacts_f64(const OrWorld* o, double* rows) {
    BOTH({
        for (size_t k = 0; k < w->contacts.size(); ++k) {
            const auto& c = w->contacts[k];
            for (int j = 0; j < 4; ++j) rows[16 * k + j] = double(c.meta[j]);
            put4d(rows + 16 * k + 4, c.np); put4d(rows + 16 * k + 8, c.aa); put4d(rows + 16 * k + 12, c.ab);
        }
    });
}

void or_get_contact_keys(const OrWorld* o, uint64_t* out) { BOTH(std::copy(w->contact_keys.begin(), w->contact_keys.end(), out)); }
void or_get_features(const OrWorld* o, uint32_t* out) { BOTH(std::copy(w->features.begin(), w->features.end(), out)); }
void or_get_active(const OrWorld* o, uint32_t* out) { BOTH(std::copy(w->active.begin(), w->active.end(), out)); }
void or_get_collider_keys(const OrWorld* o, uint64_t* out) { BOTH(std::copy(w->keys.begin(), w->keys.end(), out)); }

void or_get_sorted(const OrWorld* o, uint64_t* keys, uint32_t* values) {
    BOTH({
        if (keys) std::copy(w->skeys.begin(), w->skeys.end(), keys);
        if (values) std::copy(w->svals.begin(), w->svals.end(), values);
    });
}

void or_get_aabbs(const OrWorld* o, float* out8) {
    BOTH({ for (uint32_t i = 0; i < w->C; ++i) { put4(out8 + 8 * i, w->aabb_min[i]); put4(out8 + 8 * i + 4, w->aabb_max[i]); } });
}

void or_get_world_masses(const OrWorld* o, float* out12) {
    BOTH({ for (uint32_t i = 0; i < w->B; ++i) { put4(out12 + 12 * i, w->wm[i].x); put4(out12 + 12 * i + 4, w->wm[i].y); put4(out12 + 12 * i + 8, w->wm[i].z); } });
}

void or_get_snapshot(const OrWorld* o, uint32_t slot, GpuTransform* out) {
    if (slot > 2) return;
    BOTH({ for (uint32_t i = 0; i < w->B; ++i) { put4(out[i].position, w->snap_pos[slot][i]); put4(out[i].rotation, w->snap_rot[slot][i]); } });
}

void or_get_coordinates(const OrWorld* o, GpuMechanismCoordinate* out) {
    BOTH({ for (uint32_t i = 0; i < w->Q; ++i) { out[i].angle = float(w->coords[i].x); out[i].angular_velocity = float(w->coords[i].y); } });
}

void or_set_coordinates(OrWorld* o, const GpuMechanismCoordinate* in) {
    BOTH({ for (uint32_t i = 0; i < w->Q; ++i) { w->coords[i].x = in[i].angle; w->coords[i].y = in[i].angular_velocity; } });
}

void or_get_links(const OrWorld* o, GpuLinkState* out) {
    BOTH({
        const auto& L = w->links_final_const();
        for (size_t i = 0; i < L.size(); ++i) {
            put4(out[i].position, L[i].pos); put4(out[i].rotation, L[i].rot);
            for (int k = 0; k < 4; ++k) out[i].metadata[k] = L[i].meta[k];
        }
    });
}

uint32_t or_get_manifold(const OrWorld* o, GpuContact* out, uint32_t capacity) {
    uint32_t n = 0;
    BOTH({
        std::vector<uint64_t> ks;
        for (auto& kv : w->manifold) if (kv.second.tick == w->last_tick) ks.push_back(kv.first);
        std::sort(ks.begin(), ks.end());
        for (uint64_t k : ks) {
            if (n >= capacity) break;
            const auto& m = w->manifold.at(k);
            GpuContact& c = out[n++];
            c.metadata[0] = 0; c.metadata[1] = 0; c.metadata[2] = (uint32_t)(k >> 32); c.metadata[3] = (uint32_t)k;
            put4(c.normal_penetration, m.np); put4(c.arm_a_impulse, m.pi);
            c.arm_b[0] = c.arm_b[1] = c.arm_b[2] = c.arm_b[3] = 0.0f;
        }
    });
    return n;
}

void or_set_manifold(OrWorld* o, const GpuContact* rows, uint32_t count, uint64_t last_tick) {
    DISPATCH({
        w->manifold.clear();
        for (uint32_t i = 0; i < count; ++i) {
            Manifold<float> m; m.tick = (uint32_t)last_tick; m.count = 1;
            m.np = load4<float>(rows[i].normal_penetration); m.pi = load4<float>(rows[i].arm_a_impulse);
            w->manifold[((uint64_t)rows[i].metadata[2] << 32) | rows[i].metadata[3]] = m;
        }
        w->last_tick = (uint32_t)last_tick;
    }, {
        w->manifold.clear();
        for (uint32_t i = 0; i < count; ++i) {
            Manifold<double> m; m.tick = (uint32_t)last_tick; m.count = 1;
            m.np = load4<double>(rows[i].normal_penetration); m.pi = load4<double>(rows[i].arm_a_impulse);
            w->manifold[((uint64_t)rows[i].metadata[2] << 32) | rows[i].metadata[3]] = m;
        }
        w->last_tick = (uint32_t)last_tick;
    });
}

// lbvh.wgsl:219-278 over (key, value) entries.
static int common_prefix(const uint64_t* k, const uint32_t* v, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    uint64_t d = k[i] ^ k[j];
    if (d != 0) return __builtin_clzll(d);
    uint32_t e = v[i] ^ v[j];
    return 64 + (e ? __builtin_clz(e) : 32);
}

void or_get_karras(const OrWorld* o, uint32_t* children) {
    BOTH({
        const uint64_t* k = w->skeys.data();
        const uint32_t* v = w->svals.data();
        int64_t n = w->C;
        for (int64_t i = 0; i + 1 < n; ++i) {
            int dir = common_prefix(k, v, n, i, i + 1) > common_prefix(k, v, n, i, i - 1) ? 1 : -1;
            int min_prefix = common_prefix(k, v, n, i, i - dir);
            int64_t max_len = 2;
            while (common_prefix(k, v, n, i, i + max_len * dir) > min_prefix) max_len *= 2;
            int64_t len = 0;
            for (int64_t step = max_len / 2; step >= 1; step /= 2)
                if (common_prefix(k, v, n, i, i + (len + step) * dir) > min_prefix) len += step;
            int64_t other = i + len * dir;
            int node_prefix = common_prefix(k, v, n, i, other);
            int64_t split_off = 0;
            int64_t step = (len + 1) / 2;
            while (step >= 1) {
                if (common_prefix(k, v, n, i, i + (split_off + step) * dir) > node_prefix) split_off += step;
                if (step == 1) break;
                step = (step + 1) / 2;
            }
            int64_t split = i + split_off * dir + std::min(dir, 0);
            int64_t first = std::min(i, other), last = std::max(i, other);
            uint32_t leaf_base = (uint32_t)(n - 1);
            children[2 * i] = split == first ? leaf_base + (uint32_t)split : (uint32_t)split;
            children[2 * i + 1] = split + 1 == last ? leaf_base + (uint32_t)(split + 1) : (uint32_t)(split + 1);
        }
    });
}

static Obb<float> box_from(const float* b) {
    Obb<float> o;
    o.c = v3<float>(b[0], b[1], b[2]);
    o.h = v3<float>(b[3], b[7], b[11]);
    o.ax[0] = v3<float>(b[4], b[5], b[6]);
    o.ax[1] = v3<float>(b[8], b[9], b[10]);
    o.ax[2] = v3<float>(b[12], b[13], b[14]);
    return o;
}

uint32_t or_obb_sat_f32(const float* box_a, const float* box_b, float* np) {
    Obb<float> a = box_from(box_a), b = box_from(box_b);
    Sat<float> s = World<float>::obb_sat(a, b);
    np[0] = s.normal.x; np[1] = s.normal.y; np[2] = s.normal.z; np[3] = s.pen;
    return s.axis | (s.near << 8) | (s.early << 16);
}

void or_contact_point_f32(const float* box_a, const float* box_b, const float* n, float* p3) {
    Obb<float> a = box_from(box_a), b = box_from(box_b);
    World<float> tmp;
    V3<float> p = tmp.contact_point(a, V4<float>{0, 0, 0, 1}, b, V4<float>{0, 0, 0, 1}, v3<float>(n[0], n[1], n[2]), true);
    p3[0] = p.x; p3[1] = p.y; p3[2] = p.z;
}

// collision.rs:43-183 (CPU reference narrowphase; glam operation order is
// approximated with the same vector helpers).
static Obb<float> cpu_obb(const float* c, const float* q, const float* h) {
    Obb<float> o;
    V4<float> r = {q[0], q[1], q[2], q[3]};
    o.c = v3<float>(c[0], c[1], c[2]);
    o.h = v3<float>(h[0], h[1], h[2]);
    o.ax[0] = quat_rotate(r, v3<float>(1, 0, 0));
    o.ax[1] = quat_rotate(r, v3<float>(0, 1, 0));
    o.ax[2] = quat_rotate(r, v3<float>(0, 0, 1));
    return o;
}

static bool cpu_sat(const Obb<float>& a, const Obb<float>& b, V3<float>& normal, float& pen) {
    V3<float> delta = b.c - a.c;
    normal = v3<float>(1, 0, 0);
    pen = INFINITY;
    auto test = [&](V3<float> axis) -> bool {
        float ra = World<float>::projection_radius(a.ax, a.h, axis);
        float rb = World<float>::projection_radius(b.ax, b.h, axis);
        float sd = dot(delta, axis);
        float p = ra + rb - std::fabs(sd);
        if (p < -1.0e-6f) return false;
        if (p < pen) { pen = mx(p, 0.0f); normal = sd < 0.0f ? -axis : axis; }
        return true;
    };
    for (int i = 0; i < 3; ++i) if (!test(a.ax[i])) return false;
    for (int i = 0; i < 3; ++i) if (!test(b.ax[i])) return false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            V3<float> c = cross(a.ax[i], b.ax[j]);
            if (dot(c, c) > 1.0e-10f)
                if (!test(normalize(c))) return false;
        }
    return true;
}

int or_cpu_obb_sat(const float* ca, const float* qa, const float* ha, const float* cb, const float* qb,
                   const float* hb, float* np) {
    Obb<float> a = cpu_obb(ca, qa, ha), b = cpu_obb(cb, qb, hb);
    V3<float> n; float p;
    if (!cpu_sat(a, b, n, p)) return 0;
    np[0] = n.x; np[1] = n.y; np[2] = n.z; np[3] = p;
    return 1;
}

int or_cpu_contact_manifold(const float* ca, const float* qa, const float* ha, const float* cb, const float* qb,
                            const float* hb, float* np, float* points) {
    Obb<float> a = cpu_obb(ca, qa, ha), b = cpu_obb(cb, qb, hb);
    V3<float> n; float p;
    if (!cpu_sat(a, b, n, p)) return 0;
    auto verts = [](const Obb<float>& o, V3<float>* out) {
        V3<float> x = o.ax[0] * o.h.x, y = o.ax[1] * o.h.y, z = o.ax[2] * o.h.z;
        int k = 0;
        for (int sx = -1; sx <= 1; sx += 2)
            for (int sy = -1; sy <= 1; sy += 2)
                for (int sz = -1; sz <= 1; sz += 2)
                    out[k++] = o.c + x * float(sx) + y * float(sy) + z * float(sz);
    };
    auto contains = [](const Obb<float>& o, V3<float> pt) {
        V3<float> d = pt - o.c;
        return std::fabs(dot(o.ax[0], d)) <= o.h.x + 1.0e-5f && std::fabs(dot(o.ax[1], d)) <= o.h.y + 1.0e-5f &&
               std::fabs(dot(o.ax[2], d)) <= o.h.z + 1.0e-5f;
    };
    std::vector<V3<float>> cand;
    auto push_unique = [&](V3<float> c) {
        for (auto& q : cand) { V3<float> d = q - c; if (!(dot(d, d) > 1.0e-10f)) return; }
        cand.push_back(c);
    };
    V3<float> va[8], vb[8];
    verts(a, va); verts(b, vb);
    for (auto& v : va) if (contains(b, v)) push_unique(v);
    for (auto& v : vb) if (contains(a, v)) push_unique(v);
    if (cand.empty()) {
        auto support = [](const Obb<float>& o, V3<float> dir) {
            V3<float> pt = o.c;
            const float he[3] = {o.h.x, o.h.y, o.h.z};
            for (int k = 0; k < 3; ++k) {
                float s = dot(o.ax[k], dir);
                float sg = s > 0.0f ? 1.0f : (s < 0.0f ? -1.0f : (std::signbit(s) ? -1.0f : 1.0f));
                pt = pt + o.ax[k] * he[k] * sg;
            }
            return pt;
        };
        cand.push_back((support(a, n) + support(b, -n)) * 0.5f);
    }
    std::sort(cand.begin(), cand.end(), [](const V3<float>& l, const V3<float>& r) {
        if (l.x != r.x) return l.x < r.x;
        if (l.y != r.y) return l.y < r.y;
        return l.z < r.z;
    });
    if (cand.size() > 4) cand.resize(4);
    np[0] = n.x; np[1] = n.y; np[2] = n.z; np[3] = p;
    for (size_t i = 0; i < cand.size(); ++i) { points[3 * i] = cand[i].x; points[3 * i + 1] = cand[i].y; points[3 * i + 2] = cand[i].z; }
    return (int)cand.size();
}

uint32_t or_morton30(float x, float y, float z) { return World<float>::morton30(v3<float>(x, y, z)); }
uint64_t or_morton63(float x, float y, float z, float lx, float ly, float lz, float scale) {
    return World<float>::morton_frame(v3<float>(x, y, z), v3<float>(lx, ly, lz), scale, 2097151.0f);
}
uint64_t or_morton48(float x, float y, float z, float lx, float ly, float lz, float scale) {
    return World<float>::morton_frame(v3<float>(x, y, z), v3<float>(lx, ly, lz), scale, 65535.0f);
}
uint64_t or_morton39(float x, float y, float z, float lx, float ly, float lz, float scale) {
    return World<float>::morton_frame(v3<float>(x, y, z), v3<float>(lx, ly, lz), scale, 8191.0f);
}
uint64_t or_morton30a(float x, float y, float z, float lx, float ly, float lz, float scale) {
    return World<float>::morton_frame(v3<float>(x, y, z), v3<float>(lx, ly, lz), scale, 1023.0f);
}

}  // extern "C"
