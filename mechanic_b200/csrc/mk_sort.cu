// mk_sort.cu — stable LSD onesweep radix sort of (63-bit key, 32-bit value).
//
// Replaces the reference's bitonic network (lbvh.wgsl:132-217, 54-77
// full-buffer passes per tick) with one histogram pass over the keys plus one
// single-pass "onesweep" scatter per 8-bit digit: each tile ranks its keys
// with warp match-any, publishes per-digit counts, and learns its global
// offsets by decoupled look-back over the preceding tiles.  Stability
// (equal keys keep input order) gives the reference's (code, index)
// tie-break when the values are collider indices in ascending order.
#include "mk_device.cuh"
#include "mk_internal.h"

namespace mk {

constexpr uint32_t kSortThreads = 256;
constexpr uint32_t kRadixBins = 256;
constexpr uint32_t kLookbackWindow = 16;   // predecessor tiles read per look-back round trip

// 30-bit digit look-back words: bits 30-31 status, 0-29 count.
constexpr uint32_t kDigitAggregate = 1u << 30;
constexpr uint32_t kDigitInclusive = 2u << 30;
constexpr uint32_t kDigitCountMask = (1u << 30) - 1;

__global__ void __launch_bounds__(kSortThreads)
k_radix_histogram(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ n_ptr, uint32_t n_fixed,
                  uint32_t passes, uint32_t* __restrict__ hist /* passes x 256 */,
                  uint32_t* __restrict__ lookback, uint64_t lookback_pass_words, uint32_t tile_keys) {
    __shared__ uint32_t s_hist[8][kRadixBins];
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;   // a device count never exceeds the capacity
    // clear the look-back words the onesweep passes will use for this n only
    const uint64_t used = (uint64_t)((n + tile_keys - 1) / tile_keys) * kRadixBins;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < used * passes;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pass = w / used, off = w % used;
        lookback[pass * lookback_pass_words + off] = 0u;
    }
    for (uint32_t i = threadIdx.x; i < 8 * kRadixBins; i += blockDim.x) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&s_hist[p][(k >> (8 * p)) & 0xffu], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * kRadixBins; i += blockDim.x) {
        uint32_t v = (&s_hist[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <uint32_t kSortItems>
__global__ void __launch_bounds__(kSortThreads)
k_radix_onesweep(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                 uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                 const uint32_t* __restrict__ n_ptr, uint32_t n_fixed, uint32_t shift,
                 const uint32_t* __restrict__ digit_hist /* 256 */, uint32_t* __restrict__ lookback,
                 uint32_t* __restrict__ ticket, uint32_t* __restrict__ error_flags) {
    constexpr uint32_t kTile = kSortThreads * kSortItems;
    __shared__ uint64_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_warp[kSortThreads / 32][kRadixBins];
    __shared__ uint32_t s_local_start[kRadixBins];
    __shared__ uint32_t s_global_base[kRadixBins];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_digit_offsets[kRadixBins];

    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;   // a device count never exceeds the capacity
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t lane = lane_id(), w = warp_id();
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);   // in flight during the offsets scan
    {   // this pass's digit offsets: exclusive scan of its histogram (kSortThreads == kRadixBins)
        uint32_t total_all;
        s_digit_offsets[threadIdx.x] = block_exclusive_scan(digit_hist[threadIdx.x], s_scan, &total_all);
    }

    for (;;) {
        for (uint32_t i = threadIdx.x; i < (kSortThreads / 32) * kRadixBins; i += kSortThreads)
            (&s_warp[0][0])[i] = 0;
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= tiles) break;
        const uint32_t tile_base = tile * kTile;

        // ---- load every item first (one memory round trip), then rank within
        // each warp, item by item (warp-striped)
        uint64_t k[kSortItems];
        uint32_t v[kSortItems];
        uint32_t rank[kSortItems];
        uint32_t dig[kSortItems];
#pragma unroll
        for (uint32_t i = 0; i < kSortItems; ++i) {
            const uint32_t idx = tile_base + w * 32 * kSortItems + i * 32 + lane;
            const bool valid = idx < n;
            k[i] = valid ? __ldcg(keys_in + idx) : 0ull;
            v[i] = (valid && vals_in) ? __ldcg(vals_in + idx) : 0u;
        }
#pragma unroll
        for (uint32_t i = 0; i < kSortItems; ++i) {
            const uint32_t idx = tile_base + w * 32 * kSortItems + i * 32 + lane;
            const bool valid = idx < n;
            uint32_t d = valid ? (uint32_t)((k[i] >> shift) & 0xffu) : kRadixBins;
            dig[i] = d;
            uint32_t peers = __match_any_sync(0xffffffffu, d);
            uint32_t leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (lane == leader && valid) base = s_warp[w][d];
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[i] = base + __popc(peers & lanemask_lt());
            if (lane == leader && valid) s_warp[w][d] = base + __popc(peers);
            __syncwarp();
        }
        __syncthreads();

        // ---- per digit: prefix over warps, tile count, tile-local start
        const uint32_t d = threadIdx.x;   // kSortThreads == kRadixBins
        uint32_t count = 0;
#pragma unroll
        for (uint32_t ww = 0; ww < kSortThreads / 32; ++ww) {
            uint32_t c = s_warp[ww][d];
            s_warp[ww][d] = count;
            count += c;
        }
        uint32_t total;
        uint32_t local_start = block_exclusive_scan(count, s_scan, &total);
        s_local_start[d] = local_start;

        // ---- decoupled look-back for digit d (one thread per digit), reading a
        // window of kLookbackWindow predecessors per round trip: with every tile
        // starting at once, a one-word walk advances the inclusive prefixes by
        // about two tiles per L2 round trip, a window by kLookbackWindow + 1
        uint32_t* lb = lookback + (size_t)tile * kRadixBins + d;
        uint32_t prefix = 0;
        // (relaxed stores: a word carries its own status and count, and a
        // release store's fence costs about an L2 round trip per tile)
        if (tile == 0) {
            st_relaxed_u32(lb, kDigitInclusive | count);
        } else {
            st_relaxed_u32(lb, kDigitAggregate | count);
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            for (;;) {
                uint32_t s[kLookbackWindow];
#pragma unroll
                for (uint32_t j = 0; j < kLookbackWindow; ++j)   // below tile 0: an inclusive 0
                    s[j] = t >= (int64_t)j ? ld_relaxed_u32(lookback + (size_t)(t - j) * kRadixBins + d)
                                           : kDigitInclusive;
                uint32_t advanced = 0;
                bool stop = false, done = false;
#pragma unroll
                for (uint32_t j = 0; j < kLookbackWindow; ++j) {   // nearest first, up to the first gap
                    const uint32_t status = s[j] >> 30;
                    if (!stop) {
                        if (status == 0) {
                            stop = true;
                        } else {
                            prefix += s[j] & kDigitCountMask;
                            ++advanced;
                            if (status == 2) stop = done = true;
                        }
                    }
                }
                if (done) break;
                if (advanced == 0) {
                    if (++spins > kSpinLimit) { if (error_flags) atomicOr(error_flags, MK_DEVICE_WAIT_TIMEOUT_FLAG); break; }
                    continue;
                }
                t -= advanced;
            }
            st_relaxed_u32(lb, kDigitInclusive | (prefix + count));
        }
        s_global_base[d] = s_digit_offsets[d] + prefix - local_start;
        __syncthreads();

        // ---- reorder through shared memory, then scatter by digit runs
#pragma unroll
        for (uint32_t i = 0; i < kSortItems; ++i) {
            if (dig[i] < kRadixBins) {
                uint32_t r = s_local_start[dig[i]] + s_warp[w][dig[i]] + rank[i];
                s_keys[r] = k[i];
                if (vals_out) s_vals[r] = v[i];
            }
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < total; j += kSortThreads) {
            uint64_t kk = s_keys[j];
            uint32_t dd = (uint32_t)((kk >> shift) & 0xffu);
            uint32_t dst = s_global_base[dd] + j;
            keys_out[dst] = kk;
            if (vals_out) vals_out[dst] = s_vals[j];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);   // every thread has read s_tile
    }
}

uint32_t sort_passes(uint32_t key_bits) { return (key_bits + 7) / 8; }

// Keys per thread of the onesweep tile: smaller tiles spread small sorts over
// more SMs, larger tiles amortise the look-back on large ones.  The choice is
// a tuning parameter (set_sort_items overrides the size-based default).
static uint32_t g_sort_items_override = 0;
void set_sort_items(uint32_t items) { g_sort_items_override = items; }
uint32_t sort_items_for(uint32_t n) {
    if (g_sort_items_override == 2 || g_sort_items_override == 4 || g_sort_items_override == 8)
        return g_sort_items_override;
    (void)n;
    return 8u;   // measured fastest for 0.4M-14M keys on B200 (look-back chains dominate small tiles)
}

// The histogram bins and tile tickets of a sort's scratch: the region that must
// be zero when the sort starts (launch_sort clears it unless told it is clear).
void sort_clear_region(void* scratch, uint32_t n, uint32_t key_bits, bool values, void** ptr, uint64_t* bytes) {
    const uint32_t passes = sort_passes(key_bits);
    char* p = (char*)scratch;
    p += align256((uint64_t)n * 8);
    p += align256((uint64_t)(values ? n : 0) * 4);
    *ptr = p;
    *bytes = align256((uint64_t)passes * kRadixBins * 4) + (uint64_t)passes * 4;
}

uint64_t sort_scratch_bytes(uint32_t n, uint32_t key_bits, bool values) {
    uint32_t passes = sort_passes(key_bits);
    uint64_t tiles = (n + 2 * kSortThreads - 1) / (2 * kSortThreads);   // smallest tile: 512 keys
    uint64_t b = 0;
    b += align256((uint64_t)n * 8);                       // ping-pong keys
    b += align256((uint64_t)(values ? n : 0) * 4);        // ping-pong values
    b += align256((uint64_t)passes * kRadixBins * 4);     // histograms / offsets
    b += align256((uint64_t)passes * 4);                  // tile tickets
    b += align256((uint64_t)passes * (tiles ? tiles : 1) * kRadixBins * 4);   // look-back words
    return b;
}

template <uint32_t kItems>
static void launch_pass(const uint64_t* sk, const uint32_t* sv, uint64_t* dk, uint32_t* dv, const uint32_t* n_dev,
                        uint32_t n, uint32_t shift, const uint32_t* offsets, uint32_t* lookback, uint32_t* ticket,
                        uint32_t* error_flags, uint32_t grid, cudaStream_t stream) {
    k_radix_onesweep<kItems><<<grid, kSortThreads, 0, stream>>>(sk, sv, dk, dv, n_dev, n, shift, offsets, lookback,
                                                                ticket, error_flags);
}

// Stream-ordered sort.  `n_dev` (device count) may be null, then n is used;
// with a device count, n is the capacity that sizes the grid and scratch.
cudaError_t launch_sort(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out, uint32_t* vals_out,
                        uint32_t n, const uint32_t* n_dev, uint32_t key_bits, void* scratch,
                        uint64_t scratch_bytes, uint32_t* error_flags, cudaStream_t stream, int sm_count,
                        uint32_t items_override, uint32_t ctas_per_sm, bool precleared) {
    if (n == 0) return cudaSuccess;
    uint32_t passes = sort_passes(key_bits);
    if (passes == 0 || passes > 8) return cudaErrorInvalidValue;
    const bool values = vals_in != nullptr;
    if (scratch_bytes < sort_scratch_bytes(n, key_bits, values)) return cudaErrorInvalidValue;
    const uint32_t items = (items_override == 2 || items_override == 4 || items_override == 8) ? items_override
                                                                                              : sort_items_for(n);
    const uint32_t tile_keys = kSortThreads * items;
    const uint64_t tiles = (n + tile_keys - 1) / tile_keys;
    const uint64_t tiles_max = (n + 2 * kSortThreads - 1) / (2 * kSortThreads);
    char* p = (char*)scratch;
    uint64_t* tmp_keys = (uint64_t*)p; p += align256((uint64_t)n * 8);
    uint32_t* tmp_vals = values ? (uint32_t*)p : nullptr; p += align256((uint64_t)(values ? n : 0) * 4);
    uint32_t* hist = (uint32_t*)p; p += align256((uint64_t)passes * kRadixBins * 4);
    uint32_t* tickets = (uint32_t*)p; p += align256((uint64_t)passes * 4);
    uint32_t* lookback = (uint32_t*)p;
    // histogram bins and tile tickets are cleared here; look-back words by the
    // histogram kernel, only as many as the device-side count needs
    if (!precleared) {
        cudaError_t e = cudaMemsetAsync(hist, 0, (uint64_t)((char*)tickets - (char*)hist) + passes * 4, stream);
        if (e != cudaSuccess) return e;
    }
    uint32_t hist_blocks = (uint32_t)std::min<uint64_t>((n + 4095) / 4096, (uint64_t)sm_count * 4);
    if (hist_blocks == 0) hist_blocks = 1;
    k_radix_histogram<<<hist_blocks, 256, 0, stream>>>(keys_in, n_dev, n, passes, hist, lookback,
                                                       tiles_max * kRadixBins, tile_keys);
    const uint32_t per_sm = ctas_per_sm ? ctas_per_sm : (items == 8 ? 3u : 6u);
    uint32_t grid = (uint32_t)std::min<uint64_t>(tiles, (uint64_t)sm_count * per_sm);
    if (grid == 0) grid = 1;
    // passes alternate between (tmp, out) so that the last pass writes `out`.
    const uint64_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        bool to_out = ((passes - 1 - pass) % 2) == 0;
        uint64_t* dk = to_out ? keys_out : tmp_keys;
        uint32_t* dv = values ? (to_out ? vals_out : tmp_vals) : nullptr;
        uint32_t* lb = lookback + (size_t)pass * tiles_max * kRadixBins;
        if (items == 2)
            launch_pass<2>(src_k, src_v, dk, dv, n_dev, n, 8 * pass, hist + pass * kRadixBins, lb, tickets + pass,
                           error_flags, grid, stream);
        else if (items == 4)
            launch_pass<4>(src_k, src_v, dk, dv, n_dev, n, 8 * pass, hist + pass * kRadixBins, lb, tickets + pass,
                           error_flags, grid, stream);
        else
            launch_pass<8>(src_k, src_v, dk, dv, n_dev, n, 8 * pass, hist + pass * kRadixBins, lb, tickets + pass,
                           error_flags, grid, stream);
        src_k = dk;
        src_v = dv;
    }
    return cudaGetLastError();
}

}  // namespace mk
