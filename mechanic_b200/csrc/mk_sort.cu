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

#include <atomic>

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
                  uint32_t* __restrict__ lookback, uint64_t lookback_pass_words, uint32_t tile_keys,
                  uint32_t small_n) {
    __shared__ uint32_t s_hist[8][kRadixBins];
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;   // a device count never exceeds the capacity
    if (n <= small_n) return;   // sorted by k_radix_small
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

// Ranks this warp's items by digit, item by item: lanes with the same digit
// are found by eight ballots (one per digit bit) under the valid-lane mask,
// and s_warp_row counts each digit over the warp's earlier items.  Digit
// kRadixBins marks an invalid item.
template <uint32_t kItems>
__device__ __forceinline__ void warp_rank(const uint32_t (&dig)[kItems], uint32_t (&rank)[kItems],
                                          uint32_t* s_warp_row, uint32_t lane) {
#pragma unroll
    for (uint32_t i = 0; i < kItems; ++i) {
        const uint32_t di = dig[i];
        const bool valid = di < kRadixBins;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (uint32_t bit = 0; bit < 8; ++bit) {
            const uint32_t on = (di >> bit) & 1u;
            const uint32_t bal = __ballot_sync(0xffffffffu, on);
            peers &= on ? bal : ~bal;
        }
        const uint32_t leader = __ffs(peers) - 1;   // invalid lanes: unused
        uint32_t base = 0;
        if (valid && lane == leader) base = s_warp_row[di];
        base = __shfl_sync(0xffffffffu, base, valid ? leader : lane);
        rank[i] = base + __popc(peers & lanemask_lt());
        if (valid && lane == leader) s_warp_row[di] = base + __popc(peers);
        __syncwarp();
    }
}

// Sorts up to kSmallSortKeys keys in one CTA, every pass in shared memory (no
// look-back, no histogram kernel: the tile's digit counts are the whole
// sort's); only the warps that hold keys rank.  Light ticks sort at most a few
// thousand pair keys: one launch instead of a histogram and one onesweep launch
// per digit.  With a device count above kSmallSortKeys it returns at once and
// the onesweep passes sort (one SM ranking 8,192 keys per pass was slower than
// four tiles on four SMs).
constexpr uint32_t kSmallThreads = 512, kSmallItems = 8;
constexpr uint32_t kSmallSortKeys = kSmallThreads * kSmallItems;
constexpr size_t kSmallSmem = (size_t)kSmallSortKeys * 12 + (kSmallThreads / 32) * kRadixBins * 4;

__global__ void __launch_bounds__(kSmallThreads)
k_radix_small(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
              uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, const uint32_t* __restrict__ n_ptr,
              uint32_t n_fixed, uint32_t passes) {
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
    if (n == 0 || n > kSmallSortKeys) return;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(s_dyn);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_dyn + (size_t)kSmallSortKeys * 8);
    uint32_t (*s_warp)[kRadixBins] = reinterpret_cast<uint32_t (*)[kRadixBins]>(s_dyn + (size_t)kSmallSortKeys * 12);
    __shared__ uint32_t s_local_start[kRadixBins];
    __shared__ uint32_t s_scan[33];
    const uint32_t lane = lane_id(), w = warp_id();
    const uint32_t d = threadIdx.x;   // the digit of threads below kRadixBins
    const uint32_t warps = (n + 32 * kSmallItems - 1) / (32 * kSmallItems);   // warps holding keys
    uint64_t k[kSmallItems];
    uint32_t v[kSmallItems], dig[kSmallItems], rank[kSmallItems];
#pragma unroll
    for (uint32_t i = 0; i < kSmallItems; ++i) {   // warp-striped: items in index order
        const uint32_t idx = w * 32 * kSmallItems + i * 32 + lane;
        k[i] = idx < n ? keys_in[idx] : 0ull;
        v[i] = (idx < n && vals_in) ? vals_in[idx] : 0u;
    }
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t shift = 8 * pass;
        for (uint32_t q = threadIdx.x; q < warps * kRadixBins; q += kSmallThreads) (&s_warp[0][0])[q] = 0;
        __syncthreads();
#pragma unroll
        for (uint32_t i = 0; i < kSmallItems; ++i) {
            const uint32_t idx = w * 32 * kSmallItems + i * 32 + lane;
            dig[i] = idx < n ? (uint32_t)((k[i] >> shift) & 0xffu) : kRadixBins;
        }
        if (w < warps) warp_rank<kSmallItems>(dig, rank, s_warp[w], lane);
        __syncthreads();
        uint32_t count = 0;
        if (d < kRadixBins) {
            for (uint32_t ww = 0; ww < warps; ++ww) {
                const uint32_t c = s_warp[ww][d];
                s_warp[ww][d] = count;
                count += c;
            }
        }
        uint32_t total;
        const uint32_t start = block_exclusive_scan(count, s_scan, &total);
        if (d < kRadixBins) s_local_start[d] = start;
        __syncthreads();
#pragma unroll
        for (uint32_t i = 0; i < kSmallItems; ++i) {
            if (dig[i] < kRadixBins) {
                const uint32_t r = s_local_start[dig[i]] + s_warp[w][dig[i]] + rank[i];
                s_keys[r] = k[i];
                s_vals[r] = v[i];
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t i = 0; i < kSmallItems; ++i) {
            const uint32_t idx = w * 32 * kSmallItems + i * 32 + lane;
            if (idx < n) {
                k[i] = s_keys[idx];
                v[i] = s_vals[idx];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (uint32_t i = 0; i < kSmallItems; ++i) {
        const uint32_t idx = w * 32 * kSmallItems + i * 32 + lane;
        if (idx < n) {
            keys_out[idx] = k[i];
            if (vals_out) vals_out[idx] = v[i];
        }
    }
}

// Shared-memory layout of a onesweep tile of kThreads x kItems keys: the
// reordered keys and values and one digit counter row per warp (dynamic
// shared memory: a 256 x 16 tile takes 56 KB).
template <uint32_t kThreads, uint32_t kItems>
struct SortTile {
    static constexpr uint32_t kTile = kThreads * kItems;
    static constexpr uint32_t kWarps = kThreads / 32;
    static constexpr size_t kValsOff = (size_t)kTile * 8;
    static constexpr size_t kWarpOff = kValsOff + (size_t)kTile * 4;
    static constexpr size_t kBytes = kWarpOff + (size_t)kWarps * kRadixBins * 4;
};

template <uint32_t kThreads, uint32_t kItems>
__global__ void __launch_bounds__(kThreads)
k_radix_onesweep(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                 uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                 const uint32_t* __restrict__ n_ptr, uint32_t n_fixed, uint32_t shift,
                 const uint32_t* __restrict__ digit_hist /* 256 */, uint32_t* __restrict__ lookback,
                 uint32_t* __restrict__ ticket, uint32_t* __restrict__ error_flags, uint32_t small_n) {
    static_assert(kThreads >= kRadixBins && kThreads % 32 == 0, "one thread per digit at least");
    using L = SortTile<kThreads, kItems>;
    constexpr uint32_t kTile = L::kTile;
    constexpr uint32_t kWarps = L::kWarps;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(s_dyn);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_dyn + L::kValsOff);
    uint32_t (*s_warp)[kRadixBins] = reinterpret_cast<uint32_t (*)[kRadixBins]>(s_dyn + L::kWarpOff);
    __shared__ uint32_t s_local_start[kRadixBins];
    __shared__ uint32_t s_global_base[kRadixBins];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_digit_offsets[kRadixBins];

    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;   // a device count never exceeds the capacity
    const uint32_t tiles = (n + kTile - 1) / kTile;
    // a small device count was sorted by k_radix_small; CTAs past the tile count
    // leave before taking a ticket (the grid is sized for the capacity)
    if (n <= small_n || blockIdx.x >= tiles) return;
    const uint32_t lane = lane_id(), w = warp_id();
    const bool digit_thread = threadIdx.x < kRadixBins;
    const uint32_t d = threadIdx.x;   // the digit of a digit thread
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    const uint32_t hist_d = digit_thread ? digit_hist[d] : 0u;   // scanned while the first tile loads
    bool have_offsets = false;

    for (;;) {
        for (uint32_t i = threadIdx.x; i < kWarps * kRadixBins; i += kThreads) (&s_warp[0][0])[i] = 0;
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= tiles) break;
        const uint32_t tile_base = tile * kTile;

        // ---- load every item first (one memory round trip), warp-striped
        uint64_t k[kItems];
        uint32_t v[kItems];
        uint32_t rank[kItems];
        uint32_t dig[kItems];
#pragma unroll
        for (uint32_t i = 0; i < kItems; ++i) {
            const uint32_t idx = tile_base + w * 32 * kItems + i * 32 + lane;
            const bool valid = idx < n;
            k[i] = valid ? __ldcg(keys_in + idx) : 0ull;
            v[i] = (valid && vals_in) ? __ldcg(vals_in + idx) : 0u;
            dig[i] = valid ? (uint32_t)((k[i] >> shift) & 0xffu) : kRadixBins;
        }
        if (!have_offsets) {   // this pass's digit offsets: exclusive scan of its histogram
            uint32_t total_all;
            const uint32_t off = block_exclusive_scan(hist_d, s_scan, &total_all);
            if (digit_thread) s_digit_offsets[d] = off;
            have_offsets = true;
        }

        // ---- rank within each warp
        warp_rank<kItems>(dig, rank, s_warp[w], lane);
        __syncthreads();

        // ---- per digit: prefix over warps, tile count, tile-local start
        uint32_t count = 0;
        if (digit_thread) {
#pragma unroll 8
            for (uint32_t ww = 0; ww < kWarps; ++ww) {
                const uint32_t c = s_warp[ww][d];
                s_warp[ww][d] = count;
                count += c;
            }
        }
        uint32_t total;
        const uint32_t local_start = block_exclusive_scan(count, s_scan, &total);

        if (digit_thread) {
            s_local_start[d] = local_start;
            // ---- decoupled look-back for digit d (one thread per digit), reading a
            // window of kLookbackWindow predecessors per round trip: with every tile
            // starting at once, a one-word walk advances the inclusive prefixes by
            // about two tiles per L2 round trip, a window by kLookbackWindow + 1
            // (relaxed stores: a word carries its own status and count, and a
            // release store's fence costs about an L2 round trip per tile)
            uint32_t* lb = lookback + (size_t)tile * kRadixBins + d;
            uint32_t prefix = 0;
            if (tile == 0) {
                st_relaxed_u32(lb, kDigitInclusive | count);
            } else {
                st_relaxed_u32(lb, kDigitAggregate | count);
                int64_t t = (int64_t)tile - 1;
                uint32_t spins = 0;
                for (;;) {
                    uint32_t sw[kLookbackWindow];
#pragma unroll
                    for (uint32_t j = 0; j < kLookbackWindow; ++j)   // below tile 0: an inclusive 0
                        sw[j] = t >= (int64_t)j ? ld_relaxed_u32(lookback + (size_t)(t - j) * kRadixBins + d)
                                                : kDigitInclusive;
                    uint32_t advanced = 0;
                    bool stop = false, done = false;
#pragma unroll
                    for (uint32_t j = 0; j < kLookbackWindow; ++j) {   // nearest first, up to the first gap
                        const uint32_t status = sw[j] >> 30;
                        if (!stop) {
                            if (status == 0) {
                                stop = true;
                            } else {
                                prefix += sw[j] & kDigitCountMask;
                                ++advanced;
                                if (status == 2) stop = done = true;
                            }
                        }
                    }
                    if (done) break;
                    if (advanced == 0) {
                        if (++spins > kSpinLimit) {
                            if (error_flags) atomicOr(error_flags, MK_DEVICE_WAIT_TIMEOUT_FLAG);
                            break;
                        }
                        continue;
                    }
                    t -= advanced;
                }
                st_relaxed_u32(lb, kDigitInclusive | (prefix + count));
            }
            s_global_base[d] = s_digit_offsets[d] + prefix - local_start;
        }
        __syncthreads();

        // ---- reorder through shared memory, then scatter by digit runs
#pragma unroll
        for (uint32_t i = 0; i < kItems; ++i) {
            if (dig[i] < kRadixBins) {
                const uint32_t r = s_local_start[dig[i]] + s_warp[w][dig[i]] + rank[i];
                s_keys[r] = k[i];
                if (vals_out) s_vals[r] = v[i];
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t i = 0; i < kItems; ++i) {
            const uint32_t j = threadIdx.x + i * kThreads;
            if (j < total) {
                const uint64_t kk = s_keys[j];
                const uint32_t dst = s_global_base[(uint32_t)((kk >> shift) & 0xffu)] + j;
                keys_out[dst] = kk;
                if (vals_out) vals_out[dst] = s_vals[j];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);   // every thread has read s_tile
    }
}

uint32_t sort_passes(uint32_t key_bits) { return (key_bits + 7) / 8; }

// Keys per thread of a 256-thread onesweep tile.  The pass is latency bound:
// its critical path is one tile's ranking (issue bound, so two tiles on one SM
// take twice as long) plus the look-back chain (one L2 round trip per
// kLookbackWindow tiles), so fewer, larger tiles win over spreading a sort
// across every SM.  Measured per pass on B200: 100k keys 10.8 us at 8 keys per
// thread (15.5 at 4); 400k 12.9 us at 11 or 16 (17.1 at 8); 1.6M 29.5 us at
// 11; 6.4M 82 us at 16.  set_sort_items overrides the default (a tuning
// parameter).
// 32 names the 8,192-key tile of 512 threads x 16 keys (the same keys per 256
// threads as 32 keys each): half the tiles of the 4,096-key shape, so the
// look-back frontier, which advances a window of tiles per L2 round trip,
// covers twice the keys per round trip.
static uint32_t g_sort_items_override = 0;
bool valid_sort_items(uint32_t items) {
    return items == 2 || items == 4 || items == 6 || items == 8 || items == 11 || items == 16 || items == 32;
}
void set_sort_items(uint32_t items) { g_sort_items_override = items; }

// The pair-key sort's tile is fixed when the tick is captured (its key count
// is only known on the device).  The 8,192-key tile: on the 100,000-body
// start (14.0M pairs) the five passes take 0.32 ms less than with 2,048-key
// tiles, and ticks with 8k-40k pairs about 20 us more each (one B200).
static uint32_t g_pair_sort_items = 0;
constexpr uint32_t kPairSortItemsDefault = 32;
uint32_t pair_sort_items() { return valid_sort_items(g_pair_sort_items) ? g_pair_sort_items : kPairSortItemsDefault; }
void set_pair_sort_items(uint32_t items) { g_pair_sort_items = valid_sort_items(items) ? items : 0u; }
uint32_t sort_items_for(uint32_t n, int sm_count) {
    if (valid_sort_items(g_sort_items_override)) return g_sort_items_override;
    (void)sm_count;
    // above 2M keys the 8,192-key tile (standalone sort with values, one B200: 3.6M keys
    // 245 against 271 us at 16 keys per thread, 14M keys 817 against 868 us)
    return n <= (1u << 16) ? 8u : n <= (1u << 21) ? 11u : 32u;
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
    uint64_t tiles = (n + 511) / 512;   // smallest tile: 512 keys
    uint64_t b = 0;
    b += align256((uint64_t)n * 8);                       // ping-pong keys
    b += align256((uint64_t)(values ? n : 0) * 4);        // ping-pong values
    b += align256((uint64_t)passes * kRadixBins * 4);     // histograms / offsets
    b += align256((uint64_t)passes * 4);                  // tile tickets
    b += align256((uint64_t)passes * (tiles ? tiles : 1) * kRadixBins * 4);   // look-back words
    return b;
}

template <uint32_t kThreads, uint32_t kItems>
static void launch_pass(const uint64_t* sk, const uint32_t* sv, uint64_t* dk, uint32_t* dv, const uint32_t* n_dev,
                        uint32_t n, uint32_t shift, const uint32_t* offsets, uint32_t* lookback, uint32_t* ticket,
                        uint32_t* error_flags, uint32_t grid, uint32_t small_n, cudaStream_t stream) {
    k_radix_onesweep<kThreads, kItems><<<grid, kThreads, SortTile<kThreads, kItems>::kBytes, stream>>>(
        sk, sv, dk, dv, n_dev, n, shift, offsets, lookback, ticket, error_flags, small_n);
}

// Dynamic shared memory of every tile shape, set once per device (outside
// stream capture: the first sort on a device, or handle creation).
cudaError_t sort_prepare() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return cudaSuccess;
#define MK_SORT_ATTR(T, I)                                                                                    \
    if (e == cudaSuccess)                                                                                    \
        e = cudaFuncSetAttribute(k_radix_onesweep<T, I>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                 (int)SortTile<T, I>::kBytes);
    MK_SORT_ATTR(kSortThreads, 2)
    MK_SORT_ATTR(kSortThreads, 4)
    MK_SORT_ATTR(kSortThreads, 6)
    MK_SORT_ATTR(kSortThreads, 8)
    MK_SORT_ATTR(kSortThreads, 11)
    MK_SORT_ATTR(kSortThreads, 16)
    MK_SORT_ATTR(2 * kSortThreads, 16)
#undef MK_SORT_ATTR
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_radix_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem);
    if (e == cudaSuccess) done.fetch_or(bit);
    return e;
}

// Stream-ordered sort.  `n_dev` (device count) may be null, then n is used;
// with a device count, n is the capacity that sizes the grid and scratch.
cudaError_t launch_sort(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out, uint32_t* vals_out,
                        uint32_t n, const uint32_t* n_dev, uint32_t key_bits, void* scratch,
                        uint64_t scratch_bytes, uint32_t* error_flags, cudaStream_t stream, int sm_count,
                        uint32_t items_override, uint32_t ctas_per_sm, bool precleared) {
    if (n == 0) return cudaSuccess;
    cudaError_t ep = sort_prepare();
    if (ep != cudaSuccess) return ep;
    uint32_t passes = sort_passes(key_bits);
    if (passes == 0 || passes > 8) return cudaErrorInvalidValue;
    const bool values = vals_in != nullptr;
    if (scratch_bytes < sort_scratch_bytes(n, key_bits, values)) return cudaErrorInvalidValue;
    // at most kSmallSortKeys keys: one CTA sorts them in shared memory; with a
    // device count it runs first and the histogram and passes skip small counts
    if (n_dev || n <= kSmallSortKeys)
        k_radix_small<<<1, kSmallThreads, kSmallSmem, stream>>>(keys_in, vals_in, keys_out, vals_out, n_dev, n, passes);
    if (!n_dev && n <= kSmallSortKeys) return cudaGetLastError();
    const uint32_t small_n = n_dev ? kSmallSortKeys : 0u;
    const uint32_t items = valid_sort_items(items_override) ? items_override : sort_items_for(n, sm_count);
    const uint32_t tile_keys = kSortThreads * items;
    const uint64_t tiles = (n + tile_keys - 1) / tile_keys;
    const uint64_t tiles_max = (n + 511) / 512;
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
                                                       tiles_max * kRadixBins, tile_keys, small_n);
    const uint32_t per_sm = ctas_per_sm ? ctas_per_sm : default_sort_ctas(items);
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
        const uint32_t* offs = hist + pass * kRadixBins;
#define MK_SORT_PASS(T, I)                                                                                       \
    launch_pass<T, I>(src_k, src_v, dk, dv, n_dev, n, 8 * pass, offs, lb, tickets + pass, error_flags, grid, small_n, \
                      stream)
        switch (items) {
            case 2: MK_SORT_PASS(kSortThreads, 2); break;
            case 4: MK_SORT_PASS(kSortThreads, 4); break;
            case 6: MK_SORT_PASS(kSortThreads, 6); break;
            case 8: MK_SORT_PASS(kSortThreads, 8); break;
            case 11: MK_SORT_PASS(kSortThreads, 11); break;
            case 32: MK_SORT_PASS(2 * kSortThreads, 16); break;
            default: MK_SORT_PASS(kSortThreads, 16); break;
        }
#undef MK_SORT_PASS
        src_k = dk;
        src_v = dv;
    }
    return cudaGetLastError();
}

}  // namespace mk
