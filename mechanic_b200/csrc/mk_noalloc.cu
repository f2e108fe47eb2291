// mk_noalloc.cu — the LBVH key sort for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc at the point where they need the sort:
// allocators and memory-pool hooks that must not recurse into the allocator,
// and embedders whose memory budget is fixed up front and must not grow.  For
// them this file keeps the sort's scratch in one statically sized device array
// that the library owns, so a call needs only the caller's input and output
// buffers.  The call still launches kernels on the caller's stream, so it is
// not for code running inside a CUDA host function (cudaLaunchHostFunc or a
// stream callback), where CUDA forbids every CUDA API call.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it until the process exits.  In host code its name is only a
// host-side stand-in, never a device address, so the first call on each
// device (with that device current) looks up the real address with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture, because the lookup may load the module.  The cached address belongs
// to the device's primary context: after cudaDeviceReset (or anything else that
// destroys and recreates that context) it is stale, and this entry point must
// not be called again in that process.  Every call shares the one
// array and it keeps the previous call's contents: the sort clears what must
// start at zero (bins, tile tickets, look-back words) itself, and two calls
// whose work overlaps on the GPU (different streams, or several host threads)
// race on the array, so callers must order them.
#include <cstdio>
#include <mutex>

#include "mk_device.cuh"
#include "mk_internal.h"

namespace {

// Largest key count the static scratch serves.
constexpr uint32_t kStaticSortMaxKeys = 1u << 19;   // 524,288 keys (~14 MB of scratch)

// Same layout as the caller-scratch sort: ping-pong keys and values,
// 8 histograms, 8 tile tickets, look-back words for 512-key tiles.
constexpr uint64_t a256(uint64_t b) { return (b + 255) & ~255ull; }
constexpr uint64_t kStaticSortScratchBytes =
    a256((uint64_t)kStaticSortMaxKeys * 8) + a256((uint64_t)kStaticSortMaxKeys * 4) + a256(8ull * 256 * 4) +
    a256(8ull * 4) + a256(8ull * ((kStaticSortMaxKeys + 511) / 512) * 256 * 4);

__device__ __align__(256) unsigned char g_sort_scratch[kStaticSortScratchBytes];

static_assert(kStaticSortMaxKeys == MK_STATIC_SORT_MAX_KEYS, "header and scratch size disagree");

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

int fail(int code, const char* msg) {
    mk::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" {

int mk_op_sort_keys_static(const uint64_t* keys_in, const uint32_t* values_in, uint64_t* keys_out,
                           uint32_t* values_out, uint32_t n, uint32_t key_bits, void* stream) {
    char msg[160];
    if (n == 0) return MK_OK;
    if (!keys_in || !values_in || !keys_out || !values_out || key_bits == 0 || key_bits > 64)
        return fail(MK_ERR_INVALID_ARGUMENT, "sort_keys_static: null pointer or key_bits outside 1..64");
    if (n > kStaticSortMaxKeys) {
        std::snprintf(msg, sizeof(msg), "sort_keys_static: %u keys exceed the static scratch limit of %u keys", n,
                      kStaticSortMaxKeys);
        return fail(MK_ERR_INVALID_ARGUMENT, msg);
    }
    if (mk::sort_buffers_overlap(keys_in, values_in, keys_out, values_out, n))
        return fail(MK_ERR_INVALID_ARGUMENT, "sort_keys_static: input and output buffers overlap");
    if (mk::sort_scratch_bytes(n, key_bits, true) > kStaticSortScratchBytes)
        return fail(MK_ERR_INVALID_ARGUMENT, "sort_keys_static: scratch layout exceeds the static array");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(MK_ERR_DEVICE_FAILURE, "sort_keys_static: no usable current device");
    void* scratch = nullptr;
    {
        // Once per device, with that device current: the device address of the array.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_address[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
            if (e != cudaSuccess || !p) {
                std::snprintf(msg, sizeof(msg), "sort_keys_static: cudaGetSymbolAddress failed: %s",
                              cudaGetErrorString(e));
                return fail(MK_ERR_DEVICE_FAILURE, msg);
            }
            g_scratch_address[dev] = p;
        }
        scratch = g_scratch_address[dev];
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = mk::launch_sort(keys_in, values_in, keys_out, values_out, n, nullptr, key_bits, scratch,
                                          kStaticSortScratchBytes, nullptr, (cudaStream_t)stream, sms);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof(msg), "sort_keys_static: %s", cudaGetErrorString(e));
        return fail(MK_ERR_DEVICE_FAILURE, msg);
    }
    return MK_OK;
}

}  // extern "C"
