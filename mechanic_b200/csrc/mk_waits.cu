// mk_waits.cu — self-test of the bounded device waits.
//
// Every spin-wait in the library's kernels has an iteration limit: the grid
// barrier of the cooperative launches, the decoupled look-back of the ordered
// appends and the mbarrier wait of the tensor-core kernels give up after it,
// raise MK_DEVICE_WAIT_TIMEOUT_FLAG and return, so a participant that never
// arrives costs a wrong result and a flag, never a hung GPU.  The reference's
// waits (the storageBarrier refit of lbvh.wgsl:290-319) assume arrival and
// have no such path.
//
// The self-test runs the same device functions on waits that nothing can
// satisfy, with a small limit, so the give-up path can be exercised without
// a fault: a grid barrier expecting one block more than were launched, a
// look-back tile whose predecessor never publishes, and an mbarrier that no
// thread arrives on.  Each probe is a few small blocks that all end by
// themselves once the limit is reached.
#include <cstdio>

#include "mk_device.cuh"
#include "mk_internal.h"
#include "mk_tc.cuh"

namespace {

// Two barriers in a row, each waiting for `participants` blocks while only
// gridDim.x run: every block gives up at both and reaches the end.
__global__ void k_probe_grid_barrier(uint32_t* state, uint32_t* flags, uint32_t participants, uint32_t limit,
                                     uint32_t* done) {
    mk::grid_barrier(state, flags, participants, limit);
    mk::grid_barrier(state, flags, participants, limit);
    if (threadIdx.x == 0) atomicAdd(done, 1u);
}

// One warp plays tile 1 of an ordered append; tile 0's word stays empty.
__global__ void k_probe_lookback(uint64_t* states, uint32_t* flags, uint32_t limit, uint64_t* prefix_out,
                                 uint32_t* done) {
    if (threadIdx.x >= 32) return;
    const uint64_t prefix = mk::tile_lookback(states, 1, 5, flags, limit);
    if (threadIdx.x == 0) {
        *prefix_out = prefix;
        atomicAdd(done, 1u);
    }
}

// A shared-memory mbarrier expecting one arrival that never comes.
__global__ void k_probe_mbarrier(uint32_t* flags, uint32_t limit, uint32_t* done) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mk::tc::mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!mk::tc::mbar_wait(&bar, 0, limit)) atomicOr(flags, MK_DEVICE_WAIT_TIMEOUT_FLAG);
        atomicAdd(done, 1u);
    }
}

struct Probe {
    uint32_t flags, done, barrier, pad;
    uint64_t prefix;
    uint64_t states[4];
};

}  // namespace

extern "C" int mk_selftest_bounded_wait(uint32_t which, uint32_t spin_limit, MkWaitProbe* out, MkError* err) {
    char msg[200];
    auto fail = [&](int code, const char* what) {
        if (err) {
            err->code = code;
            std::snprintf(err->message, sizeof(err->message), "%s", what);
        }
        mk::set_last_error(what);
        return code;
    };
    if (!out) return fail(MK_ERR_INVALID_ARGUMENT, "selftest_bounded_wait: null result");
    if (which > MK_WAIT_PROBE_MBARRIER) return fail(MK_ERR_INVALID_ARGUMENT, "selftest_bounded_wait: unknown probe");
    if (spin_limit == 0 || spin_limit > (1u << 16))
        return fail(MK_ERR_INVALID_ARGUMENT, "selftest_bounded_wait: spin_limit must be in 1..65536");
    Probe* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(Probe));
    cudaStream_t s = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(Probe), s);
    uint32_t blocks = 1;
    if (e == cudaSuccess) e = cudaEventRecord(t0, s);
    if (e == cudaSuccess) {
        switch (which) {
            case MK_WAIT_PROBE_GRID_BARRIER:
                blocks = 4;   // the barrier expects 5
                k_probe_grid_barrier<<<blocks, 128, 0, s>>>(&d->barrier, &d->flags, blocks + 1, spin_limit, &d->done);
                break;
            case MK_WAIT_PROBE_LOOKBACK:
                k_probe_lookback<<<1, 32, 0, s>>>(d->states, &d->flags, spin_limit, &d->prefix, &d->done);
                break;
            default:
                k_probe_mbarrier<<<1, 32, 0, s>>>(&d->flags, spin_limit, &d->done);
                break;
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(t1, s);
    Probe h{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(Probe), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (s) cudaStreamDestroy(s);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof(msg), "selftest_bounded_wait: %s", cudaGetErrorString(e));
        return fail(MK_ERR_DEVICE_FAILURE, msg);
    }
    out->error_flags = h.flags;
    out->blocks_finished = h.done;
    out->blocks_launched = blocks;
    out->lookback_prefix = h.prefix;
    out->elapsed_ms = (double)ms;
    return MK_OK;
}
