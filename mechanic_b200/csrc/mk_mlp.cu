// mk_mlp.cu — the network of the learned parts on the 5th-generation tensor
// cores (tcgen05, bf16 operands, f32 accumulation in tensor memory).
//
// One network shape serves both learned parts: 16 inputs (slot 15 is the
// constant 1 that carries the first layer's bias), two hidden layers of 64
// with ReLU, 16 outputs (the caller uses the first few):
//   h1 = relu(W1 x),  h2 = relu(W2 h1 + b2),  y = W3 h2 + b3.
// Parameters are one f32 array (row-major [out][in]): W1 64x16 | W2 64x64 |
// W3 16x64 | b2 64 | b3 16; the kernels read bf16 copies of the weights.
//
// A CTA of 128 threads takes 128-sample tiles.  Thread t owns sample t of
// the tile, which is TMEM lane t of every accumulator, so the epilogues are
// one tcgen05.ld per 16 columns and no shuffles.  The backward pass reuses
// the activations where they lie: the same shared-memory tiles are read
// K-major by the data-gradient MMAs and MN-major by the weight-gradient MMAs
// (which reduce over the 128 samples of the tile), so nothing is transposed.
// The two 64-row weight gradients are stacked into one M = 128 MMA
// ([dH2; dH1] x [H1; X]^T), whose off-diagonal blocks are unused except the
// column of the constant input, which is the sum of dH2 over samples (db2).
// Weight gradients accumulate in TMEM across a CTA's tiles; each CTA writes
// one partial and a second kernel sums the partials in CTA order, so the
// gradient of a batch is deterministic.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "mk_device.cuh"
#include "mk_internal.h"
#include "mk_mlp.h"
#include "mk_tc.cuh"

namespace mk {
namespace mlp {

constexpr uint32_t kTile = 128, kThreads = 128, kCH = 2048;   // bytes per 8-column chunk of a 128-row tile
constexpr uint32_t kTmemCols = 256;
// accumulator columns: layer 1 / dH1, layer 2 / dH2, layer 3, dW3^T block, [dW2 | db2 | dW1] block
constexpr uint32_t cAcc1 = 0, cAcc2 = 64, cAcc3 = 128, cDB = 144, cDA = 160;
constexpr uint32_t kWaitLimit = 1u << 20;

template <bool kTrain>
struct Layout {
    // F: [H1 (chunks 0-7) | X (8-9)]; G: [H2 (0-7) | dH2 (8-15) | dH1 (16-23)]; Y: dY (0-1)
    static constexpr uint32_t F = 0;
    static constexpr uint32_t G = F + 10 * kCH;
    static constexpr uint32_t Y = G + (kTrain ? 24 : 8) * kCH;
    static constexpr uint32_t W1 = Y + (kTrain ? 2 * kCH : 0);
    static constexpr uint32_t W2 = W1 + 2048;
    static constexpr uint32_t W3 = W2 + 8192;
    static constexpr uint32_t B2 = W3 + 2048;
    static constexpr uint32_t B3 = B2 + 256;
    static constexpr uint32_t RED = B3 + 64;              // 4 warps x 17 floats (db3, loss)
    static constexpr uint32_t BAR = RED + 4 * 17 * 4 + 16;
    static constexpr uint32_t SLOT = BAR + 8;
    static constexpr uint32_t BYTES = SLOT + 8;
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Eight consecutive columns of one row into its 16-byte slot of a tile.
__device__ __forceinline__ void store8(unsigned char* buf, uint32_t chunk, uint32_t row, const float* v) {
    uint4 u = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    *reinterpret_cast<uint4*>(buf + chunk * kCH + (row >> 3) * 128 + (row & 7) * 16) = u;
}
__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__device__ __forceinline__ void publish() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

template <bool kTrain>
__global__ void __launch_bounds__(kThreads) k_mlp(const __nv_bfloat16* __restrict__ wts, const float* __restrict__ params,
                                                   const float* __restrict__ x, uint32_t n_host, const uint32_t* n_dev,
                                                   float* __restrict__ y, uint32_t y_cols, const float* __restrict__ t,
                                                   const float* __restrict__ out_w, float* __restrict__ partials,
                                                   uint32_t* __restrict__ error_flags) {
    using L = Layout<kTrain>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* F = smem + L::F;
    unsigned char* G = smem + L::G;
    unsigned char* Yb = smem + L::Y;
    unsigned char* W1s = smem + L::W1;
    unsigned char* W2s = smem + L::W2;
    unsigned char* W3s = smem + L::W3;
    float* sb2 = reinterpret_cast<float*>(smem + L::B2);
    float* sb3 = reinterpret_cast<float*>(smem + L::B3);
    float* sred = reinterpret_cast<float*>(smem + L::RED);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + L::SLOT);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t n = n_dev ? *n_dev : n_host;

    // weights into the core-matrix layout (W1: 64 rows x 2 chunks, W2: 64 x 8, W3: 16 x 8)
    for (uint32_t u = tid; u < 128; u += kThreads) {
        const uint32_t row = u >> 1, kc = u & 1u;
        *reinterpret_cast<uint4*>(W1s + kc * 1024 + (row >> 3) * 128 + (row & 7) * 16) =
            *reinterpret_cast<const uint4*>(wts + kW1 + row * 16 + kc * 8);
    }
    for (uint32_t u = tid; u < 512; u += kThreads) {
        const uint32_t row = u >> 3, kc = u & 7u;
        *reinterpret_cast<uint4*>(W2s + kc * 1024 + (row >> 3) * 128 + (row & 7) * 16) =
            *reinterpret_cast<const uint4*>(wts + kW2 + row * 64 + kc * 8);
    }
    for (uint32_t u = tid; u < 128; u += kThreads) {
        const uint32_t row = u >> 3, kc = u & 7u;
        *reinterpret_cast<uint4*>(W3s + kc * 256 + (row >> 3) * 128 + (row & 7) * 16) =
            *reinterpret_cast<const uint4*>(wts + kW3 + row * 64 + kc * 8);
    }
    if (tid < 64) sb2[tid] = params[kB2 + tid];
    if (tid < 16) sb3[tid] = params[kB3 + tid];
    if (tid == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(tslot, kTmemCols);
    publish();
    const uint32_t tbase = *tslot;
    const uint32_t tlane = tbase + ((32u * warp) << 16);
    uint32_t phase = 0;
    bool timed_out = false;
    auto mma_wait = [&]() {
        if (!tc::mbar_wait(bar, phase, kWaitLimit) && !timed_out) {
            timed_out = true;
            atomicOr(error_flags, MK_DEVICE_WAIT_TIMEOUT_FLAG);
        }
        phase ^= 1u;
        tc::fence_after_sync();
    };
    const uint32_t sF = tc::smem_u32(F), sG = tc::smem_u32(G), sY = tc::smem_u32(Yb);
    const uint32_t sW1 = tc::smem_u32(W1s), sW2 = tc::smem_u32(W2s), sW3 = tc::smem_u32(W3s);
    constexpr uint32_t id64 = tc::idesc_bf16(128, 64, false, false);
    constexpr uint32_t id16 = tc::idesc_bf16(128, 16, false, false);
    constexpr uint32_t id64_bmn = tc::idesc_bf16(128, 64, false, true);
    constexpr uint32_t id80_mn = tc::idesc_bf16(128, 80, true, true);
    constexpr uint32_t id16_mn = tc::idesc_bf16(128, 16, true, true);

    const float coef = n > 0 ? 2.0f / (float)n : 0.0f;
    float loss = 0.0f;
    float db3[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) db3[o] = 0.0f;

    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++it) {
        const uint32_t s = tile * kTile + tid;
        const bool valid = s < n;
        float v[16];
        if (valid) {
            const float4* xr = reinterpret_cast<const float4*>(x + (size_t)s * 16);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 f = __ldg(xr + q);
                v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
            }
            v[15] = 1.0f;
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.0f;
        }
        store8(F, 8, tid, v);
        store8(F, 9, tid, v + 8);
        publish();
        // layer 1: [128 x 16] x W1^T
        if (tid == 0) {
            tc::mma_bf16(tbase + cAcc1, tc::sdesc(sF + 8 * kCH, kCH, 128), tc::sdesc(sW1, 1024, 128), id64, 0);
            tc::commit(bar);
        }
        mma_wait();
        uint64_t mask1 = 0, mask2 = 0;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            tc::tmem_ld16(tlane + cAcc1 + 16 * q, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (v[i] > 0.0f) mask1 |= 1ull << (16 * q + i);
                else v[i] = 0.0f;
            }
            store8(F, 2 * q, tid, v);
            store8(F, 2 * q + 1, tid, v + 8);
        }
        publish();
        // layer 2: H1 [128 x 64] x W2^T
        if (tid == 0) {
#pragma unroll
            for (uint32_t ks = 0; ks < 4; ++ks)
                tc::mma_bf16(tbase + cAcc2, tc::sdesc(sF + 2 * ks * kCH, kCH, 128), tc::sdesc(sW2 + 2 * ks * 1024, 1024, 128),
                             id64, ks > 0);
            tc::commit(bar);
        }
        mma_wait();
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            tc::tmem_ld16(tlane + cAcc2 + 16 * q, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] += sb2[16 * q + i];
                if (v[i] > 0.0f) mask2 |= 1ull << (16 * q + i);
                else v[i] = 0.0f;
            }
            store8(G, 2 * q, tid, v);
            store8(G, 2 * q + 1, tid, v + 8);
        }
        publish();
        // layer 3: H2 [128 x 64] x W3^T
        if (tid == 0) {
#pragma unroll
            for (uint32_t ks = 0; ks < 4; ++ks)
                tc::mma_bf16(tbase + cAcc3, tc::sdesc(sG + 2 * ks * kCH, kCH, 128), tc::sdesc(sW3 + 2 * ks * 256, 256, 128),
                             id16, ks > 0);
            tc::commit(bar);
        }
        mma_wait();
        tc::tmem_ld16(tlane + cAcc3, v);
#pragma unroll
        for (int o = 0; o < 16; ++o) v[o] += sb3[o];
        if constexpr (!kTrain) {
            if (valid)
                for (uint32_t o = 0; o < y_cols; ++o) y[(size_t)s * y_cols + o] = v[o];
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            continue;
        } else {
            // dL/dy of L = (1/n) sum w_o (y_o - t_o)^2
            float tv[16];
            if (valid) {
                const float4* tr = reinterpret_cast<const float4*>(t + (size_t)s * 16);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 f = __ldg(tr + q);
                    tv[4 * q] = f.x; tv[4 * q + 1] = f.y; tv[4 * q + 2] = f.z; tv[4 * q + 3] = f.w;
                }
            }
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                float d = 0.0f;
                if (valid) {
                    const float e = v[o] - tv[o];
                    const float w = __ldg(out_w + o);
                    loss += w * e * e;
                    d = bf16_round(coef * w * e);
                }
                db3[o] += d;
                v[o] = d;
            }
            store8(Yb, 0, tid, v);
            store8(Yb, 1, tid, v + 8);
            publish();
            // dH2 = dY [128 x 16] x W3 (W3 read MN-major)
            if (tid == 0) {
                tc::mma_bf16(tbase + cAcc2, tc::sdesc(sY, kCH, 128), tc::sdesc(sW3, 128, 256), id64_bmn, 0);
                tc::commit(bar);
            }
            mma_wait();
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                tc::tmem_ld16(tlane + cAcc2 + 16 * q, v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (!((mask2 >> (16 * q + i)) & 1ull)) v[i] = 0.0f;
                store8(G, 8 + 2 * q, tid, v);
                store8(G, 9 + 2 * q, tid, v + 8);
            }
            publish();
            // dH1 = dH2 [128 x 64] x W2 (W2 read MN-major)
            if (tid == 0) {
#pragma unroll
                for (uint32_t ks = 0; ks < 4; ++ks)
                    tc::mma_bf16(tbase + cAcc1, tc::sdesc(sG + (8 + 2 * ks) * kCH, kCH, 128),
                                 tc::sdesc(sW2 + ks * 256, 128, 1024), id64_bmn, ks > 0);
                tc::commit(bar);
            }
            mma_wait();
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                tc::tmem_ld16(tlane + cAcc1 + 16 * q, v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (!((mask1 >> (16 * q + i)) & 1ull)) v[i] = 0.0f;
                store8(G, 16 + 2 * q, tid, v);
                store8(G, 17 + 2 * q, tid, v + 8);
            }
            publish();
            // weight gradients, reduced over the tile's samples (K = samples):
            //   [dH2; dH1]^T-stack x [H1; X]  -> dW2 | db2 and dW1
            //   [H2; dH2] x dY               -> dW3^T
            if (tid == 0) {
#pragma unroll
                for (uint32_t ks = 0; ks < 8; ++ks) {
                    const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
                    tc::mma_bf16(tbase + cDA, tc::sdesc(sG + 8 * kCH + ks * 256, 128, kCH),
                                 tc::sdesc(sF + ks * 256, 128, kCH), id80_mn, acc);
                    tc::mma_bf16(tbase + cDB, tc::sdesc(sG + ks * 256, 128, kCH), tc::sdesc(sY + ks * 256, 128, kCH),
                                 id16_mn, acc);
                }
                tc::commit(bar);
            }
            mma_wait();
        }
    }

    if constexpr (kTrain) {
        float* part = partials + (size_t)blockIdx.x * kPartialStride;
        float g[16];
        if (warp < 2) {
            const uint32_t i = 32 * warp + lane;   // hidden-2 unit (row of dW2, column of dW3)
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                if (it > 0) tc::tmem_ld16(tlane + cDA + 16 * q, g);
#pragma unroll
                for (int j = 0; j < 16; ++j) part[kW2 + i * 64 + 16 * q + j] = it > 0 ? g[j] : 0.0f;
            }
            if (it > 0) tc::tmem_ld16(tlane + cDA + 64, g);
            part[kB2 + i] = it > 0 ? g[15] : 0.0f;
            if (it > 0) tc::tmem_ld16(tlane + cDB, g);
#pragma unroll
            for (int o = 0; o < 16; ++o) part[kW3 + o * 64 + i] = it > 0 ? g[o] : 0.0f;
        } else {
            const uint32_t i = 32 * (warp - 2) + lane;   // hidden-1 unit (row of dW1)
            if (it > 0) tc::tmem_ld16(tlane + cDA + 64, g);
#pragma unroll
            for (int k = 0; k < 16; ++k) part[kW1 + i * 16 + k] = it > 0 ? g[k] : 0.0f;
        }
        // db3 and the loss: fixed-order warp trees, then the warps in order
#pragma unroll
        for (int o = 0; o < 17; ++o) {
            float r = o < 16 ? db3[o] : loss;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) r += __shfl_xor_sync(0xffffffffu, r, d);
            if (lane == 0) sred[warp * 17 + o] = r;
        }
        __syncthreads();
        if (tid < 17) {
            const float r = ((sred[tid] + sred[17 + tid]) + sred[34 + tid]) + sred[51 + tid];
            part[tid < 16 ? kB3 + tid : kLossSlot] = tid < 16 ? r : r * coef * 0.5f;   // loss = sum / n
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, kTmemCols);
}

// f32 parameters -> bf16 weights (round to nearest even)
__global__ void k_mlp_pack(const float* __restrict__ params, __nv_bfloat16* __restrict__ wts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kWeights) wts[i] = __float2bfloat16_rn(params[i]);
}

// Sum of the per-CTA partials in CTA order; optionally one Adam step.
__global__ void k_mlp_reduce_adam(const float* __restrict__ partials, uint32_t nparts, float* __restrict__ grad,
                                  float* __restrict__ loss_out, float* __restrict__ params, float* __restrict__ m,
                                  float* __restrict__ v, AdamStep a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > kLossSlot) return;
    float g = 0.0f;
    for (uint32_t c = 0; c < nparts; ++c) g += partials[(size_t)c * kPartialStride + i];
    if (grad) grad[i] = g;
    if (i == kLossSlot) {
        if (loss_out) *loss_out = g;
        return;
    }
    if (!params) return;
    const float mi = a.beta1 * m[i] + (1.0f - a.beta1) * g;
    const float vi = a.beta2 * v[i] + (1.0f - a.beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / a.bias1, vh = vi / a.bias2;
    params[i] -= a.lr * mh / (sqrtf(vh) + a.eps);
}

static int g_sm_count = 0;

static cudaError_t prepare_attributes() {
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Layout<true>::BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Layout<false>::BYTES);
    if (e == cudaSuccess) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        done = true;
    }
    return e;
}

uint64_t scratch_bytes(uint32_t max_samples) {
    (void)max_samples;
    int sms = g_sm_count > 0 ? g_sm_count : 148;
    return align256((uint64_t)kWeights * 2) + align256((uint64_t)sms * kPartialStride * 4) + align256(4);
}

cudaError_t init(void) { return prepare_attributes(); }

cudaError_t pack(const float* params, void* scratch, cudaStream_t s) {
    k_mlp_pack<<<(kWeights + 255) / 256, 256, 0, s>>>(params, reinterpret_cast<__nv_bfloat16*>(scratch));
    return cudaGetLastError();
}

cudaError_t forward(const float* params, const float* x, uint32_t n, const uint32_t* n_dev, uint32_t max_n, float* y,
                    uint32_t y_cols, void* scratch, uint32_t* error_flags, cudaStream_t s) {
    cudaError_t e = prepare_attributes();
    if (e != cudaSuccess) return e;
    const uint32_t tiles = ((n_dev ? max_n : n) + kTile - 1) / kTile;
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, 2u * (uint32_t)g_sm_count));
    k_mlp<false><<<grid, kThreads, Layout<false>::BYTES, s>>>(reinterpret_cast<const __nv_bfloat16*>(scratch), params,
                                                               x, n, n_dev, y, y_cols, nullptr, nullptr, nullptr,
                                                               error_flags);
    return cudaGetLastError();
}

cudaError_t gradient(const float* params, const float* x, const float* t, const float* out_w, uint32_t n, void* scratch,
                     float* grad, float* loss_out, float* m, float* v, float* update_params, const AdamStep& a,
                     uint32_t* error_flags, cudaStream_t s) {
    cudaError_t e = prepare_attributes();
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, (uint32_t)g_sm_count));
    char* base = reinterpret_cast<char*>(scratch);
    const __nv_bfloat16* wts = reinterpret_cast<const __nv_bfloat16*>(base);
    float* partials = reinterpret_cast<float*>(base + align256((uint64_t)kWeights * 2));
    k_mlp<true><<<grid, kThreads, Layout<true>::BYTES, s>>>(wts, params, x, n, nullptr, nullptr, 0, t, out_w, partials,
                                                             error_flags);
    k_mlp_reduce_adam<<<(kLossSlot + 256) / 256, 256, 0, s>>>(partials, grid, grad, loss_out, update_params, m, v, a);
    return cudaGetLastError();
}

}  // namespace mlp
}  // namespace mk

// ------------------------------------------------------------------ C ABI
namespace {
int check_mlp(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return MK_OK;
    char msg[256];
    std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    mk::set_last_error(msg);
    return MK_ERR_DEVICE_FAILURE;
}
int bad_mlp(const char* msg) {
    mk::set_last_error(msg);
    return MK_ERR_INVALID_ARGUMENT;
}
}  // namespace

extern "C" {

MK_API uint32_t mk_mlp_param_count(void) { return mk::mlp::kParams; }

MK_API uint64_t mk_op_mlp_scratch_bytes(uint32_t max_samples) {
    if (mk::mlp::init() != cudaSuccess) return 0;
    return mk::mlp::scratch_bytes(max_samples);
}

MK_API int mk_op_mlp_forward(const float* params, const float* x, uint32_t n, float* y, uint32_t y_cols, void* scratch,
                             uint64_t scratch_bytes, uint32_t* error_flags, void* stream) {
    if (!params || !scratch || !error_flags || (n && (!x || !y))) return bad_mlp("mlp forward: null pointer");
    if (y_cols == 0 || y_cols > 16) return bad_mlp("mlp forward: y_cols must be 1..16");
    if ((reinterpret_cast<uintptr_t>(x) & 15u) != 0) return bad_mlp("mlp forward: x must be 16-byte aligned");
    if (mk::mlp::init() != cudaSuccess) return check_mlp(cudaGetLastError(), "mlp init");
    if (scratch_bytes < mk::mlp::scratch_bytes(n)) return bad_mlp("mlp forward: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = mk::mlp::pack(params, scratch, s);
    if (e == cudaSuccess && n) e = mk::mlp::forward(params, x, n, nullptr, n, y, y_cols, scratch, error_flags, s);
    return check_mlp(e, "mlp forward");
}

MK_API int mk_op_mlp_gradient(const float* params, const float* x, const float* targets, const float* out_weights,
                              uint32_t n, float* grad, void* scratch, uint64_t scratch_bytes, uint32_t* error_flags,
                              void* stream) {
    if (!params || !x || !targets || !out_weights || !grad || !scratch || !error_flags || n == 0)
        return bad_mlp("mlp gradient: null pointer or no samples");
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(targets)) & 15u) != 0)
        return bad_mlp("mlp gradient: x and targets must be 16-byte aligned");
    if (mk::mlp::init() != cudaSuccess) return check_mlp(cudaGetLastError(), "mlp init");
    if (scratch_bytes < mk::mlp::scratch_bytes(n)) return bad_mlp("mlp gradient: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    mk::mlp::AdamStep a{0, 0, 0, 0, 1, 1};
    cudaError_t e = mk::mlp::pack(params, scratch, s);
    if (e == cudaSuccess)
        e = mk::mlp::gradient(params, x, targets, out_weights, n, scratch, grad, nullptr, nullptr, nullptr, nullptr, a,
                              error_flags, s);
    return check_mlp(e, "mlp gradient");
}

MK_API int mk_op_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* targets,
                           const float* out_weights, uint32_t n, uint32_t batch, uint32_t steps, float lr,
                           uint32_t first_step, float* losses, void* scratch, uint64_t scratch_bytes,
                           uint32_t* error_flags, void* stream) {
    if (!params || !adam_m || !adam_v || !x || !targets || !out_weights || !scratch || !error_flags || n == 0)
        return bad_mlp("mlp train: null pointer or no samples");
    if (batch == 0 || batch > n) batch = n;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(targets)) & 15u) != 0)
        return bad_mlp("mlp train: x and targets must be 16-byte aligned");
    if (mk::mlp::init() != cudaSuccess) return check_mlp(cudaGetLastError(), "mlp init");
    if (scratch_bytes < mk::mlp::scratch_bytes(batch)) return bad_mlp("mlp train: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const float b1 = 0.9f, b2 = 0.999f;
    cudaError_t e = cudaSuccess;
    uint32_t offset = 0;
    for (uint32_t k = 0; k < steps && e == cudaSuccess; ++k) {
        const float step = (float)(first_step + k + 1);
        const mk::mlp::AdamStep a{lr, b1, b2, 1.0e-8f, 1.0f - std::pow(b1, step), 1.0f - std::pow(b2, step)};
        if (offset + batch > n) offset = 0;   // batches walk the (pre-shuffled) samples cyclically
        e = mk::mlp::pack(params, scratch, s);
        if (e == cudaSuccess)
            e = mk::mlp::gradient(params, x + (size_t)offset * 16, targets + (size_t)offset * 16, out_weights, batch,
                                  scratch, nullptr, losses ? losses + k : nullptr, adam_m, adam_v, params, a,
                                  error_flags, s);
        offset += batch;
    }
    return check_mlp(e, "mlp train");
}

}  // extern "C"
