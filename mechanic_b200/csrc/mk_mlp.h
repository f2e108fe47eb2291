// mk_mlp.h — the network of the learned parts (16 -> 64 -> 64 -> 16, ReLU),
// bf16 tensor-core forward, backward and Adam on sm_100a.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mk {
namespace mlp {

// f32 parameter layout: W1 [64][16] (column 15 = first-layer bias, input
// slot 15 is the constant 1) | W2 [64][64] | W3 [16][64] | b2 [64] | b3 [16].
constexpr uint32_t kW1 = 0, kW2 = 1024, kW3 = 5120, kWeights = 6144;
constexpr uint32_t kB2 = 6144, kB3 = 6208, kParams = 6224;
constexpr uint32_t kLossSlot = kParams;           // gradient arrays carry the loss after the parameters
constexpr uint32_t kPartialStride = 6240;         // floats per CTA partial

struct AdamStep {
    float lr, beta1, beta2, eps;
    float bias1, bias2;   // 1 - beta^step
};

cudaError_t init(void);   // function attributes; call once outside stream capture
uint64_t scratch_bytes(uint32_t max_samples);
// bf16 weights into scratch (first kWeights * 2 bytes); run after every parameter change.
cudaError_t pack(const float* params, void* scratch, cudaStream_t s);
// y[n][y_cols] = net(x[n][16]); n from n_dev when non-null (then max_n bounds the grid).
cudaError_t forward(const float* params, const float* x, uint32_t n, const uint32_t* n_dev, uint32_t max_n, float* y,
                    uint32_t y_cols, void* scratch, uint32_t* error_flags, cudaStream_t s);
// Gradient of (1/n) sum_s sum_o out_w[o] (y_so - t_so)^2 into grad[kParams + 1] (loss last);
// with update_params non-null, one Adam step on update_params (moments m, v).
cudaError_t gradient(const float* params, const float* x, const float* t, const float* out_w, uint32_t n, void* scratch,
                     float* grad, float* loss_out, float* m, float* v, float* update_params, const AdamStep& a,
                     uint32_t* error_flags, cudaStream_t s);

}  // namespace mlp
}  // namespace mk
