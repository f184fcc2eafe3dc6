// The order-selection MLP: 8 features -> 64 -> 64 -> 12 classes, GELU activations.
// Classes 0..10 are Taylor orders 1..11, class 11 is "no order up to 11 meets the budget".
//
// Parameter vector (FP32, kMlpParams floats), in this order:
//   W1[64][8], b1[64], W2[64][64], b2[64], W3[12][64], b3[12], mean[8], inv_std[8]
// The last 16 values standardise the features, x' = (x - mean) * inv_std; they are fixed from the
// training set, not trained.  Inference keeps the weights in BF16 and accumulates in FP32.
#pragma once

#include "lpm_internal.h"

#include <cuda_bf16.h>
#include <cstdint>

namespace lpm {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 12;
constexpr int kMlpDirectClass = 11;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHidden;
constexpr int kOffMean = kOffB3 + kMlpOut;
constexpr int kOffInvStd = kOffMean + kMlpIn;
constexpr int kMlpTrainable = kOffMean;          // 5516 trained parameters
constexpr int kMlpParams = kOffInvStd + kMlpIn;  // 5532 floats in total

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// Convert host FP32 parameters (kMlpParams) to device BF16 weights w_dev (kMlpParams) and FP32
// standardisation norm_dev (2 * kMlpIn).  Synchronous.
int mlp_upload_bf16(lpm_ctx* ctx, const float* params_host, __nv_bfloat16* w_dev, float* norm_dev);

// Arg-max class of one feature vector: BF16 weights w (layout above; the standardisation entries are
// not read from it), FP32 standardisation `norm` = {mean[8], inv_std[8]}, FP32 accumulation.  The second
// hidden layer is streamed into the output logits one unit at a time, so only the first layer's 64
// activations stay live.
__device__ __forceinline__ int mlp_argmax_bf16(const __nv_bfloat16* __restrict__ w, const float* __restrict__ norm,
                                               const float* f) {
    float x[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) x[i] = (f[i] - norm[i]) * norm[kMlpIn + i];
    float h1[kMlpHidden];
#pragma unroll
    for (int o = 0; o < kMlpHidden; ++o) {
        float a = __bfloat162float(w[kOffB1 + o]);
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) a = fmaf(__bfloat162float(w[kOffW1 + o * kMlpIn + i]), x[i], a);
        h1[o] = gelu_f(a);
    }
    float z[kMlpOut];
#pragma unroll
    for (int c = 0; c < kMlpOut; ++c) z[c] = __bfloat162float(w[kOffB3 + c]);
#pragma unroll 1
    for (int o = 0; o < kMlpHidden; ++o) {
        float a = __bfloat162float(w[kOffB2 + o]);
        const __nv_bfloat162* row = reinterpret_cast<const __nv_bfloat162*>(w + kOffW2 + o * kMlpHidden);
#pragma unroll
        for (int i = 0; i < kMlpHidden / 2; ++i) {
            const float2 v = __bfloat1622float2(row[i]);
            a = fmaf(v.x, h1[2 * i], a);
            a = fmaf(v.y, h1[2 * i + 1], a);
        }
        const float h = gelu_f(a);
#pragma unroll
        for (int c = 0; c < kMlpOut; ++c) z[c] = fmaf(__bfloat162float(w[kOffW3 + c * kMlpHidden + o]), h, z[c]);
    }
    int best = 0;
    float bv = z[0];
#pragma unroll
    for (int c = 1; c < kMlpOut; ++c)
        if (z[c] > bv) {
            bv = z[c];
            best = c;
        }
    return best;
}

}  // namespace lpm
