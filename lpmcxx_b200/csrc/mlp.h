// The order-selection MLP: 8 features -> 64 -> 64 -> 12 classes, GELU activations.
// Classes 0..10 are Taylor orders 1..11, class 11 is "no order up to 11 meets the budget".
//
// Parameter vector (FP32, kMlpParams floats), in this order:
//   W1[64][8], b1[64], W2[64][64], b2[64], W3[12][64], b3[12], mean[8], inv_std[8]
// The last 16 values standardise the features, x' = (x - mean) * inv_std; they are fixed from the
// training set, not trained.  Inference (mlp_warp_argmax) runs on the tensor cores: BF16 weights and
// activations, FP32 accumulation.
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

// GELU of the inference path: erf by Abramowitz & Stegun 7.1.26, erf(u) = 1 - (a1 t + ... + a5 t^5) exp(-u^2),
// t = 1 / (1 + p u) for u >= 0 (odd extension), |error| <= 1.5e-7, with the approximate reciprocal and exp2
// (one MUFU op each).  The activations it feeds are rounded to BF16 (relative step 2^-8), so this matches
// gelu_f up to rounding ties; it takes about half the instructions of erff, and the selector's hidden layers
// evaluate 128 activations per lane per call.
__device__ __forceinline__ float gelu_fast(float x) {
    const float u = fabsf(x) * 0.70710678118654752f;
    float t, g;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(t) : "f"(fmaf(0.3275911f, u, 1.0f)));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(g) : "f"(-u * u * 1.4426950408889634f));  // exp(-u^2)
    const float poly = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f),
                                0.254829592f);
    const float erf_u = fmaf(-poly, g, 1.0f);  // erf(|x| / sqrt 2)
    return 0.5f * x * (1.0f + copysignf(erf_u, x));
}

// Convert host FP32 parameters (kMlpParams) to device BF16 weights w_dev (kMlpParams) and FP32
// standardisation norm_dev (2 * kMlpIn).  Synchronous.
int mlp_upload_bf16(lpm_ctx* ctx, const float* params_host, __nv_bfloat16* w_dev, float* norm_dev);

// ---------------------------------------------------------------------------------------------------
// Warp-cooperative inference on the tensor cores: the 32 lanes' feature vectors form a 32 x 8 batch,
// each layer is a 32 x K by K x N product done with mma.sync m16n8k16 (BF16 operands, FP32 accumulation),
// the FP32 accumulators of one layer become, after bias and GELU, the BF16 A operands of the next
// (the accumulator layout of two adjacent n-tiles is the A layout of one k-step).  Activations are
// rounded to BF16 between layers; weights are BF16.  All 32 lanes must call it (lanes without a pair
// pass any finite features and ignore the result).  xs: 32 x 16 BF16 of per-warp shared memory.

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One hidden layer: A (2 m-tiles x KS k-steps of 16) times W^T (W: 64 x in_dim rows, BF16) plus bias,
// GELU, repacked as the next layer's A (2 m-tiles x 4 k-steps).
template <int KS>
__device__ __forceinline__ void mlp_warp_hidden(const uint32_t (&a)[2][KS][4], const __nv_bfloat16* __restrict__ W,
                                                int in_dim, const __nv_bfloat16* __restrict__ bias, int lane,
                                                uint32_t (&out)[2][4][4]) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const __nv_bfloat16* wr = W + (size_t)(8 * nt + g) * in_dim;  // row n = 8 nt + g of W
        float acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const int k0 = 16 * ks + 2 * t;
            const uint32_t b0 = k0 < in_dim ? *reinterpret_cast<const uint32_t*>(wr + k0) : 0u;
            const uint32_t b1 = k0 + 8 < in_dim ? *reinterpret_cast<const uint32_t*>(wr + k0 + 8) : 0u;
            mma_bf16_16816(acc[0], a[0][ks], b0, b1);
            mma_bf16_16816(acc[1], a[1][ks], b0, b1);
        }
        const float bb0 = __bfloat162float(bias[8 * nt + 2 * t]), bb1 = __bfloat162float(bias[8 * nt + 2 * t + 1]);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const uint32_t lo = pack_bf16x2(gelu_fast(acc[mt][0] + bb0), gelu_fast(acc[mt][1] + bb1));  // row g
            const uint32_t hi = pack_bf16x2(gelu_fast(acc[mt][2] + bb0), gelu_fast(acc[mt][3] + bb1));  // row g + 8
            // n-tile nt is half (nt & 1) of k-step nt / 2 of the next layer
            out[mt][nt >> 1][(nt & 1) ? 2 : 0] = lo;
            out[mt][nt >> 1][(nt & 1) ? 3 : 1] = hi;
        }
    }
}

__device__ __forceinline__ int mlp_warp_argmax(const __nv_bfloat16* __restrict__ w, const float* __restrict__ norm,
                                               const float* f, __nv_bfloat16* xs) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // standardised features of this lane's pair -> row `lane` of xs (K padded to 16 with zeros)
#pragma unroll
    for (int i = 0; i < 16; ++i)
        xs[lane * 16 + i] = __float2bfloat16_rn(i < kMlpIn ? (f[i] - norm[i]) * norm[kMlpIn + i] : 0.0f);
    __syncwarp();
    uint32_t a0[2][1][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const __nv_bfloat16* r0 = xs + (16 * mt + g) * 16;
        const __nv_bfloat16* r1 = xs + (16 * mt + g + 8) * 16;
        a0[mt][0][0] = *reinterpret_cast<const uint32_t*>(r0 + 2 * t);
        a0[mt][0][1] = *reinterpret_cast<const uint32_t*>(r1 + 2 * t);
        a0[mt][0][2] = *reinterpret_cast<const uint32_t*>(r0 + 2 * t + 8);
        a0[mt][0][3] = *reinterpret_cast<const uint32_t*>(r1 + 2 * t + 8);
    }
    uint32_t a1[2][4][4], a2[2][4][4];
    mlp_warp_hidden<1>(a0, w + kOffW1, kMlpIn, w + kOffB1, lane, a1);
    mlp_warp_hidden<4>(a1, w + kOffW2, kMlpHidden, w + kOffB2, lane, a2);
    // output layer: 12 classes in two n-tiles (columns 12..15 are zero weights and ignored)
    float z[2][2][4];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        const int n = 8 * nt + g;
        const __nv_bfloat16* wr = w + kOffW3 + (size_t)(n < kMlpOut ? n : 0) * kMlpHidden;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) z[mt][nt][0] = z[mt][nt][1] = z[mt][nt][2] = z[mt][nt][3] = 0.0f;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const int k0 = 16 * ks + 2 * t;
            const uint32_t b0 = n < kMlpOut ? *reinterpret_cast<const uint32_t*>(wr + k0) : 0u;
            const uint32_t b1 = n < kMlpOut ? *reinterpret_cast<const uint32_t*>(wr + k0 + 8) : 0u;
            mma_bf16_16816(z[0][nt], a2[0][ks], b0, b1);
            mma_bf16_16816(z[1][nt], a2[1][ks], b0, b1);
        }
    }
    // per row: arg-max over the 4 columns this thread holds, then over the 4 threads of its group
    int my = 0;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float bv = -3.0e38f;
            int bi = 0;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int col = 8 * nt + 2 * t + j;
                    if (col < kMlpOut) {
                        const float v = z[mt][nt][2 * half + j] + __bfloat162float(w[kOffB3 + col]);
                        if (v > bv) {
                            bv = v;
                            bi = col;
                        }
                    }
                }
#pragma unroll
            for (int o = 1; o < 4; o <<= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > bv || (ov == bv && oi < bi)) {
                    bv = ov;
                    bi = oi;
                }
            }
            // group g now holds the class of row 16 mt + 8 half + g; lane l takes row l's from group l & 7
            const int v = __shfl_sync(0xffffffffu, bi, 4 * (lane & 7));
            if ((lane >> 4) == mt && ((lane >> 3) & 1) == half) my = v;
        }
    __syncwarp();
    return my;
}

}  // namespace lpm
