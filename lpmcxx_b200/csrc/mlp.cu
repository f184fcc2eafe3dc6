// Training and inference kernels of the order-selection MLP (layout in mlp.h).
//
// Training: softmax cross-entropy over the 12 classes, mini-batch Adam.  One block handles 64 samples:
// forward and backward per sample (one thread each, activations in shared memory), then the block forms
// its parameter gradients as sums over its samples (one thread per parameter slice, no atomics) and a
// second kernel adds the blocks' partial gradients in a fixed order and applies the Adam update, so a
// training run is deterministic.
#include "lpm_internal.h"
#include "mlp.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

namespace lpm {
namespace {

constexpr int kTrainBlock = 64;  // samples (threads) per block
// per-sample rows padded to odd strides: thread s reading row s and thread p reading column p of the
// same row both hit distinct shared-memory banks
constexpr int kSX = kMlpIn + 1, kSH = kMlpHidden + 1, kSZ = kMlpOut + 1;
constexpr int kTrainSmemFloats = kMlpParams + kTrainBlock * (kSX + 4 * kSH + kSZ + 1);

__device__ __forceinline__ float gelu_grad(float a) {
    const float cdf = 0.5f * (1.0f + erff(a * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * a * a);
    return cdf + a * pdf;
}

struct TrainArgs {
    const float* params;
    const float* feats;     // n x 8
    const int32_t* labels;  // n
    const int32_t* order;   // sample order (permutation) or null
    int64_t n, start;
    int nb;                 // samples in this mini-batch
    float scale;            // 1 / nb
    float* partial;         // gridDim x kMlpTrainable
    float* loss_partial;    // gridDim
};

__global__ void __launch_bounds__(kTrainBlock) mlp_fwd_bwd_kernel(TrainArgs A) {
    extern __shared__ float sm[];
    float* W = sm;
    float* X = W + kMlpParams;
    float* A1 = X + kTrainBlock * kSX;
    float* H1 = A1 + kTrainBlock * kSH;
    float* A2 = H1 + kTrainBlock * kSH;
    float* H2 = A2 + kTrainBlock * kSH;
    float* DZ = H2 + kTrainBlock * kSH;
    float* LS = DZ + kTrainBlock * kSZ;
    for (int i = threadIdx.x; i < kMlpParams; i += kTrainBlock) W[i] = A.params[i];
    __syncthreads();
    const int s = threadIdx.x;
    const int64_t k = (int64_t)blockIdx.x * kTrainBlock + s;
    const bool valid = k < A.nb && A.start + k < A.n;
    int64_t id = 0;
    int label = 0;
    float* x = X + s * kSX;
    if (valid) {
        id = A.order ? A.order[A.start + k] : A.start + k;
        label = A.labels[id];
    }
    for (int i = 0; i < kMlpIn; ++i)
        x[i] = valid ? (A.feats[id * kMlpIn + i] - W[kOffMean + i]) * W[kOffInvStd + i] : 0.0f;
    float* a1 = A1 + s * kSH;
    float* h1 = H1 + s * kSH;
    float* a2 = A2 + s * kSH;
    float* h2 = H2 + s * kSH;
    float* dz = DZ + s * kSZ;
    for (int o = 0; o < kMlpHidden; ++o) {
        float a = W[kOffB1 + o];
        for (int i = 0; i < kMlpIn; ++i) a = fmaf(W[kOffW1 + o * kMlpIn + i], x[i], a);
        a1[o] = a;
        h1[o] = gelu_f(a);
    }
    for (int o = 0; o < kMlpHidden; ++o) {
        float a = W[kOffB2 + o];
        for (int i = 0; i < kMlpHidden; ++i) a = fmaf(W[kOffW2 + o * kMlpHidden + i], h1[i], a);
        a2[o] = a;
        h2[o] = gelu_f(a);
    }
    float zmax = -3.0e38f;
    for (int o = 0; o < kMlpOut; ++o) {
        float a = W[kOffB3 + o];
        for (int i = 0; i < kMlpHidden; ++i) a = fmaf(W[kOffW3 + o * kMlpHidden + i], h2[i], a);
        dz[o] = a;
        zmax = fmaxf(zmax, a);
    }
    float zs = 0.0f;
    for (int o = 0; o < kMlpOut; ++o) {
        dz[o] = expf(dz[o] - zmax);
        zs += dz[o];
    }
    const float inv = 1.0f / zs;
    LS[s] = valid ? -logf(fmaxf(dz[label] * inv, 1e-30f)) : 0.0f;
    for (int o = 0; o < kMlpOut; ++o) dz[o] = valid ? (dz[o] * inv - (o == label ? 1.0f : 0.0f)) * A.scale : 0.0f;
    // back-propagate through layers 3 and 2 (da2 overwrites a2, da1 overwrites a1)
    for (int j = 0; j < kMlpHidden; ++j) {
        float g = 0.0f;
        for (int o = 0; o < kMlpOut; ++o) g = fmaf(W[kOffW3 + o * kMlpHidden + j], dz[o], g);
        a2[j] = g * gelu_grad(a2[j]);
    }
    for (int j = 0; j < kMlpHidden; ++j) {
        float g = 0.0f;
        for (int o = 0; o < kMlpHidden; ++o) g = fmaf(W[kOffW2 + o * kMlpHidden + j], a2[o], g);
        a1[j] = g * gelu_grad(a1[j]);
    }
    __syncthreads();
    // parameter gradients of this block: sums over its samples
    float* out = A.partial + (size_t)blockIdx.x * kMlpTrainable;
    for (int p = threadIdx.x; p < kMlpTrainable; p += kTrainBlock) {
        float g = 0.0f;
        if (p < kOffB1) {
            const int o = p / kMlpIn, i = p % kMlpIn;
            for (int q = 0; q < kTrainBlock; ++q) g = fmaf(A1[q * kSH + o], X[q * kSX + i], g);
        } else if (p < kOffW2) {
            const int o = p - kOffB1;
            for (int q = 0; q < kTrainBlock; ++q) g += A1[q * kSH + o];
        } else if (p < kOffB2) {
            const int o = (p - kOffW2) / kMlpHidden, i = (p - kOffW2) % kMlpHidden;
            for (int q = 0; q < kTrainBlock; ++q) g = fmaf(A2[q * kSH + o], H1[q * kSH + i], g);
        } else if (p < kOffW3) {
            const int o = p - kOffB2;
            for (int q = 0; q < kTrainBlock; ++q) g += A2[q * kSH + o];
        } else if (p < kOffB3) {
            const int o = (p - kOffW3) / kMlpHidden, i = (p - kOffW3) % kMlpHidden;
            for (int q = 0; q < kTrainBlock; ++q) g = fmaf(DZ[q * kSZ + o], H2[q * kSH + i], g);
        } else {
            const int o = p - kOffB3;
            for (int q = 0; q < kTrainBlock; ++q) g += DZ[q * kSZ + o];
        }
        out[p] = g;
    }
    if (threadIdx.x == 0) {
        float l = 0.0f;
        for (int q = 0; q < kTrainBlock; ++q) l += LS[q];
        A.loss_partial[blockIdx.x] = l;
    }
}

// Sum the blocks' partial gradients in block order; optionally write the gradient out and apply Adam.
__global__ void mlp_reduce_adam_kernel(float* __restrict__ params, const float* __restrict__ partial, int nblocks,
                                       float* __restrict__ m, float* __restrict__ v, float lr, float b1t, float b2t,
                                       float* __restrict__ grad_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpTrainable) return;
    float g = 0.0f;
    for (int b = 0; b < nblocks; ++b) g += partial[(size_t)b * kMlpTrainable + p];
    if (grad_out) grad_out[p] = g;
    if (lr > 0.0f) {
        const float beta1 = 0.9f, beta2 = 0.999f;
        const float mm = beta1 * m[p] + (1.0f - beta1) * g;
        const float vv = beta2 * v[p] + (1.0f - beta2) * g * g;
        m[p] = mm;
        v[p] = vv;
        const float mh = mm / (1.0f - b1t), vh = vv / (1.0f - b2t);
        params[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
    }
}

__global__ void mlp_to_bf16_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kMlpParams) w[p] = __float2bfloat16_rn(params[p]);
}

// The treecode's inference path (mlp_warp_argmax): 32 samples per warp on the tensor cores.
__global__ void __launch_bounds__(128) mlp_predict_bf16_kernel(const __nv_bfloat16* __restrict__ w,
                                                               const float* __restrict__ norm,
                                                               const float* __restrict__ feats, int64_t n,
                                                               int32_t* __restrict__ cls) {
    __shared__ __align__(16) __nv_bfloat16 xs[4][32 * 16];
    const int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    if (base >= n) return;  // uniform per warp
    const int64_t i = base + (threadIdx.x & 31);
    float f[kMlpIn];
    for (int k = 0; k < kMlpIn; ++k) f[k] = i < n ? feats[i * kMlpIn + k] : norm[k];
    const int c = mlp_warp_argmax(w, norm, f, xs[threadIdx.x >> 5]);
    if (i < n) cls[i] = c;
}

int train_smem_bytes() { return kTrainSmemFloats * (int)sizeof(float); }

}  // namespace

int mlp_upload_bf16(lpm_ctx* ctx, const float* params_host, __nv_bfloat16* w_dev, float* norm_dev) {
    float* tmp = (float*)scratch(ctx, kSlotMisc0, kMlpParams * sizeof(float));
    if (!tmp) return LPM_ERR_OOM;
    LPM_CUDA_TRY(cudaMemcpyAsync(tmp, params_host, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_LAUNCH(ctx, "mlp_to_bf16_kernel", mlp_to_bf16_kernel, grid_for(kMlpParams, 256), 256, 0, tmp, w_dev);
    LPM_CUDA_TRY(cudaMemcpyAsync(norm_dev, params_host + kOffMean, 2 * kMlpIn * sizeof(float), cudaMemcpyHostToDevice,
                                 ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return LPM_OK;
}

}  // namespace lpm

using namespace lpm;

namespace {

// One pass over `n` samples in mini-batches of `nb` (order: optional permutation); lr <= 0 computes the
// mean-loss gradient of a single batch holding all samples.
int mlp_pass(lpm_ctx* ctx, float* d_params, const float* d_feats, const int32_t* d_labels, const int32_t* d_order,
             int64_t n, int nb, float lr, float* d_m, float* d_v, int64_t* step, float* loss_sum, float* d_grad) {
    const int nblk_max = (nb + kTrainBlock - 1) / kTrainBlock;
    float* partial = (float*)scratch(ctx, kSlotMisc1, (size_t)nblk_max * kMlpTrainable * sizeof(float));
    float* lpart = (float*)scratch(ctx, kSlotMisc2, (size_t)nblk_max * sizeof(float) + 256);
    if (!partial || !lpart) return LPM_ERR_OOM;
    LPM_CUDA_TRY(cudaFuncSetAttribute(mlp_fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      train_smem_bytes()));
    std::vector<float> lp(nblk_max);
    double total = 0.0;
    for (int64_t s0 = 0; s0 < n; s0 += nb) {
        const int cur = (int)std::min<int64_t>(nb, n - s0);
        const int nblk = (cur + kTrainBlock - 1) / kTrainBlock;
        TrainArgs A{d_params, d_feats, d_labels, d_order, n, s0, cur, 1.0f / (float)cur, partial, lpart};
        LPM_LAUNCH(ctx, "mlp_fwd_bwd_kernel", mlp_fwd_bwd_kernel, nblk, kTrainBlock, train_smem_bytes(), A);
        *step += 1;
        const float b1t = powf(0.9f, (float)*step), b2t = powf(0.999f, (float)*step);
        LPM_LAUNCH(ctx, "mlp_reduce_adam_kernel", mlp_reduce_adam_kernel, grid_for(kMlpTrainable, 256), 256, 0,
                   d_params, partial, nblk, d_m, d_v, lr, b1t, b2t, d_grad);
        LPM_CUDA_TRY(cudaMemcpyAsync(lp.data(), lpart, nblk * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (int b = 0; b < nblk; ++b) total += lp[b];
    }
    *loss_sum = (float)total;
    return LPM_OK;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int lpm_mlp_train(lpm_ctx* ctx, const float* feats, const int32_t* labels, int64_t n, int epochs,
                             int minibatch, float lr, uint64_t seed, float* params, float* loss_out) {
    if (!ctx || !feats || !labels || !params || n <= 0 || n >= INT32_MAX || epochs < 0 || minibatch < 1 ||
        !(lr > 0.0f)) {
        set_error("lpm_mlp_train: bad argument");
        return LPM_ERR_ARG;
    }
    for (int64_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kMlpOut) {
            set_error("lpm_mlp_train: label %d out of range at %lld", labels[i], (long long)i);
            return LPM_ERR_ARG;
        }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    DevBuf bp, bf, bl, bo, bm, bv;
    LPM_CUDA_TRY(cudaMalloc(&bp.p, kMlpParams * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bf.p, (size_t)n * kMlpIn * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bl.p, (size_t)n * sizeof(int32_t)));
    LPM_CUDA_TRY(cudaMalloc(&bo.p, (size_t)n * sizeof(int32_t)));
    LPM_CUDA_TRY(cudaMalloc(&bm.p, kMlpTrainable * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bv.p, kMlpTrainable * sizeof(float)));
    LPM_CUDA_TRY(cudaMemcpyAsync(bp.p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(bf.p, feats, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(bl.p, labels, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    LPM_CUDA_TRY(cudaMemsetAsync(bm.p, 0, kMlpTrainable * sizeof(float), ctx->stream));
    LPM_CUDA_TRY(cudaMemsetAsync(bv.p, 0, kMlpTrainable * sizeof(float), ctx->stream));
    std::vector<int32_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    int64_t step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        LPM_CUDA_TRY(cudaMemcpyAsync(bo.p, order.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice,
                                     ctx->stream));
        float loss = 0.0f;
        int rc = mlp_pass(ctx, (float*)bp.p, (const float*)bf.p, (const int32_t*)bl.p, (const int32_t*)bo.p, n,
                          minibatch, lr, (float*)bm.p, (float*)bv.p, &step, &loss, nullptr);
        if (rc) return rc;
        if (loss_out) loss_out[ep] = loss / (float)n;
    }
    LPM_CUDA_TRY(cudaMemcpyAsync(params, bp.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return LPM_OK;
}

extern "C" int lpm_mlp_grad(lpm_ctx* ctx, const float* params, const float* feats, const int32_t* labels, int64_t n,
                            float* grad, float* loss) {
    if (!ctx || !params || !feats || !labels || !grad || n <= 0 || n > (1 << 20)) {
        set_error("lpm_mlp_grad: bad argument");
        return LPM_ERR_ARG;
    }
    for (int64_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kMlpOut) {
            set_error("lpm_mlp_grad: label %d out of range at %lld", labels[i], (long long)i);
            return LPM_ERR_ARG;
        }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    DevBuf bp, bf, bl, bg;
    LPM_CUDA_TRY(cudaMalloc(&bp.p, kMlpParams * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bf.p, (size_t)n * kMlpIn * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bl.p, (size_t)n * sizeof(int32_t)));
    LPM_CUDA_TRY(cudaMalloc(&bg.p, kMlpTrainable * sizeof(float)));
    LPM_CUDA_TRY(cudaMemcpyAsync(bp.p, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(bf.p, feats, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(bl.p, labels, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    int64_t step = 0;
    float l = 0.0f;
    int rc = mlp_pass(ctx, (float*)bp.p, (const float*)bf.p, (const int32_t*)bl.p, nullptr, n, (int)n, 0.0f, nullptr,
                      nullptr, &step, &l, (float*)bg.p);
    if (rc) return rc;
    LPM_CUDA_TRY(cudaMemcpyAsync(grad, bg.p, kMlpTrainable * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = l / (float)n;
    return LPM_OK;
}

extern "C" int lpm_mlp_predict(lpm_ctx* ctx, const float* params, const float* feats, int64_t n, int32_t* classes) {
    if (!ctx || !params || (n > 0 && (!feats || !classes)) || n < 0) {
        set_error("lpm_mlp_predict: bad argument");
        return LPM_ERR_ARG;
    }
    if (n == 0) return LPM_OK;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    DevBuf bw, bn, bf, bc;
    LPM_CUDA_TRY(cudaMalloc(&bw.p, kMlpParams * sizeof(__nv_bfloat16)));
    LPM_CUDA_TRY(cudaMalloc(&bn.p, 2 * kMlpIn * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bf.p, (size_t)n * kMlpIn * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bc.p, (size_t)n * sizeof(int32_t)));
    int rc = mlp_upload_bf16(ctx, params, (__nv_bfloat16*)bw.p, (float*)bn.p);
    if (rc) return rc;
    LPM_CUDA_TRY(cudaMemcpyAsync(bf.p, feats, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    LPM_LAUNCH(ctx, "mlp_predict_bf16_kernel", mlp_predict_bf16_kernel, grid_for(n, 128), 128, 0,
               (const __nv_bfloat16*)bw.p, (const float*)bn.p, (const float*)bf.p, n, (int32_t*)bc.p);
    LPM_CUDA_TRY(cudaMemcpyAsync(classes, bc.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return LPM_OK;
}
