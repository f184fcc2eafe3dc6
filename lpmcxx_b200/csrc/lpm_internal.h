// Internal declarations shared by the library's translation units.
#pragma once

#include "../../include/lpm_b200.h"

#include <cstdint>
#include <cstdio>
#include <string>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#include <vector>
#endif

namespace lpm {

// Thread-local last-error message behind lpm_last_error().
void set_error(const char* fmt, ...);

}  // namespace lpm

#ifdef __CUDACC__

// A growable device buffer owned by a context.  Buffers only grow; they are freed with the
// context.  Growth happens outside any stream capture (the RK4 graph is captured after warm-up).
struct LpmBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// One profiled launch: events recorded around it on the launching stream.
struct LpmProfRecord {
    const char* name;
    cudaEvent_t start, stop;
};

struct lpm_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    // per-kernel CUDA-event timing (lpm_ctx_set_profiling); off by default and never on during capture
    bool profiling = false;
    std::vector<LpmProfRecord>* prof = nullptr;
    // scratch slots, indexed by the enum below
    LpmBuffer buf[32];
    // pinned host staging (host-facing entry points)
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // incremented whenever a scratch slot is reallocated: a CUDA graph captured before holds the old address
    uint64_t generation = 0;
    // FP32 direct sums: targets per thread of the tile kernels (2, 4 or 8; lpm_ctx_set_param "direct_targets")
    int direct_tpt = 4;
};

namespace lpm {

enum ScratchSlot {
    kSlotSrcPack = 0,   // packed sources (double4)
    kSlotTgtPack,       // packed targets (double4)
    kSlotOut,           // outputs (component-major)
    kSlotSrc32,         // FP32 source copies
    kSlotTgt32,         // FP32 target copies
    kSlotMisc0,
    kSlotMisc1,
    kSlotMisc2,
    kSlotMisc3,
    kSlotTree0,
    kSlotTree1,
    kSlotTree2,
    kSlotTree3,
    kSlotTree4,
    kSlotTree5,
    kSlotTree6,
    kSlotTree7,
    kSlotTree8,
    kSlotTree9,
    kSlotTree10,
    kSlotTree11,
    kSlotTree12,
    kSlotSideCounts,    // radix digit counts of the target sort (runs on a second stream beside the tree build)
    kSlotSideSums,      // scan block sums of the same
    kSlotRk0,
    kSlotRk1,
    kSlotRk2,
    kSlotRk3,
    kSlotRk4,
    kSlotRk5,
    kSlotCount
};

// Ensure ctx scratch slot `slot` holds at least `bytes`; returns nullptr (and sets the error)
// on allocation failure.
void* scratch(lpm_ctx* ctx, int slot, size_t bytes);
void* pinned(lpm_ctx* ctx, size_t bytes);

int cuda_status(cudaError_t e, const char* what);
// cudaMalloc through the library's allocation-failure injection point (lpm_debug_fail_allocations).
cudaError_t dev_alloc(void** p, size_t bytes);

#define LPM_CUDA_TRY(call)                                              \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::lpm::cuda_status(e_, #call);    \
    } while (0)

#define LPM_LAUNCH_CHECK(ctx)                                           \
    do {                                                                \
        (ctx)->launches += 1;                                           \
        cudaError_t e_ = cudaGetLastError();                            \
        if (e_ != cudaSuccess) return ::lpm::cuda_status(e_, "kernel launch"); \
    } while (0)

// Launch `kernel<<<grid, block, smem, ctx->stream>>>(args...)`, count it, and when profiling is on
// bracket it with CUDA events on the same stream under `name`.
#define LPM_LAUNCH(ctx, name, kernel, grid, block, smem, ...)                                 \
    do {                                                                                      \
        ::LpmProfRecord rec_{name, nullptr, nullptr};                                    \
        if ((ctx)->profiling) ::lpm::prof_begin(ctx, rec_);                                   \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);                      \
        if ((ctx)->profiling) ::lpm::prof_end(ctx, rec_);                                     \
        LPM_LAUNCH_CHECK(ctx);                                                                \
    } while (0)

void prof_begin(lpm_ctx* ctx, LpmProfRecord& r);
void prof_end(lpm_ctx* ctx, LpmProfRecord& r);

inline unsigned grid_for(int64_t n, int per_block) { return (unsigned)((n + per_block - 1) / per_block); }

// direct sums (direct_sum.cu)
// FP64 sums; a singular scalar kernel skips source coinc_off + i for target i < coinc_n.
int direct_sum_f64(lpm_ctx* ctx, const lpm_kernel_desc& k, const double4* src, int64_t n_src, const double4* tgt,
                   int64_t n_tgt, double* out, int64_t out_stride, int64_t coinc_n = 0, int64_t coinc_off = 0);
// FP32 sums: src.w = 2*strength for Biot-Savart; targets 0..coinc_n-1 sit on sources coinc_off.. .
int direct_sum_f32_impl(lpm_ctx* ctx, const lpm_kernel_desc& k, const float4* src, int64_t n_src, const float4* tgt,
                        const double4* tgt64, int64_t n_tgt, double* out, int64_t out_stride, int64_t coinc_n,
                        int64_t coinc_off);
int direct_sum_any(lpm_ctx* ctx, const lpm_kernel_desc& k, int precision, const double4* src, int64_t n_src,
                   const double4* tgt, int64_t n_tgt, double* out, int64_t coinc_n, int64_t coinc_off);
int pack_f32(lpm_ctx* ctx, const double4* in, int64_t n, float4* out, bool scale_w2);
int check_kernel_desc(const lpm_kernel_desc* k);
int check_f32_kind(const lpm_kernel_desc& k);  // LPM_ERR_KERNEL unless Biot-Savart or 3D Poisson

// Packed FP32 (fma.rn.f32x2, sm_100): two FP32 FMAs in one instruction, each lane rounded like fmaf.
// (d0, d1) = (a0 b + c0, a1 b + c1).
__device__ __forceinline__ void fma2p(float& d0, float& d1, float a0, float a1, float b, float c0, float c1) {
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %4};\n\tmov.b64 rc, {%5, %6};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b), "f"(c0), "f"(c1));
}

// (d0, d1) = (a0 b0 + c0, a1 b1 + c1).
__device__ __forceinline__ void fma2v(float& d0, float& d1, float a0, float a1, float b0, float b1, float c0,
                                      float c1) {
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b0), "f"(b1), "f"(c0), "f"(c1));
}

}  // namespace lpm

#endif  // __CUDACC__
