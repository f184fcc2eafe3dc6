// Allocation-free FP32 direct sum.
//
// Some callers cannot allocate device memory at call time: hosts whose memory pool is reserved up front
// (a solver embedded in a larger simulation whose own allocator owns every byte of the device, so a
// cudaMalloc here would fail or steal from it), and real-time loops that may not block on the allocator
// or grow the process's device footprint after start-up.  The regular FP32 entry point (lpm_direct_sum_dev with LPM_PREC_F32) converts its FP64
// inputs into FP32 copies held in per-context scratch that it grows with cudaMalloc.  This variant keeps
// those copies in one file-scope device array instead, so it allocates nothing: the caller passes the
// inputs, the output and a stream, and no context is needed.
//
// Limits and sharing: sources + targets together may hold at most kStaticScratchPoints points
// (8 MiB of float4 per device, reserved by every GPU that loads this library until the process exits);
// larger calls are rejected with LPM_ERR_CAPACITY.  Every call on a device uses the same array, so calls
// whose work overlaps on the GPU (different streams, or different host threads) race on it and must be
// serialised by the caller.  The array keeps the previous call's contents; each call overwrites every
// entry it reads before reading it, so nothing has to start at zero.
#include "lpm_internal.h"

#include <mutex>

namespace lpm {
namespace {

constexpr int64_t kStaticScratchPoints = 1 << 19;  // float4 entries (8 MiB)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float4 g_static_scratch[kStaticScratchPoints];

std::mutex g_setup_mutex;
float4* g_scratch_addr[kMaxDevices] = {};

// The array's device address on `device` (the host-side name is only a stand-in, never a device
// address).  Looked up once per device with that device current.
int scratch_address(int device, float4** out) {
    if (device < 0 || device >= kMaxDevices) {
        set_error("device %d out of range for the static scratch table", device);
        return LPM_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress (static scratch)");
        g_scratch_addr[device] = (float4*)p;
    }
    *out = g_scratch_addr[device];
    return LPM_OK;
}

}  // namespace
}  // namespace lpm

using namespace lpm;

extern "C" int lpm_direct_sum_f32_noalloc(const lpm_kernel_desc* kernel, const double* src, int64_t n_src,
                                          const double* tgt, int64_t n_tgt, int64_t n_coincident, double* out,
                                          void* cuda_stream) {
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    rc = check_f32_kind(*kernel);
    if (rc) return rc;
    if (n_src < 0 || n_tgt < 0 || (n_src > 0 && !src) || (n_tgt > 0 && (!tgt || !out)) || n_coincident < 0 ||
        n_coincident > std::min(n_src, n_tgt)) {
        set_error("lpm_direct_sum_f32_noalloc: bad sizes or null pointers");
        return LPM_ERR_ARG;
    }
    if (n_src + n_tgt > kStaticScratchPoints) {
        set_error("lpm_direct_sum_f32_noalloc: %lld sources + %lld targets exceed the static scratch of %lld points",
                  (long long)n_src, (long long)n_tgt, (long long)kStaticScratchPoints);
        return LPM_ERR_CAPACITY;
    }
    int device = 0;
    LPM_CUDA_TRY(cudaGetDevice(&device));
    float4* s32 = nullptr;
    rc = scratch_address(device, &s32);
    if (rc) return rc;
    float4* t32 = s32 + n_src;
    // a context on the stack: launches only, no buffers, no profiling events
    lpm_ctx local;
    local.device = device;
    local.stream = (cudaStream_t)cuda_stream;
    rc = pack_f32(&local, (const double4*)src, n_src, s32, kernel->kind == LPM_KERNEL_BIOT_SAVART_SPHERE);
    if (rc) return rc;
    rc = pack_f32(&local, (const double4*)tgt, n_tgt, t32, false);
    if (rc) return rc;
    return direct_sum_f32_impl(&local, *kernel, s32, n_src, t32, (const double4*)tgt, n_tgt, out, n_tgt, n_coincident,
                               0);
}
