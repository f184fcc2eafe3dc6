// Context, error reporting and scratch memory.  A context stands in for the reference's
// per-rank MPI state (MPIReplicatedData + MPI_COMM_WORLD): one device, one stream, and the
// device buffers the solvers reuse between calls.
#include "lpm_internal.h"

#include <cstdarg>
#include <cstring>
#include <new>

namespace lpm {

namespace {
thread_local char g_err[512] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
    set_error("CUDA error in %s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return LPM_ERR_OOM;
    return LPM_ERR_CUDA;
}

void* scratch(lpm_ctx* ctx, int slot, size_t bytes) {
    if (slot < 0 || slot >= kSlotCount) {
        set_error("bad scratch slot %d", slot);
        return nullptr;
    }
    LpmBuffer& b = ctx->buf[slot];
    if (bytes == 0) bytes = 256;
    if (b.bytes >= bytes) return b.ptr;
    if (b.ptr) {
        // the old contents may still be read by queued work
        cudaStreamSynchronize(ctx->stream);
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 8;  // grow with headroom
    want = (want + 255) & ~size_t(255);
    if (cudaMalloc(&b.ptr, want) != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        set_error("device allocation of %zu bytes failed (scratch slot %d)", want, slot);
        return nullptr;
    }
    b.bytes = want;
    return b.ptr;
}

void* pinned(lpm_ctx* ctx, size_t bytes) {
    if (ctx->pinned_bytes >= bytes) return ctx->pinned;
    if (ctx->pinned) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
    }
    size_t want = (bytes + bytes / 8 + 4095) & ~size_t(4095);
    if (cudaMallocHost(&ctx->pinned, want) != cudaSuccess) {
        cudaGetLastError();
        ctx->pinned = nullptr;
        set_error("pinned host allocation of %zu bytes failed", want);
        return nullptr;
    }
    ctx->pinned_bytes = want;
    return ctx->pinned;
}

}  // namespace lpm

extern "C" {

const char* lpm_last_error(void) { return lpm::g_err; }

int lpm_ctx_create(int device, lpm_ctx** out) {
    if (!out) {
        lpm::set_error("lpm_ctx_create: null output pointer");
        return LPM_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        lpm::set_error("no CUDA device available");
        return LPM_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) {
        lpm::set_error("device %d out of range (have %d)", device, ndev);
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    LPM_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        lpm::set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return LPM_ERR_NO_DEVICE;
    }
    lpm_ctx* c = new (std::nothrow) lpm_ctx();
    if (!c) {
        lpm::set_error("host allocation failed");
        return LPM_ERR_OOM;
    }
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return lpm::cuda_status(e, "cudaStreamCreate");
    }
    c->stream = c->own_stream;
    *out = c;
    return LPM_OK;
}

int lpm_ctx_destroy(lpm_ctx* ctx) {
    if (!ctx) return LPM_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->buf)
        if (b.ptr) cudaFree(b.ptr);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return LPM_OK;
}

int lpm_ctx_set_stream(lpm_ctx* ctx, void* cuda_stream) {
    if (!ctx) {
        lpm::set_error("null context");
        return LPM_ERR_ARG;
    }
    ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    return LPM_OK;
}

int lpm_ctx_synchronize(lpm_ctx* ctx) {
    if (!ctx) {
        lpm::set_error("null context");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return LPM_OK;
}

int64_t lpm_ctx_launch_count(const lpm_ctx* ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"
