// Context, error reporting and scratch memory.  A context stands in for the reference's
// per-rank MPI state (MPIReplicatedData + MPI_COMM_WORLD): one device, one stream, and the
// device buffers the solvers reuse between calls.
#include "lpm_internal.h"

#include <atomic>
#include <string>

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

// Allocation-failure injection for tests: after `g_fail_after` more successful device allocations, the next
// one reports cudaErrorMemoryAllocation without allocating (once; negative = off).
static std::atomic<int64_t> g_fail_after{-1};

cudaError_t dev_alloc(void** p, size_t bytes) {
    int64_t v = g_fail_after.load();
    while (v >= 0) {
        if (g_fail_after.compare_exchange_weak(v, v - 1)) {
            if (v == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
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
    ++ctx->generation;  // graphs captured with the old address must be captured again
    size_t want = bytes + bytes / 8;  // grow with headroom
    want = (want + 255) & ~size_t(255);
    if (dev_alloc(&b.ptr, want) != cudaSuccess) {
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

void prof_begin(lpm_ctx* ctx, LpmProfRecord& r) {
    if (cudaEventCreate(&r.start) != cudaSuccess || cudaEventCreate(&r.stop) != cudaSuccess) {
        cudaGetLastError();
        r.start = r.stop = nullptr;
        return;
    }
    cudaEventRecord(r.start, ctx->stream);
}

void prof_end(lpm_ctx* ctx, LpmProfRecord& r) {
    if (!r.start) return;
    cudaEventRecord(r.stop, ctx->stream);
    if (!ctx->prof) ctx->prof = new std::vector<LpmProfRecord>();
    ctx->prof->push_back(r);
}

static void prof_clear(lpm_ctx* ctx) {
    if (!ctx->prof) return;
    for (auto& r : *ctx->prof) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    ctx->prof->clear();
}

}  // namespace lpm

extern "C" {

int lpm_ctx_set_profiling(lpm_ctx* ctx, int on) {
    if (!ctx) {
        lpm::set_error("null context");
        return LPM_ERR_ARG;
    }
    cudaStreamSynchronize(ctx->stream);
    lpm::prof_clear(ctx);
    ctx->profiling = on != 0;
    return LPM_OK;
}

int lpm_ctx_profile_report(lpm_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || len == 0) {
        lpm::set_error("lpm_ctx_profile_report: bad argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    // aggregate by kernel name, in first-seen order
    std::vector<const char*> names;
    std::vector<double> ms;
    std::vector<int64_t> count;
    if (ctx->prof) {
        for (auto& r : *ctx->prof) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, r.start, r.stop) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            size_t k = 0;
            while (k < names.size() && std::strcmp(names[k], r.name) != 0) ++k;
            if (k == names.size()) {
                names.push_back(r.name);
                ms.push_back(0.0);
                count.push_back(0);
            }
            ms[k] += t;
            count[k] += 1;
        }
    }
    size_t off = (size_t)snprintf(buf, len, "{");
    for (size_t k = 0; k < names.size() && off < len; ++k)
        off += (size_t)snprintf(buf + off, len - off, "%s\"%s\": {\"ms\": %.6f, \"launches\": %lld}", k ? ", " : "",
                                names[k], ms[k], (long long)count[k]);
    if (off < len) snprintf(buf + off, len - off, "}");
    lpm::prof_clear(ctx);
    return LPM_OK;
}

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
    lpm::prof_clear(ctx);
    delete ctx->prof;
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
    ctx->stream = (cudaStream_t)cuda_stream;
    return LPM_OK;
}

void* lpm_ctx_own_stream(const lpm_ctx* ctx) { return ctx ? (void*)ctx->own_stream : nullptr; }

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

extern "C" int lpm_debug_fail_allocations(int64_t after) {
    lpm::g_fail_after.store(after < 0 ? -1 : after);
    return LPM_OK;
}

extern "C" int lpm_ctx_set_param(lpm_ctx* ctx, const char* name, double value) {
    if (!ctx || !name) {
        lpm::set_error("lpm_ctx_set_param: null argument");
        return LPM_ERR_ARG;
    }
    const std::string n(name);
    if (n == "direct_targets" && (value == 2.0 || value == 4.0 || value == 8.0)) {
        ctx->direct_tpt = (int)value;
        return LPM_OK;
    }
    lpm::set_error("lpm_ctx_set_param: unknown parameter or value out of range: %s = %g", name, value);
    return LPM_ERR_ARG;
}

extern "C" int lpm_ctx_get_param(const lpm_ctx* ctx, const char* name, double* value) {
    if (!ctx || !name || !value) {
        lpm::set_error("lpm_ctx_get_param: null argument");
        return LPM_ERR_ARG;
    }
    if (std::string(name) == "direct_targets") {
        *value = ctx->direct_tpt;
        return LPM_OK;
    }
    lpm::set_error("lpm_ctx_get_param: unknown parameter %s", name);
    return LPM_ERR_ARG;
}
