// RK4 stage loop for Lagrangian particles on the sphere.
//
// The reference's C++ tree has no time integrator (the RK4 solver of the Fortran original is only
// described in README.md:75).  This file defines the build's semantics, restated identically by
// the CPU oracle: vertices and face-centroid particles move independently, each carrying a constant
// strength; stage velocities come from a full solver evaluation at the stage positions; stage
// positions and the new position are re-projected onto the sphere x <- R x/|x|.
//
//   k1 = u(X)                 X1 = P(X + dt/2 k1)
//   k2 = u(X1)                X2 = P(X + dt/2 k2)
//   k3 = u(X2)                X3 = P(X + dt   k3)
//   k4 = u(X3)                X <- P(X + dt/6 (k1 + 2 k2 + 2 k3 + k4))
//
// One fused update kernel per stage accumulates k, forms the next stage position in FP64 and writes
// the FP32 copy the FP32 solvers read.  A whole step can be captured once into a CUDA graph and
// replayed.
#include "lpm_internal.h"
#include "treecode.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

struct lpm_rk4 {
    lpm_ctx* ctx = nullptr;
    lpm_kernel_desc kernel{};
    lpm_solver_desc solver{};
    int64_t n_src = 0, n = 0;
    double4* X = nullptr;    // state (x, y, z, w)
    double4* Xs = nullptr;   // stage position
    float4* Xs32 = nullptr;  // FP32 copy of the stage position (w pre-scaled for the kernel)
    double* U = nullptr;     // stage velocity, 3 x n
    double* K = nullptr;     // k1 + 2 k2 + 2 k3, 3 x n
    lpm::TreeSolver* tree = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    int64_t graph_nodes = 0;
    bool warmed = false;
    lpm_ensemble* owner = nullptr;  // the ensemble whose captured step replays this instance, if any
    uint64_t graph_ctx_gen = 0, graph_tree_gen = 0;  // buffer generations the graph was captured with
};

namespace lpm {
// Drops the owning ensemble's captured step (its launches hold this instance's parameters); ensemble.cu.
int ensemble_invalidate(lpm_ensemble* e);

namespace {

__global__ void rk4_update_kernel(double4* __restrict__ X, double4* __restrict__ Xs, float4* __restrict__ Xs32,
                                  const double* __restrict__ U, double* __restrict__ K, int64_t n, int stage,
                                  double dt, double radius, float wscale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double u0 = U[i], u1 = U[n + i], u2 = U[2 * n + i];
    const double4 x = X[i];
    double a, v0, v1, v2;
    if (stage == 1) {
        K[i] = u0; K[n + i] = u1; K[2 * n + i] = u2;
        a = 0.5 * dt; v0 = u0; v1 = u1; v2 = u2;
    } else if (stage < 4) {
        const double k0 = K[i] + 2.0 * u0, k1 = K[n + i] + 2.0 * u1, k2 = K[2 * n + i] + 2.0 * u2;
        K[i] = k0; K[n + i] = k1; K[2 * n + i] = k2;
        a = stage == 2 ? 0.5 * dt : dt; v0 = u0; v1 = u1; v2 = u2;
    } else {
        a = dt / 6.0;
        v0 = K[i] + u0; v1 = K[n + i] + u1; v2 = K[2 * n + i] + u2;
    }
    double px = x.x + a * v0, py = x.y + a * v1, pz = x.z + a * v2;
    const double s = radius / sqrt(px * px + py * py + pz * pz);
    px *= s; py *= s; pz *= s;
    const double4 p = make_double4(px, py, pz, x.w);
    if (stage == 4) X[i] = p;
    Xs[i] = p;
    if (Xs32) Xs32[i] = make_float4((float)px, (float)py, (float)pz, (float)(x.w * wscale));
}

__global__ void copy_state_kernel(const double4* __restrict__ X, double4* __restrict__ Xs, float4* __restrict__ Xs32,
                                  int64_t n, float wscale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = X[i];
    Xs[i] = p;
    if (Xs32) Xs32[i] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)(p.w * wscale));
}

float wscale_for(const lpm_kernel_desc& k) { return k.kind == LPM_KERNEL_BIOT_SAVART_SPHERE ? 2.0f : 1.0f; }

}  // namespace

// Velocity of every particle (3 x n, component-major) at positions Xs / Xs32.
int rk4_velocity(lpm_rk4* rk, double* U) {
    lpm_ctx* ctx = rk->ctx;
    if (rk->solver.method == LPM_METHOD_DIRECT) {
        if (rk->solver.precision == LPM_PREC_F64)
            return direct_sum_f64(ctx, rk->kernel, rk->Xs, rk->n_src, rk->Xs, rk->n, U, rk->n);
        return direct_sum_f32_impl(ctx, rk->kernel, rk->Xs32, rk->n_src, rk->Xs32, rk->Xs, rk->n, U, rk->n, rk->n_src,
                                   0);
    }
    return tree_velocity(rk->tree, rk->Xs, rk->n_src, rk->Xs, rk->n, U);
}

// The stage update from the stage velocity U: accumulates k, forms the next stage position (stage 4: the new
// state).
int rk4_stage_update(lpm_rk4* rk, int stage, double dt) {
    lpm_ctx* ctx = rk->ctx;
    LPM_LAUNCH(ctx, "rk4_update_kernel", rk4_update_kernel, grid_for(rk->n, 256), 256, 0, rk->X, rk->Xs, rk->Xs32,
               rk->U, rk->K, rk->n, stage, dt, rk->kernel.radius, wscale_for(rk->kernel));
    return LPM_OK;
}

static int rk4_one_step(lpm_rk4* rk, double dt) {
    for (int stage = 1; stage <= 4; ++stage) {
        int rc = rk4_velocity(rk, rk->U);
        if (rc) return rc;
        rc = rk4_stage_update(rk, stage, dt);
        if (rc) return rc;
    }
    return LPM_OK;
}

// The stage velocity of the fused ensemble step up to the far and near fields, which the ensemble's fused
// launches add (treecode instances); a direct-sum instance computes its whole stage velocity here.
int rk4_stage_begin(lpm_rk4* rk) {
    if (rk->tree) return tree_fused_prepare(rk->tree, rk->Xs, rk->Xs, rk->U);
    return rk4_velocity(rk, rk->U);
}
TreeSolver* rk4_tree(lpm_rk4* rk) { return rk->tree; }
double* rk4_stage_velocity(lpm_rk4* rk) { return rk->U; }

// One uncaptured-or-captured RK4 step of rk on its context's current stream (for the ensemble).
int rk4_step_enqueue(lpm_rk4* rk, double dt) { return rk4_one_step(rk, dt); }
// Generations of the buffers a step of rk uses (its context's scratch, its treecode's arrays).
uint64_t rk4_buffer_generation(const lpm_rk4* rk) {
    return rk->ctx->generation * 1000003ull + (rk->tree ? tree_generation(rk->tree) : 0);
}
lpm_ctx* rk4_context(lpm_rk4* rk) { return rk->ctx; }
int rk4_tree_check(lpm_rk4* rk) { return rk->tree ? tree_check(rk->tree) : LPM_OK; }
void rk4_set_owner(lpm_rk4* rk, lpm_ensemble* e) { rk->owner = e; }
int rk4_set_param_internal(lpm_rk4* rk, const char* name, double value) {
    if (!rk->tree) {
        set_error("ensemble: the instances do not use the treecode");
        return LPM_ERR_ARG;
    }
    return tree_set_param(rk->tree, name, value);
}
int rk4_set_mlp_internal(lpm_rk4* rk, const float* params) {
    if (!rk->tree) {
        set_error("ensemble: the instances do not use the treecode");
        return LPM_ERR_ARG;
    }
    return tree_set_mlp(rk->tree, params);
}

static void drop_graph(lpm_rk4* rk) {
    if (rk->graph_exec) cudaGraphExecDestroy(rk->graph_exec);
    if (rk->graph) cudaGraphDestroy(rk->graph);
    rk->graph_exec = nullptr;
    rk->graph = nullptr;
    rk->graph_nodes = 0;
}

static int capture_step(lpm_rk4* rk, double dt) {
    lpm_ctx* ctx = rk->ctx;
    drop_graph(rk);
    // capture on the context's own stream (the legacy default stream cannot capture)
    cudaStream_t user = ctx->stream;
    LPM_CUDA_TRY(cudaStreamSynchronize(user));
    ctx->stream = ctx->own_stream;
    const int64_t before = ctx->launches;
    const bool prof = ctx->profiling;
    ctx->profiling = false;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        ctx->stream = user;
        ctx->profiling = prof;
        return cuda_status(e, "cudaStreamBeginCapture");
    }
    int rc = rk4_one_step(rk, dt);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->stream = user;
    ctx->launches = before;
    ctx->profiling = prof;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    rk->graph = g;
    size_t nodes = 0;
    LPM_CUDA_TRY(cudaGraphGetNodes(g, nullptr, &nodes));
    rk->graph_nodes = (int64_t)nodes;
    LPM_CUDA_TRY(cudaGraphInstantiate(&rk->graph_exec, g, 0));
    rk->graph_dt = dt;
    rk->graph_ctx_gen = ctx->generation;
    rk->graph_tree_gen = rk->tree ? tree_generation(rk->tree) : 0;
    return LPM_OK;
}

}  // namespace lpm

using namespace lpm;

extern "C" int lpm_rk4_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver,
                              int64_t n_src, int64_t n_pts, lpm_rk4** out) {
    if (!ctx || !out || !solver) {
        set_error("lpm_rk4_create: null argument");
        return LPM_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    if (kernel->kind != LPM_KERNEL_BIOT_SAVART_SPHERE) {
        set_error("invalid kernel: RK4 advects particles with a vector kernel");
        return LPM_ERR_KERNEL;
    }
    if (n_src < 0 || n_pts < n_src || n_pts <= 0) {
        set_error("lpm_rk4_create: need 0 <= n_src <= n_pts, n_pts > 0");
        return LPM_ERR_ARG;
    }
    if (solver->method != LPM_METHOD_DIRECT && solver->method != LPM_METHOD_TREE) {
        set_error("lpm_rk4_create: unknown method %d", solver->method);
        return LPM_ERR_ARG;
    }
    if (solver->precision != LPM_PREC_F64 && solver->precision != LPM_PREC_F32) {
        set_error("lpm_rk4_create: unknown precision %d", solver->precision);
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    lpm_rk4* rk = new (std::nothrow) lpm_rk4();
    if (!rk) return LPM_ERR_OOM;
    rk->ctx = ctx;
    rk->kernel = *kernel;
    rk->solver = *solver;
    rk->n_src = n_src;
    rk->n = n_pts;
    const size_t n = (size_t)n_pts;
    cudaError_t e = cudaSuccess;
    e = dev_alloc((void**)&rk->X, n * sizeof(double4));
    if (e == cudaSuccess) e = dev_alloc((void**)&rk->Xs, n * sizeof(double4));
    if (e == cudaSuccess) e = dev_alloc((void**)&rk->Xs32, n * sizeof(float4));
    if (e == cudaSuccess) e = dev_alloc((void**)&rk->U, 3 * n * sizeof(double));
    if (e == cudaSuccess) e = dev_alloc((void**)&rk->K, 3 * n * sizeof(double));
    if (e != cudaSuccess) {
        lpm_rk4_destroy(rk);
        return cuda_status(e, "cudaMalloc (RK4 state)");
    }
    if (solver->method == LPM_METHOD_TREE) {
        rc = tree_solver_create(ctx, *kernel, *solver, n_src, n_pts, &rk->tree);
        // the source octree's root is Box3d(maxR) of the vertex particles, as TreeSum's mesh constructor
        // (src/LpmTreeSum.cpp:221-238) takes maxR of the mesh vertices
        if (!rc && n_pts > n_src) rc = tree_set_param(rk->tree, "root_first", (double)n_src);
        if (rc) {
            lpm_rk4_destroy(rk);
            return rc;
        }
    }
    *out = rk;
    return LPM_OK;
}

extern "C" int lpm_rk4_destroy(lpm_rk4* rk) {
    if (!rk) return LPM_OK;
    cudaSetDevice(rk->ctx->device);
    cudaStreamSynchronize(rk->ctx->stream);
    drop_graph(rk);
    if (rk->tree) tree_solver_destroy(rk->tree);
    cudaFree(rk->X);
    cudaFree(rk->Xs);
    cudaFree(rk->Xs32);
    cudaFree(rk->U);
    cudaFree(rk->K);
    delete rk;
    return LPM_OK;
}

static int refresh_stage(lpm_rk4* rk) {
    lpm_ctx* ctx = rk->ctx;
    LPM_LAUNCH(ctx, "copy_state_kernel", copy_state_kernel, grid_for(rk->n, 256), 256, 0, rk->X, rk->Xs, rk->Xs32,
               rk->n, wscale_for(rk->kernel));
    return LPM_OK;
}

extern "C" int lpm_rk4_set_state_dev(lpm_rk4* rk, const double* xyzw) {
    if (!rk || !xyzw) {
        set_error("lpm_rk4_set_state_dev: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaMemcpyAsync(rk->X, xyzw, (size_t)rk->n * sizeof(double4), cudaMemcpyDeviceToDevice,
                                 rk->ctx->stream));
    return refresh_stage(rk);
}

extern "C" int lpm_rk4_get_state_dev(lpm_rk4* rk, double* xyzw) {
    if (!rk || !xyzw) {
        set_error("lpm_rk4_get_state_dev: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaMemcpyAsync(xyzw, rk->X, (size_t)rk->n * sizeof(double4), cudaMemcpyDeviceToDevice,
                                 rk->ctx->stream));
    return LPM_OK;
}

extern "C" int lpm_rk4_set_state(lpm_rk4* rk, const double* xyzw) {
    if (!rk || !xyzw) {
        set_error("lpm_rk4_set_state: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaMemcpyAsync(rk->X, xyzw, (size_t)rk->n * sizeof(double4), cudaMemcpyHostToDevice,
                                 rk->ctx->stream));
    int rc = refresh_stage(rk);
    if (rc) return rc;
    LPM_CUDA_TRY(cudaStreamSynchronize(rk->ctx->stream));
    return LPM_OK;
}

extern "C" int lpm_rk4_get_state(lpm_rk4* rk, double* xyzw) {
    if (!rk || !xyzw) {
        set_error("lpm_rk4_get_state: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaMemcpyAsync(xyzw, rk->X, (size_t)rk->n * sizeof(double4), cudaMemcpyDeviceToHost,
                                 rk->ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(rk->ctx->stream));
    return LPM_OK;
}

extern "C" int lpm_rk4_step(lpm_rk4* rk, double dt, int nsteps, int use_graph) {
    if (!rk || nsteps < 0 || !std::isfinite(dt)) {
        set_error("lpm_rk4_step: bad argument");
        return LPM_ERR_ARG;
    }
    lpm_ctx* ctx = rk->ctx;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    int s = 0;
    if (use_graph && !rk->warmed && nsteps > 0) {
        // the first step runs uncaptured so every scratch buffer reaches its final size
        int rc = rk4_one_step(rk, dt);
        if (rc) return rc;
        rk->warmed = true;
        s = 1;
    }
    if (!use_graph) {
        for (; s < nsteps; ++s) {
            int rc = rk4_one_step(rk, dt);
            if (rc) return rc;
        }
        rk->warmed = true;
        return LPM_OK;
    }
    // a graph holds the buffer addresses of its capture: after any reallocation (an uncaptured evaluation
    // regrew the interaction lists, the per-node arrays or a scratch slot) it is captured again
    const bool stale = rk->graph_exec && (rk->graph_ctx_gen != ctx->generation ||
                                          (rk->tree && rk->graph_tree_gen != tree_generation(rk->tree)));
    if (s < nsteps && (!rk->graph_exec || rk->graph_dt != dt || stale)) {
        int rc = capture_step(rk, dt);
        if (rc) return rc;
    }
    for (; s < nsteps; ++s) {
        LPM_CUDA_TRY(cudaGraphLaunch(rk->graph_exec, ctx->stream));
        ctx->launches += rk->graph_nodes;
    }
    // replays cannot grow the treecode's buffers: report an overflow instead of returning wrong data
    if (rk->tree) return tree_check(rk->tree);
    return LPM_OK;
}

extern "C" int lpm_rk4_tree_stats(lpm_rk4* rk, int64_t* out10) {
    if (!rk || !out10) {
        set_error("lpm_rk4_tree_stats: null argument");
        return LPM_ERR_ARG;
    }
    if (!rk->tree) {
        set_error("lpm_rk4_tree_stats: the integrator does not use the treecode");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    return tree_stats(rk->tree, out10);
}

extern "C" int lpm_rk4_set_mlp(lpm_rk4* rk, const float* params) {
    if (!rk || !rk->tree) {
        set_error("lpm_rk4_set_mlp: the integrator does not use the treecode");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaStreamSynchronize(rk->ctx->stream));
    if (rk->owner) {
        int rc = ensemble_invalidate(rk->owner);
        if (rc) return rc;
    }
    drop_graph(rk);
    rk->warmed = false;  // the next graph step first runs uncaptured so the lists can resize
    return tree_set_mlp(rk->tree, params);
}

extern "C" int lpm_rk4_set_param(lpm_rk4* rk, const char* name, double value) {
    if (!rk || !rk->tree) {
        set_error("lpm_rk4_set_param: the integrator does not use the treecode");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    LPM_CUDA_TRY(cudaStreamSynchronize(rk->ctx->stream));
    if (rk->owner) {
        int rc = ensemble_invalidate(rk->owner);
        if (rc) return rc;
    }
    drop_graph(rk);
    rk->warmed = false;  // the next graph step first runs uncaptured so the lists can resize
    return tree_set_param(rk->tree, name, value);
}

extern "C" int lpm_rk4_get_param(const lpm_rk4* rk, const char* name, double* value) {
    if (!rk || !rk->tree) {
        set_error("lpm_rk4_get_param: the integrator does not use the treecode");
        return LPM_ERR_ARG;
    }
    return tree_get_param(rk->tree, name, value);
}

extern "C" int lpm_rk4_source_tree(lpm_rk4* rk, lpm_tree** out) {
    if (!rk || !out || !rk->tree) {
        set_error("lpm_rk4_source_tree: null argument, or the integrator does not use the treecode");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    int64_t n = 0;
    const Octree& t = tree_source_octree(rk->tree, &n);
    return tree_view_create(rk->ctx, t, n, out);
}

extern "C" int lpm_rk4_velocity_dev(lpm_rk4* rk, double* out) {
    if (!rk || !out) {
        set_error("lpm_rk4_velocity_dev: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(rk->ctx->device));
    int rc = refresh_stage(rk);
    if (rc) return rc;
    return rk4_velocity(rk, out);
}

// ---------------------------------------------------------------------------------- checkpoint / resume
// File layout (host byte order): "LPMCKPT" + NUL, uint32 version (1), uint32 instance count, int64 step,
// double t, double dt; per instance int64 particle count, int64 source count and the particles as n x 4
// doubles (x, y, z, w); then the 64-bit FNV-1a checksum of every byte before it.  The state is all an RK4 step
// reads (stage positions and accumulators are rebuilt from it), so a resumed run steps bitwise as the one that
// wrote the file.
namespace lpm {
namespace {
constexpr char kCkptMagic[8] = {'L', 'P', 'M', 'C', 'K', 'P', 'T', '\0'};
constexpr uint32_t kCkptVersion = 1;

struct CkptFile {
    FILE* f = nullptr;
    uint64_t h = 1469598103934665603ull;  // FNV-1a offset basis
    bool ok = true;
    ~CkptFile() {
        if (f) std::fclose(f);
    }
    void hash(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    }
    void put(const void* p, size_t n) {
        if (ok && std::fwrite(p, 1, n, f) != n) ok = false;
        hash(p, n);
    }
    void get(void* p, size_t n) {
        if (ok && std::fread(p, 1, n, f) != n) ok = false;
        if (ok) hash(p, n);
    }
};
}  // namespace

int ckpt_write(const char* path, lpm_rk4* const* rks, int n_inst, int64_t step, double t, double dt) {
    if (!path || n_inst < 1) {
        set_error("checkpoint: bad argument");
        return LPM_ERR_ARG;
    }
    std::vector<std::vector<double>> states((size_t)n_inst);
    for (int i = 0; i < n_inst; ++i) {  // read every state before the file is touched
        states[i].resize((size_t)rks[i]->n * 4);
        int rc = lpm_rk4_get_state(rks[i], states[i].data());
        if (rc) return rc;
    }
    CkptFile c;
    c.f = std::fopen(path, "wb");
    if (!c.f) {
        set_error("checkpoint: cannot open '%s' for writing", path);
        return LPM_ERR_ARG;
    }
    const uint32_t head[2] = {kCkptVersion, (uint32_t)n_inst};
    c.put(kCkptMagic, sizeof(kCkptMagic));
    c.put(head, sizeof(head));
    c.put(&step, sizeof(step));
    c.put(&t, sizeof(t));
    c.put(&dt, sizeof(dt));
    for (int i = 0; i < n_inst; ++i) {
        const int64_t sizes[2] = {rks[i]->n, rks[i]->n_src};
        c.put(sizes, sizeof(sizes));
        c.put(states[i].data(), states[i].size() * sizeof(double));
    }
    const uint64_t sum = c.h;
    c.put(&sum, sizeof(sum));
    if (!c.ok || std::fflush(c.f) != 0) {
        set_error("checkpoint: writing '%s' failed", path);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

int ckpt_read(const char* path, lpm_rk4* const* rks, int n_inst, int64_t* step, double* t, double* dt) {
    if (!path || n_inst < 1) {
        set_error("checkpoint: bad argument");
        return LPM_ERR_ARG;
    }
    CkptFile c;
    c.f = std::fopen(path, "rb");
    if (!c.f) {
        set_error("checkpoint: cannot open '%s'", path);
        return LPM_ERR_ARG;
    }
    char magic[8];
    uint32_t head[2];
    int64_t s = 0;
    double tt = 0.0, dd = 0.0;
    c.get(magic, sizeof(magic));
    c.get(head, sizeof(head));
    c.get(&s, sizeof(s));
    c.get(&tt, sizeof(tt));
    c.get(&dd, sizeof(dd));
    if (!c.ok || std::memcmp(magic, kCkptMagic, sizeof(magic)) != 0 || head[0] != kCkptVersion) {
        set_error("checkpoint: '%s' is not an RK4 checkpoint of this library", path);
        return LPM_ERR_ARG;
    }
    if ((int)head[1] != n_inst) {
        set_error("checkpoint: '%s' holds %u instances, not %d", path, head[1], n_inst);
        return LPM_ERR_ARG;
    }
    std::vector<std::vector<double>> states((size_t)n_inst);
    for (int i = 0; i < n_inst && c.ok; ++i) {
        int64_t sizes[2] = {0, 0};
        c.get(sizes, sizeof(sizes));
        if (!c.ok) break;
        if (sizes[0] != rks[i]->n || sizes[1] != rks[i]->n_src) {
            set_error("checkpoint: instance %d of '%s' has %lld particles / %lld sources, not %lld / %lld", i, path,
                      (long long)sizes[0], (long long)sizes[1], (long long)rks[i]->n, (long long)rks[i]->n_src);
            return LPM_ERR_ARG;
        }
        states[i].resize((size_t)sizes[0] * 4);
        c.get(states[i].data(), states[i].size() * sizeof(double));
    }
    const uint64_t want = c.h;
    uint64_t sum = 0;
    if (c.ok) {
        if (std::fread(&sum, 1, sizeof(sum), c.f) != sizeof(sum)) c.ok = false;
    }
    if (!c.ok || sum != want || std::fgetc(c.f) != EOF) {
        set_error("checkpoint: '%s' is truncated, corrupted or longer than its contents", path);
        return LPM_ERR_ARG;
    }
    for (int i = 0; i < n_inst; ++i) {  // the states change only once the whole file checked out
        int rc = lpm_rk4_set_state(rks[i], states[i].data());
        if (rc) return rc;
    }
    if (step) *step = s;
    if (t) *t = tt;
    if (dt) *dt = dd;
    return LPM_OK;
}
}  // namespace lpm

extern "C" int lpm_rk4_checkpoint_write(lpm_rk4* rk, const char* path, int64_t step, double t, double dt) {
    if (!rk) {
        set_error("lpm_rk4_checkpoint_write: null RK4");
        return LPM_ERR_ARG;
    }
    return ckpt_write(path, &rk, 1, step, t, dt);
}

extern "C" int lpm_rk4_checkpoint_read(lpm_rk4* rk, const char* path, int64_t* step, double* t, double* dt) {
    if (!rk) {
        set_error("lpm_rk4_checkpoint_read: null RK4");
        return LPM_ERR_ARG;
    }
    return ckpt_read(path, &rk, 1, step, t, dt);
}
