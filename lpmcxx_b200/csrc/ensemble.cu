// Ensembles: many independent RK4 problems of uneven sizes advanced together.
//
// The instances are spread over `lanes` streams, each with its own library context (so concurrently
// running instances never share scratch memory); a lane runs its instances one after the other.  The
// assignment is longest-processing-time-first by an n log n size estimate, so that the lanes finish
// together.  After one uncaptured step (which sizes every buffer), one RK4 step of every instance is
// captured into a single CUDA graph that forks onto the lanes and joins back, and the graph is replayed
// once per step: small instances (20k particles) that cannot fill a B200 alone overlap with each other
// and with the large ones.
//
// Fused mode (the default; set_param "fused"): each RK4 stage forks onto the lanes for every instance's
// tree build, moments and interaction lists, joins, and then the far field of ALL instances runs as one
// persistent launch per Taylor order and the near field as one persistent launch per near tile shape
// (TreeFused, treecode.cu), whose blocks take (instance, batch) items in decreasing order of work over the
// whole ensemble; the stage updates fork onto the lanes again.  The results are bitwise those of the lane
// mode.  Without it, each instance's far and near launches run on its lane.  With fused_groups = G > 1 the
// lanes (and so the instances, balanced by the lane assignment) form G groups that step independently on
// their own streams, each with its own fused launches: one group's tree builds and traversals (latency-bound
// chains of small launches) overlap another group's far and near fields.
#include "lpm_internal.h"
#include "treecode.h"

#include <algorithm>
#include <cmath>
#include <new>
#include <numeric>
#include <string>
#include <vector>

namespace lpm {
int rk4_step_enqueue(lpm_rk4* rk, double dt);
lpm_ctx* rk4_context(lpm_rk4* rk);
int rk4_tree_check(lpm_rk4* rk);
int rk4_set_mlp_internal(lpm_rk4* rk, const float* params);
int rk4_set_param_internal(lpm_rk4* rk, const char* name, double value);
uint64_t rk4_buffer_generation(const lpm_rk4* rk);
void rk4_set_owner(lpm_rk4* rk, lpm_ensemble* e);
int ensemble_invalidate(lpm_ensemble* e);
int rk4_stage_begin(lpm_rk4* rk);
int rk4_stage_update(lpm_rk4* rk, int stage, double dt);
TreeSolver* rk4_tree(lpm_rk4* rk);
double* rk4_stage_velocity(lpm_rk4* rk);
}  // namespace lpm

using namespace lpm;

struct lpm_ensemble {
    lpm_ctx* ctx = nullptr;            // the caller's context: its own stream carries the graph
    std::vector<lpm_ctx*> lanes;       // one context (and stream) per lane
    std::vector<lpm_rk4*> inst;
    std::vector<int> lane_of;
    std::vector<cudaEvent_t> join;     // per lane
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double graph_dt = 0.0;
    int64_t graph_nodes = 0;
    bool warmed = false;
    std::vector<uint64_t> graph_gen;   // per instance: buffer generation at capture
    bool fused = true;                 // far and near fields of all instances in fused launches
    int groups = 2;                    // fused: groups of lanes stepping independently (set_param "fused_groups")
    std::vector<TreeFused*> fz;        // per group: the fused launches' tables
    std::vector<cudaStream_t> gstream; // per group g >= 1: its stream (group 0 uses the ensemble's stream)
    std::vector<cudaEvent_t> gfork, gjoin;  // per group: fork from / join into the ensemble's stream
};

// Whether any instance reallocated a buffer since the ensemble's graph was captured.
static bool ens_graph_stale(const lpm_ensemble* e) {
    if (e->graph_gen.size() != e->inst.size()) return true;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (e->graph_gen[i] != rk4_buffer_generation(e->inst[i])) return true;
    return false;
}

static void ens_drop_graph(lpm_ensemble* e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
    e->graph_nodes = 0;
}

namespace lpm {
// An instance's parameters or selector changed: the captured step holds launches with the old ones (and
// lists sized for them), so drop it; the next graph step first runs uncaptured to resize the lists.
int ensemble_invalidate(lpm_ensemble* e) {
    LPM_CUDA_TRY(cudaSetDevice(e->ctx->device));
    for (lpm_ctx* c : e->lanes) LPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(e->ctx->own_stream));
    ens_drop_graph(e);
    e->warmed = false;
    return LPM_OK;
}
}  // namespace lpm

extern "C" int lpm_ensemble_destroy(lpm_ensemble* e) {
    if (!e) return LPM_OK;
    cudaSetDevice(e->ctx->device);
    for (lpm_ctx* c : e->lanes) cudaStreamSynchronize(c->stream);
    ens_drop_graph(e);
    for (lpm_rk4* r : e->inst) lpm_rk4_destroy(r);
    for (cudaEvent_t ev : e->join) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    for (lpm_ctx* c : e->lanes) lpm_ctx_destroy(c);
    for (TreeFused* f : e->fz) tree_fused_destroy(f);
    for (cudaStream_t st : e->gstream)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : e->gfork) cudaEventDestroy(ev);
    for (cudaEvent_t ev : e->gjoin) cudaEventDestroy(ev);
    delete e;
    return LPM_OK;
}

static int ensemble_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solvers,
                           int solver_stride, int n_inst, const int64_t* n_src, const int64_t* n_pts, int lanes,
                           lpm_ensemble** out);

extern "C" int lpm_ensemble_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver,
                                   int n_inst, const int64_t* n_src, const int64_t* n_pts, int lanes,
                                   lpm_ensemble** out) {
    return ensemble_create(ctx, kernel, solver, 0, n_inst, n_src, n_pts, lanes, out);
}

extern "C" int lpm_ensemble_create_each(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solvers,
                                        int n_inst, const int64_t* n_src, const int64_t* n_pts, int lanes,
                                        lpm_ensemble** out) {
    return ensemble_create(ctx, kernel, solvers, 1, n_inst, n_src, n_pts, lanes, out);
}

static int ensemble_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver,
                           int solver_stride, int n_inst, const int64_t* n_src, const int64_t* n_pts, int lanes,
                           lpm_ensemble** out) {
    if (!ctx || !kernel || !solver || !n_src || !n_pts || !out || n_inst < 1 || lanes < 1 || lanes > 64) {
        set_error("lpm_ensemble_create: bad argument (1 <= lanes <= 64, n_inst >= 1)");
        return LPM_ERR_ARG;
    }
    *out = nullptr;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    lpm_ensemble* e = new (std::nothrow) lpm_ensemble();
    if (!e) return LPM_ERR_OOM;
    e->ctx = ctx;
    lanes = std::min(lanes, n_inst);
    for (int l = 0; l < lanes; ++l) {
        lpm_ctx* c = nullptr;
        int rc = lpm_ctx_create(ctx->device, &c);
        if (rc) {
            lpm_ensemble_destroy(e);
            return rc;
        }
        e->lanes.push_back(c);
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            lpm_ensemble_destroy(e);
            return cuda_status(cudaGetLastError(), "cudaEventCreate");
        }
        e->join.push_back(ev);
    }
    if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
        lpm_ensemble_destroy(e);
        return cuda_status(cudaGetLastError(), "cudaEventCreate");
    }
    // longest processing time first onto the least loaded lane
    std::vector<int> order(n_inst);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int i) { return (double)n_pts[i] * std::log2(2.0 + (double)n_pts[i]); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<double> load(lanes, 0.0);
    e->lane_of.assign(n_inst, 0);
    for (int i : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        e->lane_of[i] = l;
        load[l] += cost(i);
    }
    e->inst.assign(n_inst, nullptr);
    for (int i = 0; i < n_inst; ++i) {
        int rc = lpm_rk4_create(e->lanes[e->lane_of[i]], kernel, solver + (size_t)i * solver_stride, n_src[i],
                                n_pts[i], &e->inst[i]);
        if (rc) {
            lpm_ensemble_destroy(e);
            return rc;
        }
        rk4_set_owner(e->inst[i], e);
    }
    *out = e;
    return LPM_OK;
}

static int ens_check(lpm_ensemble* e, int i) {
    if (i < 0 || i >= (int)e->inst.size()) {
        set_error("ensemble: instance %d out of range", i);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

extern "C" int lpm_ensemble_instance(lpm_ensemble* e, int i, lpm_rk4** rk) {
    if (!e || !rk) {
        set_error("lpm_ensemble_instance: null argument");
        return LPM_ERR_ARG;
    }
    int rc = ens_check(e, i);
    if (rc) return rc;
    *rk = e->inst[i];
    return LPM_OK;
}

extern "C" int lpm_ensemble_set_mlp(lpm_ensemble* e, const float* params) {
    if (!e) {
        set_error("lpm_ensemble_set_mlp: null ensemble");
        return LPM_ERR_ARG;
    }
    int rc = ensemble_invalidate(e);
    if (rc) return rc;
    for (lpm_rk4* r : e->inst) {
        rc = rk4_set_mlp_internal(r, params);
        if (rc) return rc;
    }
    return LPM_OK;
}

extern "C" int lpm_ensemble_set_param(lpm_ensemble* e, const char* name, double value) {
    if (!e || !name) {
        set_error("lpm_ensemble_set_param: null argument");
        return LPM_ERR_ARG;
    }
    int rc = ensemble_invalidate(e);
    if (rc) return rc;
    if (std::string(name) == "fused") {
        if (value != 0.0 && value != 1.0) {
            set_error("lpm_ensemble_set_param: fused is 0 or 1");
            return LPM_ERR_ARG;
        }
        e->fused = value != 0.0;
        return LPM_OK;
    }
    if (std::string(name) == "fused_groups") {
        if (!(value >= 1.0 && value <= 64.0) || value != std::floor(value)) {
            set_error("lpm_ensemble_set_param: fused_groups is 1 .. 64");
            return LPM_ERR_ARG;
        }
        e->groups = (int)value;
        return LPM_OK;
    }
    for (lpm_rk4* r : e->inst) {
        rc = rk4_set_param_internal(r, name, value);
        if (rc) return rc;
    }
    return LPM_OK;
}

extern "C" int lpm_ensemble_get_param(const lpm_ensemble* e, const char* name, double* value) {
    if (!e || !name || !value) {
        set_error("lpm_ensemble_get_param: null argument");
        return LPM_ERR_ARG;
    }
    if (std::string(name) == "fused") {
        *value = e->fused ? 1.0 : 0.0;
        return LPM_OK;
    }
    if (std::string(name) == "fused_groups") {
        *value = (double)e->groups;
        return LPM_OK;
    }
    set_error("lpm_ensemble_get_param: unknown parameter '%s'", name);
    return LPM_ERR_ARG;
}

// Fused groups in effect (at most one per lane); the group of instance i is lane_of[i] % groups.
static int ens_groups(const lpm_ensemble* e) { return std::max(1, std::min(e->groups, (int)e->lanes.size())); }

// Streams, events and tables of every fused group in effect (created outside any capture).
static int ens_groups_ready(lpm_ensemble* e) {
    const int G = ens_groups(e);
    while ((int)e->fz.size() < G) {
        cudaStream_t st = nullptr;
        cudaEvent_t a = nullptr, b = nullptr;
        TreeFused* f = nullptr;
        cudaError_t err = e->fz.empty() ? cudaSuccess : cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
        const int rc = err == cudaSuccess ? tree_fused_create(e->ctx, &f) : cuda_status(err, "fused group");
        if (rc) {
            if (st) cudaStreamDestroy(st);
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
            return rc;
        }
        e->fz.push_back(f);
        e->gstream.push_back(st);
        e->gfork.push_back(a);
        e->gjoin.push_back(b);
    }
    return LPM_OK;
}

// Binds the treecodes of group g's instances (current buffers and parameters) to the group's fused launches,
// which run on stream og (binding synchronises it); the group's streams are idle.
static int ens_bind(lpm_ensemble* e, int g, cudaStream_t og) {
    const int G = ens_groups(e);
    std::vector<TreeSolver*> ts;
    std::vector<double*> us;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (e->lane_of[i] % G == g) {
            ts.push_back(rk4_tree(e->inst[i]));
            us.push_back(rk4_stage_velocity(e->inst[i]));
        }
    if (ts.empty()) return LPM_OK;
    cudaStream_t user = e->ctx->stream;
    e->ctx->stream = og;
    const int rc = tree_fused_bind(e->fz[g], ts.data(), us.data(), (int)ts.size());
    e->ctx->stream = user;
    return rc;
}

// One fused step of group g's instances (four stages: per-instance work on the group's lanes, the far and near
// fields of all its instances on og).  Uncaptured, the instances are bound again after each stage's lists are
// built (they may have grown); captured, the caller has bound them.
static int ens_group_step(lpm_ensemble* e, int g, double dt, cudaStream_t og, bool captured) {
    const int G = ens_groups(e);
    std::vector<size_t> lanes;
    for (size_t l = 0; l < e->lanes.size(); ++l)
        if ((int)(l % G) == g) lanes.push_back(l);
    std::vector<lpm_rk4*> mine;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (e->lane_of[i] % G == g) mine.push_back(e->inst[i]);
    if (mine.empty()) return LPM_OK;
    auto fork = [&]() -> cudaError_t {  // the group's lanes wait for og's work so far
        cudaError_t err = cudaEventRecord(e->gfork[g], og);
        for (size_t l : lanes)
            if (err == cudaSuccess) err = cudaStreamWaitEvent(e->lanes[l]->stream, e->gfork[g], 0);
        return err;
    };
    auto join = [&]() -> cudaError_t {  // og waits for the group's lanes' work so far
        cudaError_t err = cudaSuccess;
        for (size_t l : lanes) {
            if (err == cudaSuccess) err = cudaEventRecord(e->join[l], e->lanes[l]->stream);
            if (err == cudaSuccess) err = cudaStreamWaitEvent(og, e->join[l], 0);
        }
        return err;
    };
    for (int stage = 1; stage <= 4; ++stage) {
        LPM_CUDA_TRY(fork());
        for (lpm_rk4* r : mine) {
            int rc = rk4_stage_begin(r);
            if (rc) return rc;
        }
        LPM_CUDA_TRY(join());
        if (!captured) {
            LPM_CUDA_TRY(cudaStreamSynchronize(og));
            int rc = ens_bind(e, g, og);
            if (rc) return rc;
        }
        cudaStream_t user = e->ctx->stream;
        const bool prof = e->ctx->profiling;
        e->ctx->stream = og;
        e->ctx->profiling = prof && !captured;  // per-kernel timing never inside a capture
        int rc = tree_fused_run(e->fz[g]);
        e->ctx->stream = user;
        e->ctx->profiling = prof;
        if (rc) return rc;
        LPM_CUDA_TRY(fork());
        for (lpm_rk4* r : mine) {
            rc = rk4_stage_update(r, stage, dt);
            if (rc) return rc;
        }
        LPM_CUDA_TRY(join());
    }
    return LPM_OK;
}

// One fused step of every instance: the groups fork from origin onto their own streams and join back.
static int ens_enqueue_fused(lpm_ensemble* e, double dt, cudaStream_t origin, bool captured) {
    const int G = ens_groups(e);
    for (int g = 1; g < G; ++g) {
        LPM_CUDA_TRY(cudaEventRecord(e->gfork[0], origin));
        LPM_CUDA_TRY(cudaStreamWaitEvent(e->gstream[g], e->gfork[0], 0));
    }
    for (int g = 0; g < G; ++g) {
        int rc = ens_group_step(e, g, dt, g == 0 ? origin : e->gstream[g], captured);
        if (rc) return rc;
    }
    for (int g = 1; g < G; ++g) {
        LPM_CUDA_TRY(cudaEventRecord(e->gjoin[g], e->gstream[g]));
        LPM_CUDA_TRY(cudaStreamWaitEvent(origin, e->gjoin[g], 0));
    }
    return LPM_OK;
}

// Whether the fused step applies: some instance uses the treecode.
static bool ens_fusable(const lpm_ensemble* e) {
    if (!e->fused) return false;
    for (lpm_rk4* r : e->inst)
        if (rk4_tree(r)) return true;
    return false;
}

// One step of every instance, each on its lane's current stream.
static int ens_enqueue(lpm_ensemble* e, double dt) {
    if (ens_fusable(e)) {
        int rc = ens_groups_ready(e);
        if (rc) return rc;
        rc = ens_enqueue_fused(e, dt, e->ctx->own_stream, false);
        if (rc) return rc;
        LPM_CUDA_TRY(cudaStreamSynchronize(e->ctx->own_stream));
        return LPM_OK;
    }
    for (size_t i = 0; i < e->inst.size(); ++i) {
        int rc = rk4_step_enqueue(e->inst[i], dt);
        if (rc) return rc;
    }
    return LPM_OK;
}

static int ens_capture(lpm_ensemble* e, double dt) {
    ens_drop_graph(e);
    cudaStream_t origin = e->ctx->own_stream;
    for (lpm_ctx* c : e->lanes) LPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(origin));
    std::vector<cudaStream_t> user(e->lanes.size());
    std::vector<int64_t> before(e->lanes.size());
    for (size_t l = 0; l < e->lanes.size(); ++l) {
        user[l] = e->lanes[l]->stream;
        e->lanes[l]->stream = e->lanes[l]->own_stream;
        before[l] = e->lanes[l]->launches;
    }
    const int64_t before_ctx = e->ctx->launches;  // the fused launches of the capture are counted per replay
    auto restore = [&]() {
        for (size_t l = 0; l < e->lanes.size(); ++l) {
            e->lanes[l]->stream = user[l];
            e->lanes[l]->launches = before[l];
        }
        e->ctx->launches = before_ctx;
    };
    const bool fused = ens_fusable(e);
    if (fused) {  // the fused launches' tables hold the instances' buffers of this capture
        int rc = ens_groups_ready(e);
        for (int g = 0; g < ens_groups(e) && !rc; ++g) rc = ens_bind(e, g, g == 0 ? origin : e->gstream[g]);
        if (rc) {
            restore();
            return rc;
        }
    }
    cudaError_t err = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) {
        restore();
        return cuda_status(err, "cudaStreamBeginCapture");
    }
    int rc = LPM_OK;
    if (fused) {
        rc = ens_enqueue_fused(e, dt, origin, true);
    } else {
        err = cudaEventRecord(e->fork, origin);
        for (size_t l = 0; l < e->lanes.size() && err == cudaSuccess; ++l)
            err = cudaStreamWaitEvent(e->lanes[l]->stream, e->fork, 0);
        if (err == cudaSuccess) rc = ens_enqueue(e, dt);
        for (size_t l = 0; l < e->lanes.size() && err == cudaSuccess; ++l) {
            err = cudaEventRecord(e->join[l], e->lanes[l]->stream);
            if (err == cudaSuccess) err = cudaStreamWaitEvent(origin, e->join[l], 0);
        }
    }
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(origin, &g);
    restore();
    if (rc || err != cudaSuccess || end != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (rc) return rc;
        return cuda_status(err != cudaSuccess ? err : end, "ensemble graph capture");
    }
    e->graph = g;
    size_t nodes = 0;
    LPM_CUDA_TRY(cudaGraphGetNodes(g, nullptr, &nodes));
    e->graph_nodes = (int64_t)nodes;
    LPM_CUDA_TRY(cudaGraphInstantiate(&e->exec, g, 0));
    e->graph_dt = dt;
    e->graph_gen.resize(e->inst.size());
    for (size_t i = 0; i < e->inst.size(); ++i) e->graph_gen[i] = rk4_buffer_generation(e->inst[i]);
    return LPM_OK;
}

extern "C" int lpm_ensemble_step(lpm_ensemble* e, double dt, int nsteps, int use_graph) {
    if (!e || nsteps < 0 || !std::isfinite(dt)) {
        set_error("lpm_ensemble_step: bad argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(e->ctx->device));
    int s = 0;
    // work the caller enqueued on its stream (states) comes first
    LPM_CUDA_TRY(cudaStreamSynchronize(e->ctx->stream));
    if (!use_graph || !e->warmed) {
        const int n_plain = use_graph ? std::min(nsteps, 1) : nsteps;
        for (; s < n_plain; ++s) {
            int rc = ens_enqueue(e, dt);
            if (rc) return rc;
        }
        if (n_plain > 0) e->warmed = true;
    }
    if (s < nsteps) {
        // a graph holds the buffer addresses of its capture: captured again after any reallocation
        if (!e->exec || e->graph_dt != dt || ens_graph_stale(e)) {
            int rc = ens_capture(e, dt);
            if (rc) return rc;
        }
        for (lpm_ctx* c : e->lanes) LPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (; s < nsteps; ++s) {
            LPM_CUDA_TRY(cudaGraphLaunch(e->exec, e->ctx->own_stream));
            e->ctx->launches += e->graph_nodes;
        }
        LPM_CUDA_TRY(cudaStreamSynchronize(e->ctx->own_stream));
    } else {
        for (lpm_ctx* c : e->lanes) LPM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    // replays cannot grow the treecode's buffers: report an overflow instead of returning wrong data
    for (lpm_rk4* r : e->inst) {
        int rc = rk4_tree_check(r);
        if (rc) return rc;
    }
    return LPM_OK;
}

extern "C" int lpm_ensemble_lane_of(const lpm_ensemble* e, int i, int* lane) {
    if (!e || !lane || i < 0 || i >= (int)e->inst.size()) {
        set_error("lpm_ensemble_lane_of: bad argument");
        return LPM_ERR_ARG;
    }
    *lane = e->lane_of[i];
    return LPM_OK;
}

namespace lpm {
int ckpt_write(const char* path, lpm_rk4* const* rks, int n_inst, int64_t step, double t, double dt);
int ckpt_read(const char* path, lpm_rk4* const* rks, int n_inst, int64_t* step, double* t, double* dt);
}  // namespace lpm

extern "C" int lpm_ensemble_checkpoint_write(lpm_ensemble* e, const char* path, int64_t step, double t, double dt) {
    if (!e) {
        set_error("lpm_ensemble_checkpoint_write: null ensemble");
        return LPM_ERR_ARG;
    }
    return ckpt_write(path, e->inst.data(), (int)e->inst.size(), step, t, dt);
}

extern "C" int lpm_ensemble_checkpoint_read(lpm_ensemble* e, const char* path, int64_t* step, double* t, double* dt) {
    if (!e) {
        set_error("lpm_ensemble_checkpoint_read: null ensemble");
        return LPM_ERR_ARG;
    }
    return ckpt_read(path, e->inst.data(), (int)e->inst.size(), step, t, dt);
}
