// C ABI of the treecode: a reusable device-resident solver object (lpm_treesum) and the
// host-facing TreeSum::meshSolve counterpart.
#include "treecode.h"

#include <algorithm>
#include <cmath>
#include <new>

struct lpm_treesum {
    lpm_ctx* ctx = nullptr;
    lpm::TreeSolver* solver = nullptr;
    int64_t n_src = 0, n_tgt = 0;
};

using namespace lpm;

extern "C" int lpm_treesum_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver,
                                  int64_t n_src, int64_t n_tgt, lpm_treesum** out) {
    if (!ctx || !kernel || !solver || !out || n_src < 0 || n_tgt < 0) {
        set_error("lpm_treesum_create: bad argument");
        return LPM_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    if (kernel->kind != LPM_KERNEL_BIOT_SAVART_SPHERE && kernel->kind != LPM_KERNEL_POISSON_3D) {
        set_error("invalid kernel: the treecode takes the Biot-Savart and 3D Poisson kernels");
        return LPM_ERR_KERNEL;
    }
    if (solver->method != LPM_METHOD_TREE) {
        set_error("lpm_treesum_create: solver method must be LPM_METHOD_TREE");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    lpm_treesum* ts = new (std::nothrow) lpm_treesum();
    if (!ts) return LPM_ERR_OOM;
    ts->ctx = ctx;
    ts->n_src = n_src;
    ts->n_tgt = n_tgt;
    rc = tree_solver_create(ctx, *kernel, *solver, n_src, n_tgt, &ts->solver);
    if (rc) {
        delete ts;
        return rc;
    }
    *out = ts;
    return LPM_OK;
}

extern "C" int lpm_treesum_destroy(lpm_treesum* ts) {
    if (!ts) return LPM_OK;
    cudaSetDevice(ts->ctx->device);
    cudaStreamSynchronize(ts->ctx->stream);
    tree_solver_destroy(ts->solver);
    delete ts;
    return LPM_OK;
}

extern "C" int lpm_treesum_eval_dev(lpm_treesum* ts, const double* src, const double* tgt, double* out) {
    if (!ts || (ts->n_src > 0 && !src) || (ts->n_tgt > 0 && (!tgt || !out))) {
        set_error("lpm_treesum_eval_dev: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ts->ctx->device));
    return tree_velocity(ts->solver, (const double4*)src, ts->n_src, (const double4*)tgt, ts->n_tgt, out);
}

extern "C" int lpm_treesum_stats(lpm_treesum* ts, int64_t* out8) {
    if (!ts || !out8) {
        set_error("lpm_treesum_stats: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ts->ctx->device));
    return tree_stats(ts->solver, out8);
}

extern "C" int lpm_treesum_set_param(lpm_treesum* ts, const char* name, double value) {
    if (!ts) {
        set_error("lpm_treesum_set_param: null solver");
        return LPM_ERR_ARG;
    }
    return tree_set_param(ts->solver, name, value);
}

extern "C" int lpm_treesum_set_mlp(lpm_treesum* ts, const float* params) {
    if (!ts) {
        set_error("lpm_treesum_set_mlp: null solver");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ts->ctx->device));
    return tree_set_mlp(ts->solver, params);
}

extern "C" int lpm_treesum_sample_labels(lpm_treesum* ts, const double* src, const double* tgt, int64_t stride,
                                         int64_t max_pairs, float* feats, int32_t* labels, float* errs,
                                         int64_t* n_out) {
    if (!ts || (ts->n_src > 0 && !src) || (ts->n_tgt > 0 && !tgt)) {
        set_error("lpm_treesum_sample_labels: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ts->ctx->device));
    return tree_sample_labels(ts->solver, (const double4*)src, (const double4*)tgt, stride, max_pairs, feats, labels,
                              errs, n_out);
}

extern "C" int lpm_treesum_source_tree(lpm_treesum* ts, lpm_tree** out) {
    if (!ts || !out) {
        set_error("lpm_treesum_source_tree: null argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ts->ctx->device));
    int64_t n = 0;
    const Octree& t = tree_source_octree(ts->solver, &n);
    return tree_view_create(ts->ctx, t, n, out);
}

extern "C" int lpm_treesum_get_param(const lpm_treesum* ts, const char* name, double* value) {
    if (!ts) {
        set_error("lpm_treesum_get_param: null solver");
        return LPM_ERR_ARG;
    }
    return tree_get_param(ts->solver, name, value);
}

extern "C" int lpm_tree_sum_mesh(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver,
                                 int64_t n_verts, const double* vx, const double* vy, const double* vz, int64_t n_faces,
                                 const double* fx, const double* fy, const double* fz, const double* face_area,
                                 const uint8_t* face_divided, const double* face_src, int64_t vert_begin,
                                 int64_t vert_end, int64_t face_begin, int64_t face_end, double* vert_out0,
                                 double* vert_out1, double* vert_out2, double* face_out0, double* face_out1,
                                 double* face_out2, int64_t* mac_count) {
    if (!ctx || !solver) {
        set_error("lpm_tree_sum_mesh: null argument");
        return LPM_ERR_ARG;
    }
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    if (kernel->kind != LPM_KERNEL_BIOT_SAVART_SPHERE) {
        set_error("invalid kernel: lpm_tree_sum_mesh takes a vector kernel");
        return LPM_ERR_KERNEL;
    }
    if (n_verts < 0 || n_faces < 0 || (n_verts > 0 && (!vx || !vy || !vz)) ||
        (n_faces > 0 && (!fx || !fy || !fz || !face_area || !face_divided || !face_src))) {
        set_error("lpm_tree_sum_mesh: null input arrays");
        return LPM_ERR_ARG;
    }
    const bool do_v = vert_end >= vert_begin, do_f = face_end >= face_begin;
    if ((do_v && (vert_begin < 0 || vert_end >= n_verts || !vert_out0 || !vert_out1 || !vert_out2)) ||
        (do_f && (face_begin < 0 || face_end >= n_faces || !face_out0 || !face_out1 || !face_out2))) {
        set_error("lpm_tree_sum_mesh: target range out of bounds or null outputs");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    int64_t n_src = 0, n_ft = 0;
    for (int64_t i = 0; i < n_faces; ++i)
        if (!face_divided[i]) {
            ++n_src;
            if (do_f && i >= face_begin && i <= face_end) ++n_ft;
        }
    const int64_t n_vt = do_v ? vert_end - vert_begin + 1 : 0;
    const int64_t n_tgt = n_ft + n_vt;
    const size_t out_bytes = sizeof(double) * 3 * (size_t)n_tgt;
    double* host = (double*)pinned(ctx, sizeof(double4) * (size_t)(n_src + n_tgt) + out_bytes);
    if (!host) return LPM_ERR_OOM;
    double4* hsrc = (double4*)host;
    double4* htgt = hsrc + n_src;
    double* hout = (double*)(htgt + n_tgt);
    int64_t s = 0, t = 0;
    for (int64_t i = 0; i < n_faces; ++i) {
        if (face_divided[i]) continue;
        hsrc[s++] = make_double4(fx[i], fy[i], fz[i], face_src[i] * face_area[i]);
        if (do_f && i >= face_begin && i <= face_end) htgt[t++] = make_double4(fx[i], fy[i], fz[i], 0.0);
    }
    for (int64_t i = 0; i < n_vt; ++i) {
        const int64_t v = vert_begin + i;
        htgt[t++] = make_double4(vx[v], vy[v], vz[v], 0.0);
    }
    double4* dsrc = (double4*)scratch(ctx, kSlotSrcPack, sizeof(double4) * (size_t)std::max<int64_t>(n_src, 1));
    double4* dtgt = (double4*)scratch(ctx, kSlotTgtPack, sizeof(double4) * (size_t)std::max<int64_t>(n_tgt, 1));
    double* dout = (double*)scratch(ctx, kSlotOut, std::max<size_t>(out_bytes, 8));
    if (!dsrc || !dtgt || !dout) return LPM_ERR_OOM;
    lpm::TreeSolver* ts = nullptr;
    rc = tree_solver_create(ctx, *kernel, *solver, n_src, n_tgt, &ts);
    if (rc) return rc;
    {
        // root box Box3d(maxR) over every mesh vertex, as TreeSum's mesh constructor (src/LpmTreeSum.cpp:227,
        // Coords::maxR at src/LpmCoords.cpp:136-143: (x x + y y) + z z, largest, then the square root)
        double r2 = 0.0;
        for (int64_t i = 0; i < n_verts; ++i) {
            const double xx = vx[i] * vx[i];
            const double yy = vy[i] * vy[i];
            const double zz = vz[i] * vz[i];
            const double t2 = (xx + yy) + zz;
            if (t2 > r2) r2 = t2;
        }
        if (n_verts > 0) rc = tree_set_param(ts, "root_maxr", std::sqrt(r2));
        if (rc) {
            tree_solver_destroy(ts);
            return rc;
        }
    }
    cudaError_t e = cudaSuccess;
    if (n_src > 0)
        e = cudaMemcpyAsync(dsrc, hsrc, sizeof(double4) * (size_t)n_src, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n_tgt > 0)
        e = cudaMemcpyAsync(dtgt, htgt, sizeof(double4) * (size_t)n_tgt, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) rc = cuda_status(e, "copy inputs");
    if (!rc && n_tgt > 0) rc = tree_velocity(ts, dsrc, n_src, dtgt, n_tgt, dout);
    int64_t st[10] = {0};
    if (!rc && n_tgt > 0 && n_src > 0) rc = tree_stats(ts, st);
    if (!rc && n_tgt > 0) {
        e = cudaMemcpyAsync(hout, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "copy results");
    }
    tree_solver_destroy(ts);
    if (rc) return rc;
    if (mac_count) *mac_count = st[3];
    t = 0;
    for (int64_t i = face_begin; do_f && i <= face_end; ++i) {
        if (face_divided[i]) continue;
        face_out0[i] = hout[t];
        face_out1[i] = hout[n_tgt + t];
        face_out2[i] = hout[2 * n_tgt + t];
        ++t;
    }
    for (int64_t i = 0; i < n_vt; ++i, ++t) {
        vert_out0[vert_begin + i] = hout[t];
        vert_out1[vert_begin + i] = hout[n_tgt + t];
        vert_out2[vert_begin + i] = hout[2 * n_tgt + t];
    }
    return LPM_OK;
}
