// C ABI of the standalone octree: build over device points with an explicit root box, then read
// back the node list (depth-first order) and the leaf membership in the reference's order --
// the coordsContained index lists of its leaves, depth first, each in increasing point index
// (src/LpmTreeSum.cpp:266-290 keeps the parent's order when filtering into children).
#include "octree.h"
#include "treecode.h"

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

struct lpm_tree {
    lpm_ctx* ctx = nullptr;
    lpm::Octree t;
    int64_t n = 0, n_valid = 0, n_nodes = 0, n_leaves = 0;
    int depth = 0, flags = 0;
    bool view = false;  // the octree belongs to a tree solver (lpm_treesum_source_tree / lpm_rk4_source_tree)
};

namespace lpm {
namespace {

__global__ void leaf_of_point_kernel(const int32_t* __restrict__ perm, const int32_t* __restrict__ leaf_scan,
                                     int64_t n, int64_t n_valid, uint32_t* __restrict__ leaf_key,
                                     int32_t* __restrict__ idx) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    idx[p] = (int32_t)p;  // original indices in increasing order (the values of the stable sort)
    const int32_t orig = perm[p];
    leaf_key[orig] = p < n_valid ? (uint32_t)(leaf_scan[p + 1] - 1) : 0xffffffffu;
}

}  // namespace
}  // namespace lpm

using namespace lpm;

static int read_counts(lpm_tree* tr);

extern "C" int lpm_tree_build(lpm_ctx* ctx, const double* pts, int64_t n, const double* box, int max_per_leaf,
                              int max_depth, lpm_tree** out) {
    if (!ctx || !out || !box || n < 0 || (n > 0 && !pts) || max_per_leaf < 1 || n >= INT32_MAX) {
        set_error("lpm_tree_build: bad argument");
        return LPM_ERR_ARG;
    }
    *out = nullptr;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    lpm_tree* tr = new (std::nothrow) lpm_tree();
    if (!tr) return LPM_ERR_OOM;
    tr->ctx = ctx;
    tr->n = n;
    int rc = octree_alloc(tr->t, std::max<int64_t>(n, 1), max_per_leaf, max_depth <= 0 ? kKeyLevels : max_depth);
    if (rc) {
        delete tr;
        return rc;
    }
    RootBox rb;
    for (int a = 0; a < 3; ++a) {
        rb.lo[a] = box[2 * a];
        rb.hi[a] = box[2 * a + 1];
    }
    rc = octree_build(ctx, tr->t, (const double4*)pts, n, rb);
    if (rc) {
        octree_free(tr->t);
        delete tr;
        return rc;
    }
    rc = read_counts(tr);
    if (rc) {
        octree_free(tr->t);
        delete tr;
        return rc;
    }
    *out = tr;
    if (tr->flags) {
        set_error("lpm_tree_build: %s", (tr->flags & 2) ? "node capacity exhausted"
                                                         : "a leaf at the depth limit exceeds max_per_leaf");
        return LPM_ERR_CAPACITY;
    }
    return LPM_OK;
}

namespace lpm {
int tree_view_create(lpm_ctx* ctx, const Octree& t, int64_t n, lpm_tree** out) {
    *out = nullptr;
    lpm_tree* tr = new (std::nothrow) lpm_tree();
    if (!tr) return LPM_ERR_OOM;
    tr->ctx = ctx;
    tr->n = n;
    tr->t = t;
    tr->view = true;
    int rc = read_counts(tr);
    if (rc) {
        delete tr;
        return rc;
    }
    *out = tr;
    return LPM_OK;
}
}  // namespace lpm

static int read_counts(lpm_tree* tr) {
    lpm_ctx* ctx = tr->ctx;
    const int64_t n = tr->n;
    int32_t c[8];
    cudaError_t e = cudaMemcpyAsync(c, tr->t.counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "lpm_tree counts");
    tr->n_valid = c[0];
    tr->n_nodes = c[1];
    tr->flags = c[2];
    tr->n_leaves = c[3];
    tr->depth = c[4];
    // the reference's root holds every index it is given; only splitting filters by containment, so an
    // unsplit root keeps points that lie outside its box
    if (tr->n_nodes == 1) {
        tr->n_valid = n;
        tr->n_leaves = n > 0 ? 1 : tr->n_leaves;
    }
    return LPM_OK;
}

extern "C" int lpm_tree_build_host(lpm_ctx* ctx, const double* xyz, int64_t n, const double* box, int max_per_leaf,
                                   int max_depth, lpm_tree** out) {
    if (!ctx || !out || (n > 0 && !xyz) || n < 0) {
        set_error("lpm_tree_build_host: bad argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t bytes = sizeof(double4) * (size_t)std::max<int64_t>(n, 1);
    double4* h = (double4*)pinned(ctx, bytes);
    double4* d = (double4*)scratch(ctx, kSlotSrcPack, bytes);
    if (!h || !d) return LPM_ERR_OOM;
    for (int64_t i = 0; i < n; ++i) h[i] = make_double4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0);
    if (n > 0) LPM_CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(double4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    return lpm_tree_build(ctx, (const double*)d, n, box, max_per_leaf, max_depth, out);
}

extern "C" int lpm_tree_destroy(lpm_tree* tr) {
    if (!tr) return LPM_OK;
    cudaSetDevice(tr->ctx->device);
    cudaStreamSynchronize(tr->ctx->stream);
    if (!tr->view) octree_free(tr->t);
    delete tr;
    return LPM_OK;
}

extern "C" int lpm_tree_counts(const lpm_tree* tr, int64_t* n_in_tree, int64_t* n_nodes, int64_t* n_leaves,
                               int* depth) {
    if (!tr) {
        set_error("null tree");
        return LPM_ERR_ARG;
    }
    if (n_in_tree) *n_in_tree = tr->n_valid;
    if (n_nodes) *n_nodes = tr->n_nodes;
    if (n_leaves) *n_leaves = tr->n_leaves;
    if (depth) *depth = tr->depth;
    return LPM_OK;
}

extern "C" int lpm_tree_leaf_membership(lpm_tree* tr, int64_t* members, int64_t* leaf_offsets) {
    if (!tr || !members || !leaf_offsets) {
        set_error("lpm_tree_leaf_membership: null argument");
        return LPM_ERR_ARG;
    }
    lpm_ctx* ctx = tr->ctx;
    const int64_t n = tr->n;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    if (n == 0) {
        leaf_offsets[0] = 0;
        return LPM_OK;
    }
    if (tr->n_nodes == 1) {  // unsplit root: every given index, in order
        for (int64_t i = 0; i < n; ++i) members[i] = i;
        leaf_offsets[0] = 0;
        leaf_offsets[1] = n;
        return LPM_OK;
    }
    uint32_t* key = (uint32_t*)scratch(ctx, kSlotTree0, sizeof(uint32_t) * (size_t)n);
    int32_t* idx = (int32_t*)scratch(ctx, kSlotTree1, sizeof(int32_t) * (size_t)n);
    uint32_t* tk = (uint32_t*)scratch(ctx, kSlotTree2, sizeof(uint32_t) * (size_t)n);
    int32_t* tv = (int32_t*)scratch(ctx, kSlotTree3, sizeof(int32_t) * (size_t)n);
    if (!key || !idx || !tk || !tv) return LPM_ERR_OOM;
    LPM_LAUNCH(ctx, "leaf_of_point_kernel", leaf_of_point_kernel, grid_for(n, 256), 256, 0, tr->t.perm,
               tr->t.leaf_flag, n, tr->n_valid, key, idx);
    int rc = radix_sort_u32(ctx, key, idx, tk, tv, n, 32);
    if (rc) return rc;
    std::vector<int32_t> h(n), starts(tr->n_leaves + 1), lnode(tr->n_leaves), nstart(tr->n_nodes);
    LPM_CUDA_TRY(cudaMemcpyAsync(h.data(), idx, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(lnode.data(), tr->t.leaf_node, sizeof(int32_t) * (size_t)tr->n_leaves,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(nstart.data(), tr->t.node_start, sizeof(int32_t) * (size_t)tr->n_nodes,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < tr->n_valid; ++i) members[i] = h[i];
    for (int64_t k = 0; k < tr->n_leaves; ++k) leaf_offsets[k] = nstart[lnode[k]];
    leaf_offsets[tr->n_leaves] = tr->n_valid;
    return LPM_OK;
}

extern "C" int lpm_tree_nodes(lpm_tree* tr, int64_t* level, int64_t* parent, int64_t* count, double* box) {
    if (!tr || !level || !parent || !count || !box) {
        set_error("lpm_tree_nodes: null argument");
        return LPM_ERR_ARG;
    }
    lpm_ctx* ctx = tr->ctx;
    const int64_t m = tr->n_nodes;
    std::vector<int32_t> s(m), e(m), p(m);
    std::vector<int8_t> lv(m);
    std::vector<double> b(6 * m);
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    LPM_CUDA_TRY(cudaMemcpyAsync(s.data(), tr->t.node_start, 4 * m, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(e.data(), tr->t.node_end, 4 * m, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(p.data(), tr->t.node_parent, 4 * m, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(lv.data(), tr->t.node_level, m, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(b.data(), tr->t.node_box, 48 * m, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    // depth-first pre-order = by (range start, level)
    std::vector<int64_t> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c) {
        return s[a] != s[c] ? s[a] < s[c] : lv[a] < lv[c];
    });
    std::vector<int64_t> rank(m);
    for (int64_t k = 0; k < m; ++k) rank[order[k]] = k;
    for (int64_t k = 0; k < m; ++k) {
        const int64_t i = order[k];
        level[k] = lv[i];
        parent[k] = p[i] < 0 ? -1 : rank[p[i]];
        count[k] = p[i] < 0 ? tr->n : e[i] - s[i];  // the root holds every given index
        for (int a = 0; a < 6; ++a) box[6 * k + a] = b[6 * i + a];
    }
    return LPM_OK;
}
