// Treecode (TreeSum) internals shared between treecode.cu, octree.cu and rk4.cu.
#pragma once

#include "lpm_internal.h"
#include "octree.h"

namespace lpm {

struct TreeSolver;

// The source octree of the solver's last evaluation (valid until the next one) and its point count.
const Octree& tree_source_octree(const TreeSolver* t, int64_t* n_points);
// A read-only lpm_tree over an octree owned elsewhere (lpm_tree_destroy frees the view only).
int tree_view_create(lpm_ctx* ctx, const Octree& t, int64_t n, lpm_tree** out);

// Incremented whenever the solver reallocates a device array (interaction lists, per-node arrays): a CUDA
// graph captured before holds the old addresses and must be captured again.
uint64_t tree_generation(const TreeSolver* t);

int tree_solver_create(lpm_ctx* ctx, const lpm_kernel_desc& kernel, const lpm_solver_desc& solver, int64_t n_src,
                       int64_t n_tgt, TreeSolver** out);
void tree_solver_destroy(TreeSolver* t);
// Velocity (3 x n_tgt, component-major; Biot-Savart) or potential (1 x n_tgt; Poisson 1/(4 pi r)) at
// targets tgt[0:n_tgt] from sources src[0:n_src] (x, y, z, w).  Targets may coincide with sources (their
// self pair contributes nothing).
int tree_velocity(TreeSolver* t, const double4* src, int64_t n_src, const double4* tgt, int64_t n_tgt, double* U);
// Fused evaluations of many solvers (an ensemble's instances at one RK4 stage): each solver runs
// tree_fused_prepare on its own context's stream (everything before the far and near fields), then, once that
// work is joined into the fused context's stream, tree_fused_run enqueues there the far field of every bound
// solver as one persistent launch per Taylor order and the near field as one per near tile shape (Biot-Savart
// solvers; orders in FP64 or above the FP32 kernels' range keep the solver's own launch), bitwise the results
// of tree_velocity.  tree_fused_bind records the solvers' current buffers and parameters (it synchronises the
// fused context's stream): bind again after any reallocation (tree_generation) or parameter change, and never
// while a fused launch may be running.
struct TreeFused;
int tree_fused_create(lpm_ctx* ctx, TreeFused** out);
void tree_fused_destroy(TreeFused* f);
int tree_fused_prepare(TreeSolver* t, const double4* src, const double4* tgt, double* U);
int tree_fused_bind(TreeFused* f, TreeSolver* const* ts, double* const* Us, int n);
int tree_fused_run(TreeFused* f);
// Synchronises and reports capacity overflows of the last evaluation (LPM_ERR_CAPACITY).
int tree_check(TreeSolver* t);
// nodes, leaves, depth, far (batch, cluster) pairs, near runs, batches, overflow flags,
// far target-cluster evaluations, near target-source pairs, far coefficient evaluations (sum over far
// evaluations of the order's coefficient count) (10 values; synchronises)
int tree_stats(TreeSolver* t, int64_t* out10);
// Run-time parameters: "theta" (0 < theta < 1, acceptance criterion), "f64_from" (1..kPMax+1: far
// expansions of this order and above evaluate in FP64), "eps" (learned order's per-pair budget), "batch_level"
// (octree level whose cells target batches may not straddle; 1 .. the level chosen at creation), "order_bias"
// (learned solvers only), "root_maxr" / "root_first" (the root box of the source octree, see TreeSolver).
int tree_set_param(TreeSolver* t, const char* name, double value);
// Current value of a run-time parameter (as tree_set_param, plus "batch_level_max" and "order").
int tree_get_param(const TreeSolver* t, const char* name, double* value);
// Learned order: load the selector (LPM_MLP_PARAMS floats, host) or null for the fixed-order fallback.
int tree_set_mlp(TreeSolver* t, const float* params_host);
// Learned order: labelled training pairs from one evaluation (see lpm_treesum_sample_labels).
int tree_sample_labels(TreeSolver* t, const double4* src, const double4* tgt, int64_t stride, int64_t max_pairs,
                       float* feats, int32_t* labels, float* errs, int64_t* n_out);

}  // namespace lpm
