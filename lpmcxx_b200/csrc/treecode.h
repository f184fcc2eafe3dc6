// Treecode (TreeSum) internals shared between treecode.cu, octree.cu and rk4.cu.
#pragma once

#include "lpm_internal.h"

namespace lpm {

struct TreeSolver;

int tree_solver_create(lpm_ctx* ctx, const lpm_kernel_desc& kernel, const lpm_solver_desc& solver, int64_t n_src,
                       int64_t n_tgt, TreeSolver** out);
void tree_solver_destroy(TreeSolver* t);
// Velocity (3 x n_tgt) of targets X[0:n_tgt] from sources X[0:n_src] (X32: FP32 copy, w pre-scaled).
int tree_velocity(TreeSolver* t, const double4* X, const float4* X32, int64_t n_src, int64_t n_tgt, double* U);

}  // namespace lpm
