// Treecode (TreeSum) evaluation.
#include "treecode.h"

namespace lpm {

struct TreeSolver {
    lpm_ctx* ctx;
};

int tree_solver_create(lpm_ctx* ctx, const lpm_kernel_desc& kernel, const lpm_solver_desc& solver, int64_t n_src,
                       int64_t n_tgt, TreeSolver** out) {
    (void)ctx; (void)kernel; (void)solver; (void)n_src; (void)n_tgt;
    *out = nullptr;
    set_error("tree solver not available");
    return LPM_ERR_ARG;
}

void tree_solver_destroy(TreeSolver* t) { delete t; }

int tree_velocity(TreeSolver* t, const double4* X, const float4* X32, int64_t n_src, int64_t n_tgt, double* U) {
    (void)t; (void)X; (void)X32; (void)n_src; (void)n_tgt; (void)U;
    set_error("tree solver not available");
    return LPM_ERR_ARG;
}

}  // namespace lpm
