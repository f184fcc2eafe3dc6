/*
 * lpm_oracle.h -- FP64 CPU restatement of lpmCxx's DirectSum / TreeSum hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product never does.
 * Each function cites the reference code it restates.  The restatement itself is pinned against
 * the reference compiled from its own sources (oracle/_ref/ref_harness) through the golden
 * fixtures in tests/golden/.
 */
#ifndef LPM_ORACLE_H
#define LPM_ORACLE_H
#include <stdint.h>

/* Biot-Savart direct sum, reference formula per pair (src/LpmVectorKernel.h:24-28,
 * src/LpmDirectSum.cpp:104-166): out[c*n_tgt+i] = -1/(4 pi R) sum_j w_j (t_i x s_j)/(R^2 - t.s + d^2),
 * terms with |den| <= 1e-13 dropped.  src: n_src x 4 (x,y,z,w); tgt: n_tgt x 4. */
void oracle_bs_direct(const double* src, int64_t n_src, const double* tgt, int64_t n_tgt, double radius,
                      double delta, double* out);

/* 1/(4 pi |x-y|) direct sum, zero at x == y (DirectSum::meshfreeSolve, src/LpmDirectSum.cpp:240-252). */
void oracle_poisson_direct(const double* src, int64_t n_src, const double* tgt, int64_t n_tgt, double* out);

/* The ScalarKernel family (src/LpmScalarKernel.h:19-78) summed as DirectSum::meshSolve's scalar branch
 * (src/LpmDirectSum.cpp:36-88): out[i] = sum_j w_j K(t_i, s_j) over j != self[i] (self may be NULL; -1 =
 * skip nothing).  kind 3 SphereGreensFn (param = radius), 4 PlanarGreensFnFreeBoundaries, 5
 * SecondOrderDelta3d (param = eps), 6 SphereDelta (param = eps). */
void oracle_scalar_direct(int kind, double param, const double* src, int64_t n_src, const double* tgt, int64_t n_tgt,
                          const int64_t* self, double* out);

/* nsteps classical RK4 steps of the particles state (n x 4: x,y,z,w; the first n_src are sources) with
 * the Biot-Savart direct-sum velocity, stage and final positions re-projected onto the sphere. */
void oracle_rk4_direct(double* state, int64_t n_src, int64_t n, double radius, double delta, double dt, int nsteps);

/* Recursive octree build with the reference's semantics (see lpm_oracle.c).  pts n x 4; box =
 * {xmin,xmax,ymin,ymax,zmin,zmax}.  Outputs: members (n), leaf_offsets (n+1), node arrays (node_cap).
 * Returns a bit mask: 1 = a leaf at max_depth exceeds max_per_leaf, 2 = node_cap exhausted. */
int oracle_tree_build(const double* pts, int64_t n, const double* box, int max_per_leaf, int max_depth,
                      int64_t* members, int64_t* leaf_offsets, int64_t* n_leaves, int64_t* n_members,
                      int64_t* node_level, int64_t* node_parent, int64_t* node_count, double* node_box,
                      int64_t node_cap, int64_t* n_nodes);

/* Number of host threads the oracle uses (ORACLE_THREADS, default: all online cores). */
int oracle_threads(void);

#endif
