/*
 * lpm_oracle.c -- FP64 CPU restatement of lpmCxx's DirectSum / TreeSum hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see lpm_oracle.h): the checker, never the product.  Parity is pinned
 * against the reference itself: tests/test_oracle.py compares these functions with outputs of the
 * reference compiled from its sources (tests/golden/, made by tests/golden/make_golden.py).
 */
#include "lpm_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ---- minimal thread pool: split [0, n) into contiguous chunks over ORACLE_THREADS threads
 * (default: all online cores).  Results do not depend on the thread count: every index is
 * computed by exactly one thread with the same sequential inner loop. */
typedef void (*range_fn)(void* arg, int64_t i0, int64_t i1);
typedef struct {
    range_fn fn;
    void* arg;
    int64_t i0, i1;
} range_job;
static void* range_thread(void* p) {
    range_job* j = (range_job*)p;
    j->fn(j->arg, j->i0, j->i1);
    return NULL;
}
int oracle_threads(void) {
    const char* s = getenv("ORACLE_THREADS");
    int n = s ? atoi(s) : (int)sysconf(_SC_NPROCESSORS_ONLN);
    return n < 1 ? 1 : (n > 256 ? 256 : n);
}
static void parallel_range(int64_t n, range_fn fn, void* arg) {
    int nt = oracle_threads();
    if (n < 256 || nt == 1) {
        fn(arg, 0, n);
        return;
    }
    if (nt > n) nt = (int)n;
    pthread_t th[256];
    range_job jobs[256];
    const int64_t chunk = (n + nt - 1) / nt;
    int started = 0;
    for (int t = 0; t < nt; ++t) {
        jobs[t].fn = fn; jobs[t].arg = arg;
        jobs[t].i0 = t * chunk;
        jobs[t].i1 = (t + 1) * chunk < n ? (t + 1) * chunk : n;
        if (jobs[t].i0 >= jobs[t].i1) break;
        if (pthread_create(&th[t], NULL, range_thread, &jobs[t]) != 0) {
            range_thread(&jobs[t]);
            th[t] = 0;
        }
        started = t + 1;
    }
    for (int t = 0; t < started; ++t)
        if (th[t]) pthread_join(th[t], NULL);
}

static const double kPi = 3.1415926535897932384626433832795027975; /* src/LpmTypeDefs.h:18 */
static const double kZeroTol = 1.0e-13;                              /* src/LpmTypeDefs.h:33 */

/* BiotSavartSphere::evaluate (src/LpmVectorKernel.h:24-28) accumulated as in the vector branch of
 * DirectSum::meshSolve (src/LpmDirectSum.cpp:104-118): k = (t x s) / den, k *= strength, sum += k,
 * then sum *= -1/(4 pi R). */
typedef struct {
    const double *src, *tgt;
    int64_t n_src, n_tgt;
    double radius, delta;
    double* out;
} direct_args;

static void bs_direct_range(void* p, int64_t i0, int64_t i1) {
    const direct_args* a = (const direct_args*)p;
    const double* src = a->src;
    const double* tgt = a->tgt;
    const int64_t n_src = a->n_src, n_tgt = a->n_tgt;
    const double radius = a->radius, delta = a->delta;
    double* out = a->out;
    const double mult = -1.0 / (4.0 * kPi * radius);
    for (int64_t i = i0; i < i1; ++i) {
        const double tx = tgt[4 * i], ty = tgt[4 * i + 1], tz = tgt[4 * i + 2];
        double ux = 0.0, uy = 0.0, uz = 0.0;
        for (int64_t j = 0; j < n_src; ++j) {
            const double sx = src[4 * j], sy = src[4 * j + 1], sz = src[4 * j + 2], w = src[4 * j + 3];
            double cx = ty * sz - tz * sy, cy = tz * sx - tx * sz, cz = tx * sy - ty * sx;
            const double den = radius * radius - (tx * sx + ty * sy + tz * sz) + delta * delta;
            if (fabs(den) > kZeroTol) {
                const double inv = 1.0 / den;
                cx *= inv; cy *= inv; cz *= inv;
            } else {
                cx = 0.0; cy = 0.0; cz = 0.0;
            }
            ux += cx * w; uy += cy * w; uz += cz * w;
        }
        out[i] = ux * mult;
        out[n_tgt + i] = uy * mult;
        out[2 * n_tgt + i] = uz * mult;
    }
}

void oracle_bs_direct(const double* src, int64_t n_src, const double* tgt, int64_t n_tgt, double radius,
                      double delta, double* out) {
    direct_args a = {src, tgt, n_src, n_tgt, radius, delta, out};
    parallel_range(n_tgt, bs_direct_range, &a);
}

static void poisson_direct_range(void* p, int64_t i0, int64_t i1) {
    const direct_args* a = (const direct_args*)p;
    const double* src = a->src;
    const double* tgt = a->tgt;
    const int64_t n_src = a->n_src;
    double* out = a->out;
    for (int64_t i = i0; i < i1; ++i) {
        const double tx = tgt[4 * i], ty = tgt[4 * i + 1], tz = tgt[4 * i + 2];
        double phi = 0.0;
        for (int64_t j = 0; j < n_src; ++j) {
            const double dx = tx - src[4 * j], dy = ty - src[4 * j + 1], dz = tz - src[4 * j + 2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            phi += (r > 0.0 ? 1.0 / (4.0 * kPi * r) : 0.0) * src[4 * j + 3];
        }
        out[i] = phi;
    }
}

void oracle_poisson_direct(const double* src, int64_t n_src, const double* tgt, int64_t n_tgt, double* out) {
    direct_args a = {src, tgt, n_src, n_tgt, 0.0, 0.0, out};
    parallel_range(n_tgt, poisson_direct_range, &a);
}

/* The rest of the ScalarKernel family (src/LpmScalarKernel.h:19-78), each value formed as the reference
 * forms it, summed as DirectSum::meshSolve's scalar branch does (src/LpmDirectSum.cpp:36-88):
 * tgtVal += kval * strength over sources j, skipping j == self[i] when self[i] >= 0. */
typedef struct {
    const double* src;
    const double* tgt;
    int64_t n_src, n_tgt;
    int kind;
    double param;
    const int64_t* self;
    double* out;
} scalar_args;

static double scalar_kernel_value(int kind, double param, const double* t, const double* s) {
    switch (kind) {
        case 3: { /* SphereGreensFn(radius) (src/LpmScalarKernel.h:35-38) */
            const double inarg = param * param - (s[0] * t[0] + s[1] * t[1] + s[2] * t[2]);
            return -log(inarg) / (4.0 * kPi * param);
        }
        case 4: { /* PlanarGreensFnFreeBoundaries (src/LpmScalarKernel.h:23-26) */
            const double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
            return log(dx * dx + dy * dy + dz * dz) / (4.0 * kPi);
        }
        case 5: { /* SecondOrderDelta3d(eps) (src/LpmScalarKernel.h:51-57) */
            const double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double expfactor = exp(-pow(r / param, 3));
            const double eps3 = pow(param, 3);
            return 3.0 * expfactor / (4.0 * kPi * eps3);
        }
        case 6: { /* SphereDelta(eps) (src/LpmScalarKernel.h:68-74) */
            const double bkgrnd = 1.0 / (4.0 * kPi);
            const double d = t[0] * s[0] + t[1] * s[1] + t[2] * s[2];
            const double numer = 2.0 * param * param * d - (1.0 - d) * (1.0 - d);
            const double denom = 4.0 * kPi * (1.0 - d + param * param) * (1.0 - d + param * param);
            return numer / denom - bkgrnd;
        }
        default: return 0.0;
    }
}

static void scalar_direct_range(void* p, int64_t i0, int64_t i1) {
    const scalar_args* a = (const scalar_args*)p;
    for (int64_t i = i0; i < i1; ++i) {
        const int64_t skip = a->self ? a->self[i] : -1;
        double v = 0.0;
        for (int64_t j = 0; j < a->n_src; ++j) {
            if (j == skip) continue;
            const double kval = scalar_kernel_value(a->kind, a->param, a->tgt + 4 * i, a->src + 4 * j);
            v += kval * a->src[4 * j + 3];
        }
        a->out[i] = v;
    }
}

void oracle_scalar_direct(int kind, double param, const double* src, int64_t n_src, const double* tgt, int64_t n_tgt,
                          const int64_t* self, double* out) {
    scalar_args a = {src, tgt, n_src, n_tgt, kind, param, self, out};
    parallel_range(n_tgt, scalar_direct_range, &a);
}

/* RK4 of Lagrangian particles on the sphere with the FP64 direct-sum velocity.  The reference's C++
 * tree has no integrator (README.md:75 describes the Fortran one); these are the library's stated
 * semantics: classical RK4, stage positions and the new position re-projected x <- R x/|x|,
 * stage velocities from a full Biot-Savart direct sum with sources = the first n_src particles. */
static void project(double* p, double radius) {
    const double s = radius / sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    p[0] *= s; p[1] *= s; p[2] *= s;
}

void oracle_rk4_direct(double* state, int64_t n_src, int64_t n, double radius, double delta, double dt,
                       int nsteps) {
    double* xs = (double*)malloc(sizeof(double) * 4 * n);
    double* u = (double*)malloc(sizeof(double) * 3 * n);
    double* k = (double*)malloc(sizeof(double) * 3 * n);
    const double a[4] = {0.5 * dt, 0.5 * dt, dt, dt / 6.0};
    for (int s = 0; s < nsteps; ++s) {
        memcpy(xs, state, sizeof(double) * 4 * n);
        for (int stage = 1; stage <= 4; ++stage) {
            oracle_bs_direct(xs, n_src, xs, n, radius, delta, u);
            for (int64_t i = 0; i < n; ++i) {
                double v[3];
                for (int c = 0; c < 3; ++c) {
                    const double uc = u[c * n + i];
                    if (stage == 1) k[c * n + i] = uc;
                    else if (stage < 4) k[c * n + i] += 2.0 * uc;
                    v[c] = stage < 4 ? uc : k[c * n + i] + uc;
                }
                double p[3];
                for (int c = 0; c < 3; ++c) p[c] = state[4 * i + c] + a[stage - 1] * v[c];
                project(p, radius);
                for (int c = 0; c < 3; ++c) xs[4 * i + c] = p[c];
            }
        }
        for (int64_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) state[4 * i + c] = xs[4 * i + c];
    }
    free(xs);
    free(u);
    free(k);
}

/* ---- octree: the reference's recursive build (TreeSum::generateTreeFromMesh,
 * src/LpmTreeSum.cpp:266-290; Tree::generateTreeMaxNodes, src/LpmOctree.cpp:84-143): a node holding more
 * than max_per_leaf indices is bisected at 0.5*(min+max) on all axes (src/LpmBox3d.cpp:140-151), each
 * child keeps, in the parent's order, the indices its half-open box contains (src/LpmBox3d.h:37-39),
 * children are visited in order ix + 2 iy + 4 iz and empty children are dropped.  Nodes are recorded in
 * depth-first pre-order; leaves append their indices to `members`. */
typedef struct {
    const double* pts;
    int max_per_leaf, max_depth;
    int64_t* members;
    int64_t n_members;
    int64_t* leaf_offsets;
    int64_t n_leaves;
    int64_t *level, *parent, *count;
    double* box;
    int64_t n_nodes, node_cap;
    int overflow;
} tree_state;

static void tree_node(tree_state* s, const double* b, const int64_t* idx, int64_t cnt, int level, int64_t parent) {
    const int64_t me = s->n_nodes;
    if (me >= s->node_cap) {
        s->overflow |= 2;
        return;
    }
    s->n_nodes++;
    s->level[me] = level;
    s->parent[me] = parent;
    s->count[me] = cnt;
    memcpy(s->box + 6 * me, b, 6 * sizeof(double));
    if (cnt <= s->max_per_leaf || level >= s->max_depth) {
        if (cnt > s->max_per_leaf) s->overflow |= 1;
        s->leaf_offsets[s->n_leaves++] = s->n_members;
        memcpy(s->members + s->n_members, idx, (size_t)cnt * sizeof(int64_t));
        s->n_members += cnt;
        return;
    }
    const double mx = 0.5 * (b[0] + b[1]), my = 0.5 * (b[2] + b[3]), mz = 0.5 * (b[4] + b[5]);
    int64_t* kid = (int64_t*)malloc((size_t)cnt * sizeof(int64_t));
    for (int d = 0; d < 8; ++d) {
        double cb[6];
        cb[0] = (d & 1) ? mx : b[0]; cb[1] = (d & 1) ? b[1] : mx;
        cb[2] = (d & 2) ? my : b[2]; cb[3] = (d & 2) ? b[3] : my;
        cb[4] = (d & 4) ? mz : b[4]; cb[5] = (d & 4) ? b[5] : mz;
        int64_t k = 0;
        for (int64_t j = 0; j < cnt; ++j) {
            const double* p = s->pts + 4 * idx[j];
            if (cb[0] <= p[0] && p[0] < cb[1] && cb[2] <= p[1] && p[1] < cb[3] && cb[4] <= p[2] && p[2] < cb[5])
                kid[k++] = idx[j];
        }
        if (k > 0) tree_node(s, cb, kid, k, level + 1, me);
    }
    free(kid);
}

int oracle_tree_build(const double* pts, int64_t n, const double* box, int max_per_leaf, int max_depth,
                      int64_t* members, int64_t* leaf_offsets, int64_t* n_leaves, int64_t* n_members,
                      int64_t* node_level, int64_t* node_parent, int64_t* node_count, double* node_box,
                      int64_t node_cap, int64_t* n_nodes) {
    tree_state s = {pts, max_per_leaf, max_depth, members, 0, leaf_offsets, 0, node_level, node_parent, node_count,
                    node_box, 0, node_cap, 0};
    int64_t* all = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) all[i] = i;
    tree_node(&s, box, all, n, 0, -1);
    free(all);
    s.leaf_offsets[s.n_leaves] = s.n_members;
    *n_leaves = s.n_leaves;
    *n_members = s.n_members;
    *n_nodes = s.n_nodes;
    return s.overflow;
}
