/*
 * lpm_b200.h -- C ABI of the B200 (sm_100a) implementation of lpmCxx's velocity / potential
 * hot path: DirectSum and TreeSum evaluation of the spherical Biot-Savart vector kernel and
 * of the 3D Poisson 1/(4 pi r) scalar kernel, the octree build, Taylor moments, far-field
 * evaluation and the RK4 stage loop around them.
 *
 * Conventions
 *  - Every function returns an int status: LPM_OK (0) or one of the LPM_ERR_* codes.  The
 *    reference reports failures with C++ exceptions (std::logic_error("invalid kernel") at
 *    src/LpmDirectSum.cpp:168-172, std::bad_alloc / std::runtime_error from the data layer);
 *    the C++ drop-in classes turn these codes back into the same exception types.
 *    lpm_last_error() returns a message for the calling thread's last failure.
 *  - "_dev" functions take DEVICE pointers on the context's device and enqueue on the
 *    context's stream (asynchronous; lpm_ctx_synchronize waits).  Functions without the
 *    suffix take HOST pointers and return after the results are on the host.
 *  - Point arrays on the device are packed as n x 4 doubles (x, y, z, w): w is the source
 *    strength (vorticity x area, or charge) and is ignored for targets.
 *  - Outputs on the device are component-major: out[c * n_tgt + i], c = 0..2 (vector kernels)
 *    or c = 0 (scalar kernels) -- the layout of the reference's Field comp0/comp1/comp2 arrays
 *    (src/LpmField.h:83-85).
 *  - Index ranges [begin, end] are inclusive, as MPIReplicatedData::startIndex/endIndex
 *    (src/LpmMPIReplicatedData.cpp:12-23).
 */
#ifndef LPM_B200_H
#define LPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes */
#define LPM_OK 0
#define LPM_ERR_ARG 1        /* bad argument (null pointer, negative size, bad range) */
#define LPM_ERR_KERNEL 2     /* unsupported kernel: the reference's "invalid kernel" logic_error */
#define LPM_ERR_OOM 3        /* device or host allocation failed (std::bad_alloc) */
#define LPM_ERR_CUDA 4       /* a CUDA runtime call failed */
/* 5 is not used: no entry point waits on the device (persistent kernels take work from atomic counters and
 * never spin on a flag) */
#define LPM_ERR_CAPACITY 6   /* a fixed capacity was exceeded (tree depth / node pool / scratch) */
#define LPM_ERR_INTERNAL 7   /* an internal consistency check failed */
#define LPM_ERR_NO_DEVICE 8  /* no CUDA device / unsupported device */

/* ---- enums */
#define LPM_MESH_ICOS_TRI 1      /* IcosTriSphereSeed (src/LpmMeshSeed.h:74-82) */
#define LPM_MESH_CUBED_SPHERE 2  /* CubedSphereSeed   (src/LpmMeshSeed.h:84-92) */

#define LPM_KERNEL_BIOT_SAVART_SPHERE 1 /* BiotSavartSphere (src/LpmVectorKernel.h:19-39) */
#define LPM_KERNEL_POISSON_3D 2         /* 1/(4 pi |x-y|): the ScalarKernel subclass the reference lacks */
#define LPM_KERNEL_SPHERE_GREENS 3      /* SphereGreensFn (src/LpmScalarKernel.h:31-45) */
#define LPM_KERNEL_PLANAR_LOG 4         /* PlanarGreensFnFreeBoundaries (src/LpmScalarKernel.h:19-29) */
#define LPM_KERNEL_DELTA_3D 5           /* SecondOrderDelta3d (src/LpmScalarKernel.h:47-62) */
#define LPM_KERNEL_SPHERE_DELTA 6       /* SphereDelta (src/LpmScalarKernel.h:64-78) */

#define LPM_PREC_F64 0 /* FP64 throughout: parity path against the reference */
#define LPM_PREC_F32 1 /* FP32 pairwise arithmetic, FP64 accumulation of per-tile FP32 partial sums */

/* Kernel descriptor: the data behind the reference's ScalarKernel / VectorKernel plugin objects.
 * BIOT_SAVART_SPHERE: K(x,y) = (x cross y)/(radius^2 - x.y + delta^2), 0 when |den| <= 1e-13,
 *   sum multiplier -1/(4 pi radius), singular iff delta == 0 (src/LpmVectorKernel.h:24-34).
 * POISSON_3D: K(x,y) = 1/(4 pi |x-y|), 0 at x == y.
 * The rest of the reference's ScalarKernel family (direct sums in FP64 only; not in the treecode):
 * SPHERE_GREENS: K = -log(radius^2 - x.y)/(4 pi radius), singular.
 * PLANAR_LOG: K = log(|x-y|^2)/(4 pi), singular.
 * DELTA_3D: K = 3 exp(-(|x-y|/eps)^3)/(4 pi eps^3) with eps in `delta`, not singular.
 * SPHERE_DELTA: K = (2 eps^2 d - (1-d)^2)/(4 pi (1 - d + eps^2)^2) - 1/(4 pi), d = x.y, eps in `delta`,
 *   not singular.
 * A singular kernel's self pair (a face-centroid target and its own source; in the meshfree sum, point i
 * and itself) is skipped by index, as the reference skips j == i (src/LpmDirectSum.cpp:49-68). */
typedef struct lpm_kernel_desc {
    int32_t kind;
    int32_t reserved;
    double radius;
    double delta;
} lpm_kernel_desc;

typedef struct lpm_ctx lpm_ctx;

/* ---- context (replaces the per-rank MPI state; one context per device) */
int lpm_ctx_create(int device, lpm_ctx** out);
int lpm_ctx_destroy(lpm_ctx* ctx);
/* Enqueue all later work on an existing cudaStream_t (passed as void*, used as-is; NULL is the
 * legacy default stream).  A new context starts on its own non-blocking stream; lpm_ctx_own_stream
 * returns that stream and lpm_ctx_set_stream(ctx, lpm_ctx_own_stream(ctx)) switches back to it. */
int lpm_ctx_set_stream(lpm_ctx* ctx, void* cuda_stream);
void* lpm_ctx_own_stream(const lpm_ctx* ctx);
int lpm_ctx_synchronize(lpm_ctx* ctx);
const char* lpm_last_error(void);
/* Number of kernel launches this library has made on ctx so far (for launch accounting). */
int64_t lpm_ctx_launch_count(const lpm_ctx* ctx);
/* Per-kernel CUDA-event timing of uncaptured launches (on = 1).  lpm_ctx_profile_report synchronises,
 * writes {"kernel": {"ms": total, "launches": n}, ...} as JSON into buf and clears the records. */
/* Run-time parameters of a context (no reference counterpart): "direct_targets" = targets per thread of the
 * FP32 direct-sum tile kernels, 2, 4 (default) or 8 (results agree to FP32 rounding; the fastest depends on the
 * sizes: lpmcxx_b200/autotune.py autotune_direct picks it). */
int lpm_ctx_set_param(lpm_ctx* ctx, const char* name, double value);
int lpm_ctx_get_param(const lpm_ctx* ctx, const char* name, double* value);
int lpm_ctx_set_profiling(lpm_ctx* ctx, int on);
int lpm_ctx_profile_report(lpm_ctx* ctx, char* buf, size_t len);

/* Measured FMA-pipe peak (TFLOP/s, FMA = 2 flops) of this device for LPM_PREC_F32 or LPM_PREC_F64: the
 * roofline denominator of the pairwise and far-field kernels.  Synchronous; takes ~100 ms. */
int lpm_fma_peak(lpm_ctx* ctx, int precision, double* tflops);
#define LPM_PEAK_F32X2 2 /* lpm_fma_peak: FP32 issued as packed pairs (fma.rn.f32x2) */

/* ---- mesh generation (host).  The reference's PolyMesh2d(seed, level) constructor
 * (src/LpmPolyMesh2d.cpp:20-93) in the same vertex / face index order.  Arrays are caller-owned:
 * vert_xyz n_verts x 3, face_xyz n_faces x 3 (centroids), face_area n_faces (0 for divided
 * faces), face_divided n_faces (1 = has children). */
int lpm_mesh_counts(int kind, int level, int64_t* n_verts, int64_t* n_faces, int64_t* n_leaves);
int lpm_mesh_build(int kind, int level, double radius, double* vert_xyz, double* face_xyz, double* face_area,
                   uint8_t* face_divided);
/* Vertex indices of every face (n_faces x 3 for LPM_MESH_ICOS_TRI, x 4 for LPM_MESH_CUBED_SPHERE), in
 * the order of Faces::vertexIndices (src/LpmFaces.cpp:63-69): the connectivity lpm_write_vtk writes. */
int lpm_mesh_face_vertices(int kind, int level, int64_t* face_verts);
/* lpm_mesh_build on the GPU (PolyMesh2d(seed, level), src/LpmPolyMesh2d.cpp:20-93, refined level by level
 * by kernels): DEVICE arrays vert_xyz (n_verts x 3), face_xyz (n_faces x 3, may be NULL), face_area (n_faces,
 * may be NULL), face_divided (n_faces), face_verts (n_faces x 3|4, may be NULL).  Same index order as the
 * host generator and the reference; vertex coordinates and centroids bit-identical to them, areas within 1e-13
 * relative (the CUDA math library's atan2 / tan in L'Huilier's formula).  Allocates its
 * edge tables on the device for the call; returns after the arrays are written (level <= 12). */
int lpm_mesh_build_dev(lpm_ctx* ctx, int kind, int level, double radius, double* vert_xyz, double* face_xyz,
                       double* face_area, uint8_t* face_divided, int64_t* face_verts);
/* The RK4 particle state of a device mesh (n_leaves + n_verts) x 4: the leaf faces' centroids carrying
 * face_src x area (the leaves are the last n_leaves faces), then the vertices with strength 0 (device arrays,
 * enqueued on the context's stream). */
int lpm_mesh_particles_dev(lpm_ctx* ctx, int kind, int level, const double* vert_xyz, const double* face_xyz,
                           const double* face_area, const double* face_src, double* state);

/* ---- field output in the reference's file formats (host; fields may be device-resident) */
typedef struct lpm_field_desc {
    const char* name;   /* Field::name() */
    const char* units;  /* Field::units() */
    int32_t ndim;       /* 1, 2 or 3 components */
    int32_t on_device;  /* nonzero: data is device memory (copied to the host after a device synchronize) */
    const double* data; /* component-major: component c of item i at data[c * n + i] */
} lpm_field_desc;

/* Legacy ASCII VTK POLYDATA of a mesh and its fields, byte for byte the file
 * MeshedParticles::writeToVtkFile writes (src/LpmMeshedParticles.cpp:131-153, VtkWriter in
 * src/LpmVtkFileIO.cpp:12-118,195-236): title line, POINTS (n_verts points, xyz_stride doubles apart:
 * 3 for n x 3 arrays, 4 for the RK4 state), POLYGONS of the undivided faces (nsides vertices each from
 * face_verts, n_faces x nsides), POINT_DATA (lag_xyz, if not NULL, as "lagrangian_coords", then the
 * vertex fields, n_verts items), CELL_DATA (the face fields, n_faces items, written at undivided faces).
 * Fields are written in the order given; the reference's MeshedParticles writes them in name order.
 * Doubles print as printf "%.19g" (the reference's setprecision(digits10 of long double + 1)). */
int lpm_write_vtk(const char* path, const char* title, int64_t n_verts, const double* vert_xyz, int32_t xyz_stride,
                  int32_t xyz_on_device, const double* lag_xyz, int64_t n_faces, int32_t nsides,
                  const int64_t* face_verts, const uint8_t* face_divided, int32_t n_vert_fields,
                  const lpm_field_desc* vert_fields, int32_t n_face_fields, const lpm_field_desc* face_fields);

/* Points and fields as CSV: VtkWriter::writePointsAndFieldsToCSV (src/LpmVtkFileIO.cpp:117-193): header
 * "x,y,z" plus name (1 component) or name0,name1[,name2], one row per point, "%g" (a fresh stream's
 * precision).  The reference prints 0 for the third component of the last field when it has 3 (it reads
 * that field through get2dVector, src/LpmVtkFileIO.cpp:186-188); this writes the component's value. */
int lpm_write_csv(const char* path, int64_t n, const double* xyz, int32_t xyz_stride, int32_t xyz_on_device,
                  int32_t n_fields, const lpm_field_desc* fields);

/* ---- direct sums */

/* Device-resident direct sum: out[c*n_tgt + i] = mult * sum_j K(tgt_i, src_j) w_j.
 * src: n_src x 4 (x,y,z,w); tgt: n_tgt x 4 (x,y,z,-); out: {3|1} x n_tgt.
 * n_coincident: targets 0..n_coincident-1 sit exactly on sources 0..n_coincident-1 (face-centroid
 * targets listed first); their self pairs contribute zero, as in the reference.  Any other exactly
 * coincident (target, source) pair is handled by the FP64 path only.
 * Replaces the pair loops of DirectSum::meshSolve (src/LpmDirectSum.cpp:104-166, vector kernel)
 * and DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:240-252, scalar kernel). */
int lpm_direct_sum_dev(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, const double* src, int64_t n_src,
                       const double* tgt, int64_t n_tgt, int64_t n_coincident, double* out);

/* Allocation-free variant of lpm_direct_sum_dev at LPM_PREC_F32 (no counterpart in the reference, which
 * has no GPU path).  For callers that cannot allocate device memory while they run: hosts that reserve
 * the whole device for their own pool allocator, real-time loops that may not block in the allocator.
 * Arguments as lpm_direct_sum_dev, device pointers, enqueued on cuda_stream
 * (NULL = legacy default stream) of the current device; no context.  The FP32 copies live in one
 * file-scope device array of 524,288 points (8 MiB, held by every GPU that loads the library): n_src +
 * n_tgt above that returns LPM_ERR_CAPACITY.  Calls never call cudaMalloc / cudaFree.  The first call on a
 * device looks the array up once (cudaGetSymbolAddress) and should therefore come before any stream
 * capture.  All calls on a device share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int lpm_direct_sum_f32_noalloc(const lpm_kernel_desc* kernel, const double* src, int64_t n_src, const double* tgt,
                               int64_t n_tgt, int64_t n_coincident, double* out, void* cuda_stream);

/* Host-facing mesh direct sum with the reference's data: DirectSum::meshSolve
 * (src/LpmDirectSum.cpp:25-167).  Vertex coordinates vx/vy/vz (n_verts), face centroids fx/fy/fz,
 * face areas, divided-face mask and the face source field (n_faces) are host arrays.  Targets are
 * vertices vert_begin..vert_end and undivided faces face_begin..face_end (inclusive); sources are all
 * undivided faces with strength src*area.  Outputs (host, caller-owned) are written only at target
 * indices: vert_out0..2 (n_verts) and face_out0..2 (n_faces); divided faces are left untouched.
 * Scalar kernels (DirectSum::meshSolve's scalar branch, src/LpmDirectSum.cpp:29-93) write vert_out0 and
 * face_out0 only (the other outputs may be NULL); a singular kernel skips each face target's own source,
 * a non-singular one includes it.  FP32 takes the Biot-Savart and 3D Poisson kernels only. */
int lpm_direct_sum_mesh(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n_verts,
                        const double* vx, const double* vy, const double* vz, int64_t n_faces, const double* fx,
                        const double* fy, const double* fz, const double* face_area, const uint8_t* face_divided,
                        const double* face_src, int64_t vert_begin, int64_t vert_end, int64_t face_begin,
                        int64_t face_end, double* vert_out0, double* vert_out1, double* vert_out2, double* face_out0,
                        double* face_out1, double* face_out2);

/* Host-facing meshfree scalar direct sum: DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:175-254)
 * for the scalar kernels.  x/y/z/src(/weights, may be NULL) are host arrays of n points; targets are
 * points begin..end; out (host, n) is written at target indices.  A singular kernel skips j == i for
 * every target (the reference's singular loops stop at endIndex(i) instead of endIndex(rank),
 * src/LpmDirectSum.cpp:188,222, and run past the slice for i > 0: not restated). */
int lpm_direct_sum_meshfree(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n, const double* x,
                            const double* y, const double* z, const double* src, const double* weights, int64_t begin,
                            int64_t end, double* out);

/* ---- octree (the tree of TreeSum / Tree) */
typedef struct lpm_tree lpm_tree;

/* Build an octree over device points pts (n x 4; x,y,z used) inside the root box
 * box = {xmin, xmax, ymin, ymax, zmin, zmax} (host): nodes holding more than max_per_leaf points are
 * bisected at their FP64 midpoints, points go to the child whose half-open box holds them, empty
 * children are dropped (TreeSum::generateTreeFromMesh, src/LpmTreeSum.cpp:266-290;
 * Tree::generateTreeMaxNodes, src/LpmOctree.cpp:84-143, without box shrinking).  Points outside the root
 * box belong to no leaf.  max_depth <= 0 means the deepest supported level (21).  Returns
 * LPM_ERR_CAPACITY (tree still created) if a leaf at max_depth holds more than max_per_leaf points. */
int lpm_tree_build(lpm_ctx* ctx, const double* pts, int64_t n, const double* box, int max_per_leaf, int max_depth,
                   lpm_tree** out);
/* lpm_tree_build from host coordinates xyz (n x 3): the tree TreeSum's mesh constructor builds
 * (src/LpmTreeSum.cpp:221-238), for callers without device buffers (the drop-in TreeSum's node count). */
int lpm_tree_build_host(lpm_ctx* ctx, const double* xyz, int64_t n, const double* box, int max_per_leaf, int max_depth,
                        lpm_tree** out);
int lpm_tree_destroy(lpm_tree* tree);
int lpm_tree_counts(const lpm_tree* tree, int64_t* n_in_tree, int64_t* n_nodes, int64_t* n_leaves, int* depth);
/* Leaf membership as the reference holds it: members (host, n_in_tree) lists the point indices of every
 * leaf, leaves in depth-first order, each in increasing index order; leaf k is
 * members[leaf_offsets[k] .. leaf_offsets[k+1]) (host, n_leaves + 1). */
int lpm_tree_leaf_membership(lpm_tree* tree, int64_t* members, int64_t* leaf_offsets);
/* All nodes in depth-first pre-order (host arrays, n_nodes each; box n_nodes x 6):
 * level, parent position (-1 for the root), point count, box bounds. */
int lpm_tree_nodes(lpm_tree* tree, int64_t* level, int64_t* parent, int64_t* count, double* box);

/* ---- velocity solver selection (DirectSum or TreeSum, and the arithmetic they use) */
#define LPM_METHOD_DIRECT 0 /* all pairs (DirectSum) */
#define LPM_METHOD_TREE 1   /* octree treecode (TreeSum) */

#define LPM_ORDER_FIXED 0   /* every accepted (target leaf, cluster) pair uses `order` */
#define LPM_ORDER_LEARNED 1 /* an MLP picks the order (or direct) per pair; `order` is the fallback */

typedef struct lpm_solver_desc {
    int32_t method;       /* LPM_METHOD_* */
    int32_t precision;    /* LPM_PREC_*: direct sums' pairwise arithmetic; treecode: LPM_PREC_F64 evaluates
                             the far expansions in FP64 (the near field is FP32 with FP64 sums either way) */
    int32_t order;        /* Taylor order p: multi-indices |k| < p, as SumNode (src/LpmTreeSum.cpp:9-18) */
    int32_t max_per_leaf; /* octree leaf capacity (maxParticlesPerBox) */
    double theta;         /* multipole acceptance parameter */
    int32_t order_policy; /* LPM_ORDER_* */
    int32_t sakajo_depth; /* 0: the source tree is TreeSum's octree (split while a node holds more than
                             max_per_leaf sources); L > 0 (Biot-Savart): the tree of Sakajo (2009) as SakajoTree
                             builds it (src/LpmSakajo2009.cpp:25-63): the box Box3d(radius) bisected 3L times
                             along z, x, y in turn, every non-empty child that meets the sphere kept, leaves at
                             that fixed depth summed directly; max_per_leaf is then ignored */
    double tolerance;     /* LPM_ORDER_LEARNED: per-pair error budget relative to |mult| * sum|w| (0 = 2e-8) */
} lpm_solver_desc;

/* ---- treecode (TreeSum).  Biot-Savart on the unit sphere (radius 1, delta 0): the far field expands
 * 1/|x-y|^2 (equal to 1/(2(1 - x.y)) on the sphere) about each cluster's centre to Taylor order p
 * (|k| < p, the reference's SumNode convention).  3D Poisson 1/(4 pi r) (LPM_KERNEL_POISSON_3D, points in
 * [-1, 1]^3): the far field expands 1/|x-y| to order p with |k| <= p (the reference's TaylorSeries3d
 * convention, src/LpmTaylorSeries3d.cpp:16-50), coincident pairs excluded; the learned order is
 * Biot-Savart only.  Both accept (target batch, cluster) pairs with rho < theta (|x_batch - c| - r_batch);
 * see treecode.cu.  A reusable solver object for fixed sizes: */
typedef struct lpm_treesum lpm_treesum;
int lpm_treesum_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver, int64_t n_src,
                       int64_t n_tgt, lpm_treesum** out);
int lpm_treesum_destroy(lpm_treesum* ts);
/* Device arrays: src n_src x 4 (x,y,z,w), tgt n_tgt x 4, out 3 x n_tgt (component-major; Poisson:
 * 1 x n_tgt).  Replaces TreeSum::computeMeshMoments + meshSolve (src/LpmTreeSum.cpp:55-86,182-197) for
 * device-resident data. */
int lpm_treesum_eval_dev(lpm_treesum* ts, const double* src, const double* tgt, double* out);
/* Statistics of the last evaluation, 10 values: nodes, leaves, depth, far (batch, cluster) pairs, near
 * leaf ranges, target batches, overflow flags, far-field (target, cluster) evaluations, near-field
 * (target, source) pairs, far-field coefficient evaluations (the sum over far evaluations of the order's
 * coefficient count: 8 flops each).  Synchronises. */
int lpm_treesum_stats(lpm_treesum* ts, int64_t* out10);
/* Run-time parameters of a tree solver (no reference counterpart: the reference fixes them at
 * construction).  "theta": acceptance criterion, 0 < theta < 1; "f64_from": far expansions of this
 * order and above evaluate in FP64 (1..13; default 13 = all FP32 for LPM_PREC_F32 solvers, 1 for
 * LPM_PREC_F64); "batch_level": octree level whose cells a target batch may not straddle (1 .. the
 * level chosen at creation; coarser levels give fuller batches); "order_bias" (LPM_ORDER_LEARNED solvers
 * only, LPM_ERR_ARG otherwise; acts while selector weights are loaded): 0..3 orders added to every order the
 * selector picks, capped at 11.  "eps": the learned selector's per-pair error budget.  The near-field tile
 * shape changes the time only (and the FP32 rounding, since it moves the points where FP32 partial sums fold
 * into FP64): "near_targets" 2 or 4 targets per thread, "near_tile" 256, 512 or 1024 sources staged in shared
 * memory per tile, "near_split" 1 or 2 thread groups that each hold a whole target batch and sum their share
 * of every tile.
 * The source octree's root box is the reference's Box3d(R) with its 1e-5 padding (src/LpmBox3d.h:21-33), so
 * that its leaves are the reference TreeSum's (src/LpmTreeSum.cpp:221-238).  Biot-Savart: R = "root_maxr"
 * when positive (default 0), else maxR (Coords::maxR, src/LpmCoords.cpp:136-143) of the targets from index
 * "root_first" on (default 0; an RK4 integrator sets it to its first vertex particle, since the reference
 * takes maxR of the mesh vertices), computed on the device at every evaluation, or of the sources when that
 * range is empty.  Poisson: R = the largest |coordinate| of the sources.  Sources outside the box make the
 * evaluation fail with LPM_ERR_ARG.  Parameters take effect at the next evaluation. */
int lpm_treesum_set_param(lpm_treesum* ts, const char* name, double value);
/* Current value of a run-time parameter: those of lpm_treesum_set_param, plus "batch_level_max" (the finest
 * batch level allowed) and "order" (the fixed order in the solver's convention: Poisson reports p + 1). */
int lpm_treesum_get_param(const lpm_treesum* ts, const char* name, double* value);
/* The source octree of the solver's last evaluation as a read-only lpm_tree (lpm_tree_counts,
 * lpm_tree_leaf_membership and lpm_tree_nodes apply; member indices refer to the evaluation's source array):
 * the tree TreeSum's constructor builds (src/LpmTreeSum.cpp:221-290), for checking it against the
 * reference's.  Valid until the solver's next evaluation or destruction; lpm_tree_destroy frees the view. */
int lpm_treesum_source_tree(lpm_treesum* ts, lpm_tree** out);

/* ---- learned Taylor-order selection (no reference counterpart: the reference's TreeSum uses one
 * fixed order).  An MLP (8 -> 64 -> 64 -> 12, GELU) maps the features of an accepted (target batch,
 * cluster) pair to the smallest order 1..11 whose error stays within tolerance * |mult| * sum|w|, or to
 * "none": the cluster is then opened (or, for a leaf or a small cluster, summed directly).  Parameters are
 * LPM_MLP_PARAMS floats: W1[64][8] b1[64] W2[64][64] b2[64] W3[12][64] b3[12] mean[8] inv_std[8]. */
#define LPM_MLP_PARAMS 5532
#define LPM_MLP_TRAINABLE 5516
/* Load the selector (host array, copied and converted to BF16) into a LPM_ORDER_LEARNED solver, or pass
 * NULL to fall back to the fixed order. */
int lpm_treesum_set_mlp(lpm_treesum* ts, const float* params);
/* Training data from one evaluation of device-resident src / tgt: every stride-th accepted pair (stride
 * <= 0: max_pairs pairs spread evenly over all accepted pairs; at most max_pairs) with its 8 features
 * (feats, max_pairs x 8), label (0..10 = order 1..11, 11 = none within budget) and, if errs is not NULL,
 * the error of every order 1..11 relative to the budget (max_pairs x 11), all judged against the FP64 direct
 * sum of the pair.  Host outputs; *n_out = pairs written.  Synchronous. */
int lpm_treesum_sample_labels(lpm_treesum* ts, const double* src, const double* tgt, int64_t stride,
                              int64_t max_pairs, float* feats, int32_t* labels, float* errs, int64_t* n_out);
/* Train the selector on the GPU (softmax cross-entropy, Adam, mini-batches of `minibatch`, samples shuffled
 * per epoch with `seed`; deterministic).  params: in/out, LPM_MLP_PARAMS floats (the last 16, the feature
 * standardisation, are kept); loss_out: epochs floats (mean loss per epoch) or NULL.  Synchronous. */
int lpm_mlp_train(lpm_ctx* ctx, const float* feats, const int32_t* labels, int64_t n, int epochs, int minibatch,
                  float lr, uint64_t seed, float* params, float* loss_out);
/* Mean cross-entropy loss and its gradient (LPM_MLP_TRAINABLE floats) over n <= 2^20 samples (FP32). */
int lpm_mlp_grad(lpm_ctx* ctx, const float* params, const float* feats, const int32_t* labels, int64_t n,
                 float* grad, float* loss);
/* Classes of n feature vectors with the BF16 inference path the treecode uses. */
int lpm_mlp_predict(lpm_ctx* ctx, const float* params, const float* feats, int64_t n, int32_t* classes);
/* Host-facing TreeSum::meshSolve (src/LpmTreeSum.cpp:55-86) with the same data as lpm_direct_sum_mesh;
 * mac_count (may be NULL) receives the number of accepted far-field (batch, cluster) pairs, the
 * counterpart of the reference's macCounter. */
int lpm_tree_sum_mesh(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver, int64_t n_verts,
                      const double* vx, const double* vy, const double* vz, int64_t n_faces, const double* fx,
                      const double* fy, const double* fz, const double* face_area, const uint8_t* face_divided,
                      const double* face_src, int64_t vert_begin, int64_t vert_end, int64_t face_begin,
                      int64_t face_end, double* vert_out0, double* vert_out1, double* vert_out2, double* face_out0,
                      double* face_out1, double* face_out2, int64_t* mac_count);

/* ---- RK4 integration of the particles (vertices and face-centroid particles as independent
 * Lagrangian particles carrying constant strengths).  The reference's C++ tree has no time
 * integrator; this is the classical four-stage Runge-Kutta step, every stage position and the final
 * position re-projected onto the sphere x <- R x/|x|, stage velocities from a full evaluation of the
 * chosen solver at the stage positions.  FP64 state and update. */
typedef struct lpm_rk4 lpm_rk4;

/* n_pts particles, the first n_src of which are sources (w != 0); the rest are targets only. */
int lpm_rk4_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver, int64_t n_src,
                   int64_t n_pts, lpm_rk4** out);
int lpm_rk4_destroy(lpm_rk4* rk);
/* State as n_pts x 4 (x, y, z, w) doubles: _dev = device pointer (enqueued), host otherwise. */
int lpm_rk4_set_state_dev(lpm_rk4* rk, const double* xyzw);
int lpm_rk4_get_state_dev(lpm_rk4* rk, double* xyzw);
int lpm_rk4_set_state(lpm_rk4* rk, const double* xyzw);
int lpm_rk4_get_state(lpm_rk4* rk, double* xyzw);
/* Advance nsteps steps of size dt.  use_graph != 0 replays one captured CUDA graph per step (the graph is
 * captured on the first call, after one uncaptured warm-up step allocates all scratch). */
int lpm_rk4_step(lpm_rk4* rk, double dt, int nsteps, int use_graph);
/* Velocity (3 x n_pts, component-major, device) at the current state; for diagnostics and tests. */
int lpm_rk4_velocity_dev(lpm_rk4* rk, double* out);
/* Treecode statistics of the last velocity evaluation (the 10 values of lpm_treesum_stats). */
int lpm_rk4_tree_stats(lpm_rk4* rk, int64_t* out10);
/* lpm_treesum_set_param for the integrator's treecode; drops a captured step graph (synchronises).  On an
 * ensemble instance it also drops the ensemble's captured step, whose launches carry the old values. */
int lpm_rk4_set_param(lpm_rk4* rk, const char* name, double value);
int lpm_rk4_get_param(const lpm_rk4* rk, const char* name, double* value);
/* lpm_treesum_source_tree for the integrator's treecode: the octree of its last velocity evaluation. */
int lpm_rk4_source_tree(lpm_rk4* rk, lpm_tree** out);
/* lpm_treesum_set_mlp for the integrator's treecode; drops a captured step graph (synchronises), and the
 * owning ensemble's captured step for an ensemble instance. */
int lpm_rk4_set_mlp(lpm_rk4* rk, const float* params);

/* ---- ensembles (no reference counterpart): n_inst independent RK4 problems of uneven sizes advanced
 * together.  Instances are spread over `lanes` streams (each with its own internal context, assigned
 * longest-first by an n log n size estimate); after one uncaptured step, each step of every instance is
 * one replay of a single CUDA graph that forks onto the lanes and joins back.  In the fused mode (the
 * default), each RK4 stage builds every instance's tree and interaction lists on the lanes and then runs the
 * far field of ALL treecode instances as one persistent launch per Taylor order and their near field as one
 * persistent launch per near tile shape, whose blocks take (instance, batch) items in decreasing order of
 * work over the whole ensemble; results are bitwise those of the lane mode (set_param "fused" 0), where each
 * instance's far and near launches run on its lane.  Instance i is an lpm_rk4 (lpm_ensemble_instance) for
 * setting and reading its state; lpm_ensemble_step is synchronous. */
typedef struct lpm_ensemble lpm_ensemble;
int lpm_ensemble_create(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solver, int n_inst,
                        const int64_t* n_src, const int64_t* n_pts, int lanes, lpm_ensemble** out);
/* lpm_ensemble_create with one solver per instance (solvers: n_inst descriptors), e.g. leaf sizes and
 * acceptance parameters tuned per instance size. */
int lpm_ensemble_create_each(lpm_ctx* ctx, const lpm_kernel_desc* kernel, const lpm_solver_desc* solvers, int n_inst,
                             const int64_t* n_src, const int64_t* n_pts, int lanes, lpm_ensemble** out);
int lpm_ensemble_destroy(lpm_ensemble* ens);
int lpm_ensemble_instance(lpm_ensemble* ens, int i, lpm_rk4** rk);
int lpm_ensemble_lane_of(const lpm_ensemble* ens, int i, int* lane);
int lpm_ensemble_set_mlp(lpm_ensemble* ens, const float* params);
/* lpm_rk4_set_param on every instance; drops the captured step (the next graph step first runs uncaptured).
 * The ensemble's own parameters: "fused" (0 or 1, default 1), the fused far / near launches described above;
 * "fused_groups" (1 .. 64, default 2): the lanes form this many groups (lane l in group l mod G, at most one
 * group per lane) that step independently on their own streams, each with its own fused launches, so that one
 * group's tree builds and traversals overlap another's far and near fields. */
int lpm_ensemble_set_param(lpm_ensemble* ens, const char* name, double value);
/* The ensemble's own parameters ("fused", "fused_groups"). */
int lpm_ensemble_get_param(const lpm_ensemble* ens, const char* name, double* value);
int lpm_ensemble_step(lpm_ensemble* ens, double dt, int nsteps, int use_graph);

/* ---- checkpoint / resume (no reference counterpart: the reference's VTK / CSV output, src/LpmVtkFileIO.h:17-35,
 * is write-only).  A binary dump of an RK4 run's state: the particles (x, y, z, w) as FP64 with the particle and
 * source counts, and the step count, time and time step the caller passes, closed by a 64-bit FNV-1a checksum.
 * _read restores the state into an RK4 (every instance of an ensemble, in instance order) of the same sizes and
 * returns the stored step, t and dt (each pointer may be null); a file of other sizes, not written by these calls,
 * truncated or failing its checksum gives LPM_ERR_ARG and leaves every state as it was.  The steps after a resume
 * are bitwise those of the run that wrote the file.  Synchronous host file I/O. */
int lpm_rk4_checkpoint_write(lpm_rk4* rk, const char* path, int64_t step, double t, double dt);
int lpm_rk4_checkpoint_read(lpm_rk4* rk, const char* path, int64_t* step, double* t, double* dt);
int lpm_ensemble_checkpoint_write(lpm_ensemble* ens, const char* path, int64_t step, double t, double dt);
int lpm_ensemble_checkpoint_read(lpm_ensemble* ens, const char* path, int64_t* step, double* t, double* dt);

/* ---- testing (no reference counterpart): failure injection on the host side.  The device allocation made
 * after `after` further successful ones reports failure (LPM_ERR_OOM from the entry point that made it), once;
 * a negative value turns the injection off.  Process-wide. */
int lpm_debug_fail_allocations(int64_t after);

#ifdef __cplusplus
}
#endif

#endif /* LPM_B200_H */
