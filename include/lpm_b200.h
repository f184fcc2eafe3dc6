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
#define LPM_ERR_TIMEOUT 5    /* a bounded device-side wait gave up */
#define LPM_ERR_CAPACITY 6   /* a fixed capacity was exceeded (tree depth / node pool / scratch) */
#define LPM_ERR_INTERNAL 7   /* an internal consistency check failed */
#define LPM_ERR_NO_DEVICE 8  /* no CUDA device / unsupported device */

/* ---- enums */
#define LPM_MESH_ICOS_TRI 1      /* IcosTriSphereSeed (src/LpmMeshSeed.h:74-82) */
#define LPM_MESH_CUBED_SPHERE 2  /* CubedSphereSeed   (src/LpmMeshSeed.h:84-92) */

#define LPM_KERNEL_BIOT_SAVART_SPHERE 1 /* BiotSavartSphere (src/LpmVectorKernel.h:19-39) */
#define LPM_KERNEL_POISSON_3D 2         /* 1/(4 pi |x-y|): the ScalarKernel subclass the reference lacks */

#define LPM_PREC_F64 0 /* FP64 throughout: parity path against the reference */
#define LPM_PREC_F32 1 /* FP32 pairwise arithmetic, FP64 accumulation of per-tile FP32 partial sums */

/* Kernel descriptor: the data behind the reference's ScalarKernel / VectorKernel plugin objects.
 * BIOT_SAVART_SPHERE: K(x,y) = (x cross y)/(radius^2 - x.y + delta^2), 0 when |den| <= 1e-13,
 *   sum multiplier -1/(4 pi radius), singular iff delta == 0 (src/LpmVectorKernel.h:24-34).
 * POISSON_3D: K(x,y) = 1/(4 pi |x-y|), 0 at x == y. */
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
/* Use an existing cudaStream_t (passed as void*) for all later work; NULL = the context's own stream. */
int lpm_ctx_set_stream(lpm_ctx* ctx, void* cuda_stream);
int lpm_ctx_synchronize(lpm_ctx* ctx);
const char* lpm_last_error(void);
/* Number of kernel launches this library has made on ctx so far (for launch accounting). */
int64_t lpm_ctx_launch_count(const lpm_ctx* ctx);

/* ---- mesh generation (host).  The reference's PolyMesh2d(seed, level) constructor
 * (src/LpmPolyMesh2d.cpp:20-93) in the same vertex / face index order.  Arrays are caller-owned:
 * vert_xyz n_verts x 3, face_xyz n_faces x 3 (centroids), face_area n_faces (0 for divided
 * faces), face_divided n_faces (1 = has children). */
int lpm_mesh_counts(int kind, int level, int64_t* n_verts, int64_t* n_faces, int64_t* n_leaves);
int lpm_mesh_build(int kind, int level, double radius, double* vert_xyz, double* face_xyz, double* face_area,
                   uint8_t* face_divided);

/* ---- direct sums */

/* Device-resident direct sum: out[c*n_tgt + i] = mult * sum_j K(tgt_i, src_j) w_j.
 * src: n_src x 4 (x,y,z,w); tgt: n_tgt x 4 (x,y,z,-); out: {3|1} x n_tgt.
 * Replaces the pair loops of DirectSum::meshSolve (src/LpmDirectSum.cpp:104-166, vector kernel)
 * and DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:240-252, scalar kernel). */
int lpm_direct_sum_dev(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, const double* src, int64_t n_src,
                       const double* tgt, int64_t n_tgt, double* out);

/* Host-facing mesh direct sum with the reference's data: DirectSum::meshSolve
 * (src/LpmDirectSum.cpp:25-167).  Vertex coordinates vx/vy/vz (n_verts), face centroids fx/fy/fz,
 * face areas, divided-face mask and the face source field (n_faces) are host arrays.  Targets are
 * vertices vert_begin..vert_end and undivided faces face_begin..face_end (inclusive); sources are all
 * undivided faces with strength src*area.  Outputs (host, caller-owned) are written only at target
 * indices: vert_out0..2 (n_verts) and face_out0..2 (n_faces); divided faces are left untouched.
 * Only vector kernels (Biot-Savart) are accepted here. */
int lpm_direct_sum_mesh(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n_verts,
                        const double* vx, const double* vy, const double* vz, int64_t n_faces, const double* fx,
                        const double* fy, const double* fz, const double* face_area, const uint8_t* face_divided,
                        const double* face_src, int64_t vert_begin, int64_t vert_end, int64_t face_begin,
                        int64_t face_end, double* vert_out0, double* vert_out1, double* vert_out2, double* face_out0,
                        double* face_out1, double* face_out2);

/* Host-facing meshfree scalar direct sum: DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:175-254)
 * for the 3D Poisson kernel.  x/y/z/src(/weights, may be NULL) are host arrays of n points; targets are
 * points begin..end; out (host, n) is written at target indices. */
int lpm_direct_sum_meshfree(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n, const double* x,
                            const double* y, const double* z, const double* src, const double* weights, int64_t begin,
                            int64_t end, double* out);

#ifdef __cplusplus
}
#endif

#endif /* LPM_B200_H */
