// Sphere mesh refinement on the GPU: the PolyMesh2d(seed, level) constructor (src/LpmPolyMesh2d.cpp:20-93)
// level by level, producing the same vertex, edge and face index order as the sequential refinement
// (csrc/sphere_mesh.cpp) and bit-identical vertex coordinates and face centroids.
//
// The sequential refinement divides the undivided faces of a level in index order; dividing a face splits
// each of its edges that is not yet split (src/LpmEdges.cpp:99-120: a midpoint vertex and two child edges),
// then adds the interior edges (3 for a triangle, src/LpmTriFaces.cpp:13-142; a centre vertex and 4 for a
// quadrilateral, src/LpmQuadFaces.cpp:14-146) and the 4 children.  Every edge of a level lies between two
// faces of that level, and the lower-indexed one splits it.  So face i of a level adds d_i midpoints
// (d_i = its edges whose other face has a higher index), 2 d_i + (3 | 4) edges and (0 | 1) centre vertex, and
// exclusive prefix sums of d_i over the level's faces give every new index without running the faces one
// after the other.  Per level: a count kernel, a scan, and a divide kernel in which each face writes its
// midpoints (if it splits the edge), the ends of the child edges it created, its own side of every child
// edge, its interior edges and its children's edge lists.  A last kernel forms every face's centroid (the
// normalised mean of its vertices, read off its edges by orientation, src/LpmFaces.cpp:63-69,147-167) and
// every leaf's area (L'Huilier triangles about the centroid, src/LpmFaces.cpp:71-80,
// src/LpmXyzVector.cpp:82-90).
//
// Coordinates are formed with explicitly rounded operations (no fused multiply-add), in the sequential
// generator's operation order, so midpoints, centre vertices and centroids are bit-identical to it.  Areas
// use the CUDA math library's atan2 and tan: within 1e-13 relative of the host's (11 ulp at icos L4).
#include "lpm_internal.h"

#include <algorithm>
#include <vector>

namespace lpm {
int mesh_seed(int kind, double radius, std::vector<double>& vxyz, std::vector<int32_t>& edges,
              std::vector<int32_t>& faces);
int scan_exclusive_i32(lpm_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, int32_t* total_dev,
                       int sums_slot);

namespace {

struct MeshDev {
    int ns;      // sides per face: 3 or 4
    double r;    // sphere radius
    double* vx;  // vertices, n x 3
    int32_t *eo, *ed, *el, *er;  // edges: origin, destination, left face, right face
    int32_t* fe;                 // faces: ns edge indices each
};

struct P3 {
    double x, y, z;
};

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ P3 load3(const double* v, int i) { return {v[3 * i], v[3 * i + 1], v[3 * i + 2]}; }
__device__ __forceinline__ void store3(double* v, int i, const P3& p) {
    v[3 * i] = p.x;
    v[3 * i + 1] = p.y;
    v[3 * i + 2] = p.z;
}
__device__ __forceinline__ double norm3(const P3& a) {
    return __dsqrt_rn(add(add(mul(a.x, a.x), mul(a.y, a.y)), mul(a.z, a.z)));
}
// v / |v| * r, component by component (division, then multiplication, each rounded)
__device__ __forceinline__ P3 normalized_scaled(P3 v, double r) {
    const double n = norm3(v);
    v.x = __ddiv_rn(v.x, n); v.y = __ddiv_rn(v.y, n); v.z = __ddiv_rn(v.z, n);
    v.x = mul(v.x, r); v.y = mul(v.y, r); v.z = mul(v.z, r);
    return v;
}
__device__ __forceinline__ P3 cross3(const P3& a, const P3& b) {
    return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __forceinline__ double dot3(const P3& a, const P3& b) {
    return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z));
}
__device__ __forceinline__ double arc(const P3& a, const P3& b) { return atan2(norm3(cross3(a, b)), dot3(a, b)); }
__device__ double lhuilier(const P3& a, const P3& b, const P3& c, double r) {
    const double s1 = arc(a, b), s2 = arc(b, c), s3 = arc(c, a);
    const double hp = mul(0.5, add(add(s1, s2), s3));
    const double zz = mul(mul(mul(tan(mul(0.5, hp)), tan(mul(0.5, sub(hp, s1)))), tan(mul(0.5, sub(hp, s2)))),
                          tan(mul(0.5, sub(hp, s3))));
    return mul(mul(mul(4.0, atan2(__dsqrt_rn(zz), 1.0)), r), r);
}

__device__ __forceinline__ int other_face(const MeshDev& m, int e, int f) { return m.el[e] == f ? m.er[e] : m.el[e]; }

// Vertices of face f in the order Faces::vertexIndices reads them off its edges (src/LpmFaces.cpp:147-167).
__device__ __forceinline__ void face_vertices(const MeshDev& m, int f, int (&v)[4]) {
    for (int j = 0; j < m.ns; ++j) {
        const int e = m.fe[(int64_t)f * m.ns + j];
        v[j] = m.el[e] == f ? m.eo[e] : m.ed[e];
    }
}

// Normalised mean of the face's vertices (radius 1, as the sequential generator's centroid).
__device__ P3 centroid(const MeshDev& m, const int (&v)[4]) {
    P3 c{0.0, 0.0, 0.0};
    for (int j = 0; j < m.ns; ++j) {
        const P3 p = load3(m.vx, v[j]);
        c.x = add(c.x, p.x); c.y = add(c.y, p.y); c.z = add(c.z, p.z);
    }
    const double s = __ddiv_rn(1.0, (double)m.ns);
    c.x = mul(c.x, s); c.y = mul(c.y, s); c.z = mul(c.z, s);
    return normalized_scaled(c, 1.0);
}

// Position of edge e among the edges face g splits (g's edges in order, those whose other face is higher).
__device__ __forceinline__ int split_rank(const MeshDev& m, int g, int e) {
    int k = 0;
    for (int j = 0; j < m.ns; ++j) {
        const int ej = m.fe[(int64_t)g * m.ns + j];
        if (ej == e) return k;
        if (g < other_face(m, ej, g)) ++k;
    }
    return -1;
}

// cnt[i] = edges face f0 + i splits (i < nk); cnt[nk] = 0 so that the exclusive scan ends with the total.
__global__ void mesh_count_kernel(MeshDev m, int f0, int nk, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nk; i += gridDim.x * blockDim.x) {
        int d = 0;
        if (i < nk) {
            const int f = f0 + i;
            for (int j = 0; j < m.ns; ++j)
                if (f < other_face(m, m.fe[(int64_t)f * m.ns + j], f)) ++d;
        }
        cnt[i] = d;
    }
}

// Divide faces f0 .. f0 + nk - 1 (the leaves of the level); pre = exclusive prefix sums of the split counts;
// v0 / e0 / nf0 = first new vertex / edge / face index of the level.
__global__ void mesh_divide_kernel(MeshDev m, int f0, int nk, int v0, int e0, int nf0,
                                   const int32_t* __restrict__ pre, uint8_t* __restrict__ divided) {
    const int ns = m.ns, nint = ns == 3 ? 3 : 4;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += gridDim.x * blockDim.x) {
        const int f = f0 + i;
        int kid[4], pv[4], kv[4][4], ke[4][4];
        for (int j = 0; j < 4; ++j) kid[j] = nf0 + 4 * i + j;
        face_vertices(m, f, pv);
        for (int j = 0; j < ns; ++j) kv[j][j] = pv[j];
        for (int j = 0; j < ns; ++j) {
            const int pe = m.fe[(int64_t)f * ns + j];
            const int g = min(f, other_face(m, pe, f));  // the face that splits pe (the lower index)
            const int ig = g - f0, k = split_rank(m, g, pe);
            const int c0 = e0 + 2 * pre[ig] + nint * ig + 2 * k, c1 = c0 + 1;
            const int mid = v0 + pre[ig] + (ns == 4 ? ig : 0) + k;
            if (g == f) {  // this face splits pe: the midpoint and the ends of both children
                const int o = m.eo[pe], d = m.ed[pe];
                const P3 a = load3(m.vx, o), b = load3(m.vx, d);
                store3(m.vx, mid, normalized_scaled({mul(0.5, add(a.x, b.x)), mul(0.5, add(a.y, b.y)),
                                                     mul(0.5, add(a.z, b.z))}, m.r));
                m.eo[c0] = o; m.ed[c0] = mid;
                m.eo[c1] = mid; m.ed[c1] = d;
            }
            const int jn = (j + 1) % ns;
            if (m.el[pe] == f) {  // this face's side of the children
                ke[j][j] = c0; m.el[c0] = kid[j];
                ke[jn][j] = c1; m.el[c1] = kid[jn];
            } else {
                ke[j][j] = c1; m.er[c1] = kid[j];
                ke[jn][j] = c0; m.er[c0] = kid[jn];
            }
            if (ns == 3) {
                if (j == 0) { kv[0][1] = mid; kv[1][0] = mid; kv[3][2] = mid; }
                else if (j == 1) { kv[1][2] = mid; kv[2][1] = mid; kv[3][0] = mid; }
                else { kv[2][0] = mid; kv[0][2] = mid; kv[3][1] = mid; }
            } else {
                kv[j][jn] = mid; kv[jn][j] = mid;
            }
        }
        const int di = pre[i + 1] - pre[i];
        const int ei = e0 + 2 * pre[i] + nint * i + 2 * di;  // this face's interior edges
        auto edge = [&](int e, int o, int d, int l, int r) { m.eo[e] = o; m.ed[e] = d; m.el[e] = l; m.er[e] = r; };
        if (ns == 3) {
            ke[3][0] = ei; ke[3][1] = ei + 1; ke[3][2] = ei + 2;
            ke[0][1] = ei + 1; ke[1][2] = ei + 2; ke[2][0] = ei;
            edge(ei, kv[2][1], kv[2][0], kid[3], kid[2]);
            edge(ei + 1, kv[0][2], kv[0][1], kid[3], kid[0]);
            edge(ei + 2, kv[1][0], kv[1][2], kid[3], kid[1]);
        } else {
            const int cv = v0 + pre[i] + i + di;  // the centre vertex follows this face's midpoints
            store3(m.vx, cv, centroid(m, pv));
            for (int j = 0; j < 4; ++j) kv[j][(j + 2) % 4] = cv;
            ke[0][1] = ei; ke[0][2] = ei + 3; ke[1][3] = ei; ke[1][2] = ei + 2;
            ke[2][3] = ei + 1; ke[2][0] = ei + 2; ke[3][1] = ei + 1; ke[3][0] = ei + 3;
            edge(ei, kv[0][1], kv[0][2], kid[0], kid[1]);
            edge(ei + 1, kv[3][1], kv[3][2], kid[3], kid[2]);
            edge(ei + 2, kv[1][2], kv[1][3], kid[1], kid[2]);
            edge(ei + 3, kv[0][2], kv[0][3], kid[0], kid[3]);
        }
        for (int j = 0; j < 4; ++j)
            for (int q = 0; q < ns; ++q) m.fe[(int64_t)kid[j] * ns + q] = ke[j][q];
        divided[f] = 1;
    }
}

// Every face's centroid and vertex list; the leaves' areas (0 for divided faces).
__global__ void mesh_faces_kernel(MeshDev m, int nf, const uint8_t* __restrict__ divided, double* __restrict__ fxyz,
                                  double* __restrict__ farea, int64_t* __restrict__ fverts) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        int v[4];
        face_vertices(m, f, v);
        const P3 c = centroid(m, v);
        if (fxyz) store3(fxyz, f, c);
        if (fverts)
            for (int j = 0; j < m.ns; ++j) fverts[(int64_t)f * m.ns + j] = v[j];
        if (farea) {
            double a = 0.0;
            if (!divided[f])
                for (int j = 0; j < m.ns; ++j)
                    a = add(a, lhuilier(c, load3(m.vx, v[j]), load3(m.vx, v[(j + 1) % m.ns]), m.r));
            farea[f] = a;
        }
    }
}

__global__ void mesh_particles_kernel(const double* __restrict__ fxyz, const double* __restrict__ farea,
                                      const double* __restrict__ fsrc, const double* __restrict__ vxyz,
                                      int64_t first_leaf, int64_t n_leaves, int64_t n_verts,
                                      double4* __restrict__ state) {
    const int64_t n = n_leaves + n_verts;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (q < n_leaves) {
            const int64_t f = first_leaf + q;
            state[q] = make_double4(fxyz[3 * f], fxyz[3 * f + 1], fxyz[3 * f + 2], fsrc[f] * farea[f]);
        } else {
            const int64_t v = q - n_leaves;
            state[q] = make_double4(vxyz[3 * v], vxyz[3 * v + 1], vxyz[3 * v + 2], 0.0);
        }
    }
}

struct DevFree {
    std::vector<void*> p;
    ~DevFree() {
        for (void* q : p) cudaFree(q);
    }
};

}  // namespace
}  // namespace lpm

using namespace lpm;

extern "C" int lpm_mesh_build_dev(lpm_ctx* ctx, int kind, int level, double radius, double* vert_xyz,
                                  double* face_xyz, double* face_area, uint8_t* face_divided, int64_t* face_verts) {
    int64_t nv = 0, nf = 0, nl = 0;
    if (!ctx || !vert_xyz || !face_divided || !(radius > 0.0) ||
        lpm_mesh_counts(kind, level, &nv, &nf, &nl) != LPM_OK) {
        set_error("lpm_mesh_build_dev: bad argument (kind, 0 <= level <= 12, radius > 0, vert_xyz, face_divided)");
        return LPM_ERR_ARG;
    }
    if (nf >= INT32_MAX / 4) {
        set_error("lpm_mesh_build_dev: level %d exceeds 32-bit face indices", level);
        return LPM_ERR_CAPACITY;
    }
    std::vector<double> sv;
    std::vector<int32_t> se, sf;
    int rc = mesh_seed(kind, radius, sv, se, sf);
    if (rc) return rc;
    const bool icos = kind == LPM_MESH_ICOS_TRI;
    const int ns = icos ? 3 : 4, nint = icos ? 3 : 4;
    const int64_t roots = icos ? 20 : 6, leaf_edges0 = icos ? 30 : 12;
    // every level splits every leaf edge and adds nint interior edges per face
    int64_t ne = (int64_t)se.size() / 4;
    for (int k = 0, p4 = 1; k < level; ++k, p4 *= 4) ne += 2 * leaf_edges0 * p4 + nint * roots * p4;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    DevFree tmp;
    auto alloc = [&](void** p, size_t bytes) -> cudaError_t {
        cudaError_t e = dev_alloc(p, std::max<size_t>(bytes, 4));
        if (e == cudaSuccess) tmp.p.push_back(*p);
        return e;
    };
    MeshDev m{};
    m.ns = ns;
    m.r = radius;
    m.vx = vert_xyz;
    int32_t* cnt = nullptr;
    const int64_t max_level_faces = roots * (int64_t)1 << (2 * std::max(level - 1, 0));
    cudaError_t e = cudaSuccess;
    for (int32_t** p : {&m.eo, &m.ed, &m.el, &m.er})
        if (e == cudaSuccess) e = alloc((void**)p, sizeof(int32_t) * (size_t)ne);
    if (e == cudaSuccess) e = alloc((void**)&m.fe, sizeof(int32_t) * (size_t)nf * ns);
    if (e == cudaSuccess) e = alloc((void**)&cnt, sizeof(int32_t) * (size_t)(max_level_faces + 1));
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (mesh refinement)");
    // seed: vertices, edge records, face edge lists
    const int64_t nse = (int64_t)se.size() / 4;
    std::vector<int32_t> cols(4 * nse);
    for (int64_t i = 0; i < nse; ++i)
        for (int c = 0; c < 4; ++c) cols[c * nse + i] = se[4 * i + c];
    cudaStream_t s = ctx->stream;
    LPM_CUDA_TRY(cudaMemcpyAsync(m.vx, sv.data(), sizeof(double) * sv.size(), cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(m.eo, cols.data(), sizeof(int32_t) * nse, cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(m.ed, cols.data() + nse, sizeof(int32_t) * nse, cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(m.el, cols.data() + 2 * nse, sizeof(int32_t) * nse, cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(m.er, cols.data() + 3 * nse, sizeof(int32_t) * nse, cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(m.fe, sf.data(), sizeof(int32_t) * sf.size(), cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemsetAsync(face_divided, 0, (size_t)nf, s));
    int64_t f0 = 0, nk = roots, v0 = (int64_t)sv.size() / 3, e0 = nse;
    for (int k = 0; k < level; ++k) {
        const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nk + 1, 256), 8 * ctx->num_sms));
        LPM_LAUNCH(ctx, "mesh_count_kernel", mesh_count_kernel, g, 256, 0, m, (int)f0, (int)nk, cnt);
        rc = scan_exclusive_i32(ctx, cnt, cnt, nk + 1, nullptr, kSlotMisc2);
        if (rc) return rc;
        LPM_LAUNCH(ctx, "mesh_divide_kernel", mesh_divide_kernel, g, 256, 0, m, (int)f0, (int)nk, (int)v0, (int)e0,
                   (int)(f0 + nk), cnt, face_divided);
        const int64_t split = leaf_edges0 << (2 * k);  // every leaf edge of the level
        v0 += split + (icos ? 0 : nk);
        e0 += 2 * split + nint * nk;
        f0 += nk;
        nk *= 4;
    }
    if (v0 != nv || e0 != ne || f0 + nk != nf) {
        set_error("lpm_mesh_build_dev: internal count mismatch");
        return LPM_ERR_INTERNAL;
    }
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nf, 256), 8 * ctx->num_sms));
    LPM_LAUNCH(ctx, "mesh_faces_kernel", mesh_faces_kernel, g, 256, 0, m, (int)nf, face_divided, face_xyz, face_area,
               face_verts);
    LPM_CUDA_TRY(cudaStreamSynchronize(s));  // the temporaries are freed on return
    return LPM_OK;
}

extern "C" int lpm_mesh_particles_dev(lpm_ctx* ctx, int kind, int level, const double* vert_xyz,
                                      const double* face_xyz, const double* face_area, const double* face_src,
                                      double* state) {
    int64_t nv = 0, nf = 0, nl = 0;
    if (!ctx || !vert_xyz || !face_xyz || !face_area || !face_src || !state ||
        lpm_mesh_counts(kind, level, &nv, &nf, &nl) != LPM_OK) {
        set_error("lpm_mesh_particles_dev: bad argument");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nl + nv, 256), 8 * ctx->num_sms));
    LPM_LAUNCH(ctx, "mesh_particles_kernel", mesh_particles_kernel, g, 256, 0, face_xyz, face_area, face_src, vert_xyz,
               nf - nl, nl, nv, (double4*)state);
    return LPM_OK;
}
