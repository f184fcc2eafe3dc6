// Host-side generator of the recursively refined sphere meshes that feed the hot path:
// vertex positions, face centroids, spherical face areas and the divided-face mask, in the
// exact index order the reference's PolyMesh2d produces (src/LpmPolyMesh2d.cpp:20-93), so
// that per-index results line up with the reference's Field arrays.
//
// Refinement rules restated from the reference:
//   * seed tables: meshSeeds/icosTriSphereSeed.dat, meshSeeds/cubedSphereSeed.dat (vertices,
//     edge records orig/dest/left/right, face edge lists), read as in src/LpmMeshSeed.cpp:56-66;
//   * each level divides every undivided face in index order (src/LpmPolyMesh2d.cpp:62-69);
//   * an undivided edge splits at its normalised midpoint into (orig,mid),(mid,dest), both
//     children inheriting the parent's faces (src/LpmEdges.cpp:99-120);
//   * triangles split into 4 with 3 interior edges (src/LpmTriFaces.cpp:13-142); quads split
//     into 4 around a new centroid vertex with 4 interior edges (src/LpmQuadFaces.cpp:14-146);
//   * a face's vertices are read off its edges by orientation (src/LpmFaces.cpp:147-167),
//     its centroid is the normalised vertex mean (src/LpmXyzVector.cpp:92-100) and its area the
//     sum of L'Huilier triangle areas about the centroid (src/LpmFaces.cpp:71-80,
//     src/LpmXyzVector.cpp:82-90).
// Floating-point expressions keep the reference's operation order (this file is compiled
// with -ffp-contract=off) so the generated coordinates and areas are bit-identical.
#include "lpm_internal.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct V3 {
    double x, y, z;
};
inline V3 cross(const V3& a, const V3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(const V3& a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 normalized_scaled(V3 v, double r) {
    const double n = norm(v);
    v.x /= n; v.y /= n; v.z /= n;
    v.x *= r; v.y *= r; v.z *= r;
    return v;
}
inline double arc(const V3& a, const V3& b) { return std::atan2(norm(cross(a, b)), dot(a, b)); }
double lhuilier(const V3& a, const V3& b, const V3& c, double r) {
    const double s1 = arc(a, b), s2 = arc(b, c), s3 = arc(c, a);
    const double hp = 0.5 * (s1 + s2 + s3);
    const double zz = std::tan(0.5 * hp) * std::tan(0.5 * (hp - s1)) * std::tan(0.5 * (hp - s2)) *
                      std::tan(0.5 * (hp - s3));
    return 4.0 * std::atan2(std::sqrt(zz), 1.0) * r * r;
}

// ---- seed tables (vertex coordinates kept as the seed files' decimal strings so they parse
// to the same doubles)
const char* kIcosVerts[12][3] = {
    {"0.0", "0.0", "1.0"},
    {"0.723606797749978969640917366873", "0.525731112119133606025669084848", "0.447213595499957939281834733746"},
    {"-0.276393202250021030359082633126", "0.850650808352039932181540497063", "0.447213595499957939281834733746"},
    {"-0.894427190999915878563669467492", "0.0", "0.447213595499957939281834733746"},
    {"-0.276393202250021030359082633127", "-0.850650808352039932181540497063", "0.447213595499957939281834733746"},
    {"0.723606797749978969640917366873", "-0.525731112119133606025669084848", "0.447213595499957939281834733746"},
    {"0.894427190999915878563669467492", "0.0", "-0.447213595499957939281834733746"},
    {"0.276393202250021030359082633127", "0.850650808352039932181540497063", "-0.447213595499957939281834733746"},
    {"-0.723606797749978969640917366873", "0.525731112119133606025669084848", "-0.447213595499957939281834733746"},
    {"-0.723606797749978969640917366873", "-0.525731112119133606025669084848", "-0.447213595499957939281834733746"},
    {"0.276393202250021030359082633127", "-0.850650808352039932181540497063", "-0.447213595499957939281834733746"},
    {"0.0", "0.0", "-1.0"}};
const int kIcosEdges[30][4] = {{0, 1, 0, 4},   {1, 2, 0, 6},   {2, 0, 0, 1},   {2, 3, 1, 8},   {0, 3, 2, 1},
                               {3, 4, 2, 10},  {4, 0, 2, 3},   {4, 5, 3, 12},  {5, 0, 3, 4},   {5, 1, 4, 14},
                               {1, 6, 5, 14},  {6, 7, 5, 15},  {7, 1, 5, 6},   {7, 2, 6, 7},   {7, 8, 7, 16},
                               {8, 2, 7, 8},   {8, 3, 8, 9},   {8, 9, 9, 17},  {3, 9, 10, 9},  {9, 4, 10, 11},
                               {9, 10, 11, 18}, {10, 4, 11, 12}, {10, 5, 12, 13}, {10, 6, 13, 19}, {6, 5, 13, 14},
                               {11, 6, 19, 15}, {11, 7, 15, 16}, {8, 11, 17, 16}, {11, 9, 17, 18}, {10, 11, 19, 18}};
const int kIcosFaces[20][3] = {{0, 1, 2},    {2, 3, 4},    {4, 5, 6},    {6, 7, 8},    {8, 9, 0},
                               {10, 11, 12}, {13, 1, 12},  {13, 14, 15}, {16, 3, 15},  {16, 17, 18},
                               {19, 5, 18},  {19, 20, 21}, {22, 7, 21},  {22, 23, 24}, {10, 9, 24},
                               {26, 11, 25}, {27, 14, 26}, {28, 17, 27}, {29, 20, 28}, {25, 23, 29}};
const char* kCubeVerts[8][3] = {{"0.577350269189626", "-0.577350269189626", "0.577350269189626"},
                                {"0.577350269189626", "-0.577350269189626", "-0.577350269189626"},
                                {"0.577350269189626", "0.577350269189626", "-0.577350269189626"},
                                {"0.577350269189626", "0.577350269189626", "0.577350269189626"},
                                {"-0.577350269189626", "0.577350269189626", "-0.577350269189626"},
                                {"-0.577350269189626", "0.577350269189626", "0.577350269189626"},
                                {"-0.577350269189626", "-0.577350269189626", "-0.577350269189626"},
                                {"-0.577350269189626", "-0.577350269189626", "0.577350269189626"}};
const int kCubeEdges[12][4] = {{0, 1, 0, 3}, {1, 2, 0, 5}, {2, 3, 0, 1}, {3, 0, 0, 4}, {2, 4, 1, 5}, {4, 5, 1, 2},
                               {5, 3, 1, 4}, {4, 6, 2, 5}, {6, 7, 2, 3}, {7, 5, 2, 4}, {6, 1, 3, 5}, {0, 7, 3, 4}};
const int kCubeFaces[6][4] = {{0, 1, 2, 3}, {2, 4, 5, 6}, {5, 7, 8, 9}, {8, 10, 0, 11}, {11, 3, 6, 9}, {10, 7, 4, 1}};

class MeshBuilder {
  public:
    MeshBuilder(int nsides, double radius) : ns_(nsides), r_(radius) {}

    void add_vertex(const V3& v) { vx_.push_back(v); }
    int64_t add_edge(int64_t o, int64_t d, int64_t l, int64_t r) {
        eo_.push_back(o); ed_.push_back(d); el_.push_back(l); er_.push_back(r);
        ec0_.push_back(-1); ec1_.push_back(-1);
        return (int64_t)eo_.size() - 1;
    }
    int64_t add_face(const int64_t* edges) {
        fe_.insert(fe_.end(), edges, edges + ns_);
        fdiv_.push_back(0);
        farea_.push_back(0.0);
        return (int64_t)fdiv_.size() - 1;
    }
    int64_t nfaces() const { return (int64_t)fdiv_.size(); }
    bool divided(int64_t f) const { return fdiv_[f] != 0; }

    void face_vertices(int64_t f, int64_t* out) const {
        for (int j = 0; j < ns_; ++j) {
            const int64_t e = fe_[f * ns_ + j];
            out[j] = (el_[e] == f) ? eo_[e] : ed_[e];
        }
    }
    V3 centroid(int64_t f) const {
        int64_t vi[4];
        face_vertices(f, vi);
        V3 c{0.0, 0.0, 0.0};
        for (int j = 0; j < ns_; ++j) { c.x += vx_[vi[j]].x; c.y += vx_[vi[j]].y; c.z += vx_[vi[j]].z; }
        const double s = 1.0 / ns_;
        c.x *= s; c.y *= s; c.z *= s;
        return normalized_scaled(c, 1.0);
    }
    void compute_area(int64_t f) {
        int64_t vi[4];
        face_vertices(f, vi);
        const V3 c = centroid(f);
        double a = 0.0;
        for (int j = 0; j < ns_; ++j) a += lhuilier(c, vx_[vi[j]], vx_[vi[(j + 1) % ns_]], r_);
        farea_[f] = a;
    }
    // returns (child0, child1) of edge e, dividing it first if needed
    void edge_children(int64_t e, int64_t& c0, int64_t& c1) {
        if (ec0_[e] >= 0) { c0 = ec0_[e]; c1 = ec1_[e]; return; }
        const V3& a = vx_[eo_[e]];
        const V3& b = vx_[ed_[e]];
        const int64_t mid = (int64_t)vx_.size();
        add_vertex(normalized_scaled({0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)}, r_));
        const int64_t l = el_[e], r = er_[e], o = eo_[e], d = ed_[e];
        c0 = add_edge(o, mid, l, r);
        c1 = add_edge(mid, d, l, r);
        ec0_[e] = c0; ec1_[e] = c1;
    }

    void divide(int64_t f) {
        const int n = ns_;
        const int64_t nf = nfaces();
        int64_t kid[4] = {nf, nf + 1, nf + 2, nf + 3};
        int64_t pv[4], kv[4][4], ke[4][4];
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) { kv[a][b] = -1; ke[a][b] = -1; }
        face_vertices(f, pv);
        for (int j = 0; j < n; ++j) kv[j][j] = pv[j];
        for (int j = 0; j < n; ++j) {
            const int64_t pe = fe_[f * n + j];
            int64_t c0, c1;
            edge_children(pe, c0, c1);
            const int jn = (j + 1) % n;
            if (el_[pe] == f) {
                ke[j][j] = c0;  el_[c0] = kid[j];
                ke[jn][j] = c1; el_[c1] = kid[jn];
            } else {
                ke[j][j] = c1;  er_[c1] = kid[j];
                ke[jn][j] = c0; er_[c0] = kid[jn];
            }
            const int64_t m = ed_[c0];
            if (n == 3) {
                if (j == 0) { kv[0][1] = m; kv[1][0] = m; kv[3][2] = m; }
                else if (j == 1) { kv[1][2] = m; kv[2][1] = m; kv[3][0] = m; }
                else { kv[2][0] = m; kv[0][2] = m; kv[3][1] = m; }
            } else {
                kv[j][jn] = m; kv[jn][j] = m;
            }
        }
        const int64_t e0 = (int64_t)eo_.size();
        if (n == 3) {
            ke[3][0] = e0; ke[3][1] = e0 + 1; ke[3][2] = e0 + 2;
            ke[0][1] = e0 + 1; ke[1][2] = e0 + 2; ke[2][0] = e0;
            add_edge(kv[2][1], kv[2][0], kid[3], kid[2]);
            add_edge(kv[0][2], kv[0][1], kid[3], kid[0]);
            add_edge(kv[1][0], kv[1][2], kid[3], kid[1]);
        } else {
            const int64_t cv = (int64_t)vx_.size();
            add_vertex(centroid(f));
            for (int j = 0; j < 4; ++j) kv[j][(j + 2) % 4] = cv;
            ke[0][1] = e0;     ke[0][2] = e0 + 3; ke[1][3] = e0;     ke[1][2] = e0 + 2;
            ke[2][3] = e0 + 1; ke[2][0] = e0 + 2; ke[3][1] = e0 + 1; ke[3][0] = e0 + 3;
            add_edge(kv[0][1], kv[0][2], kid[0], kid[1]);
            add_edge(kv[3][1], kv[3][2], kid[3], kid[2]);
            add_edge(kv[1][2], kv[1][3], kid[1], kid[2]);
            add_edge(kv[0][2], kv[0][3], kid[0], kid[3]);
        }
        for (int j = 0; j < 4; ++j) add_face(ke[j]);
        fdiv_[f] = 1;
        farea_[f] = 0.0;
        for (int j = 0; j < 4; ++j) compute_area(kid[j]);
    }

    int ns_;
    double r_;
    std::vector<V3> vx_;
    std::vector<int64_t> eo_, ed_, el_, er_, ec0_, ec1_;
    std::vector<int64_t> fe_;
    std::vector<uint8_t> fdiv_;
    std::vector<double> farea_;
};

int64_t ipow4(int l) {
    int64_t r = 1;
    for (int i = 0; i < l; ++i) r *= 4;
    return r;
}

}  // namespace

namespace lpm {
// The level-0 mesh of a seed (vertices scaled by radius, n x 3; edges as orig, dest, left, right; faces as
// their edge lists, 3 or 4 per face): the start of the device refinement (mesh_refine.cu).
int mesh_seed(int kind, double radius, std::vector<double>& vxyz, std::vector<int32_t>& edges,
              std::vector<int32_t>& faces) {
    if (kind != LPM_MESH_ICOS_TRI && kind != LPM_MESH_CUBED_SPHERE) return LPM_ERR_ARG;
    const bool icos = kind == LPM_MESH_ICOS_TRI;
    const int nsv = icos ? 12 : 8, nse = icos ? 30 : 12, nsf = icos ? 20 : 6, ns = icos ? 3 : 4;
    vxyz.clear();
    edges.clear();
    faces.clear();
    for (int i = 0; i < nsv; ++i) {
        const char* const* s = icos ? kIcosVerts[i] : kCubeVerts[i];
        V3 v{std::strtod(s[0], nullptr), std::strtod(s[1], nullptr), std::strtod(s[2], nullptr)};
        v.x *= radius; v.y *= radius; v.z *= radius;
        vxyz.push_back(v.x);
        vxyz.push_back(v.y);
        vxyz.push_back(v.z);
    }
    for (int i = 0; i < nse; ++i)
        for (int k = 0; k < 4; ++k) edges.push_back(icos ? kIcosEdges[i][k] : kCubeEdges[i][k]);
    for (int i = 0; i < nsf; ++i)
        for (int j = 0; j < ns; ++j) faces.push_back(icos ? kIcosFaces[i][j] : kCubeFaces[i][j]);
    return LPM_OK;
}
}  // namespace lpm

extern "C" int lpm_mesh_counts(int kind, int level, int64_t* n_verts, int64_t* n_faces, int64_t* n_leaves) {
    if ((kind != LPM_MESH_ICOS_TRI && kind != LPM_MESH_CUBED_SPHERE) || level < 0 || level > 12 || !n_verts ||
        !n_faces || !n_leaves)
        return LPM_ERR_ARG;
    const int64_t roots = kind == LPM_MESH_ICOS_TRI ? 20 : 6;
    const int64_t vfac = kind == LPM_MESH_ICOS_TRI ? 10 : 6;
    int64_t nf = 0;
    for (int k = 0; k <= level; ++k) nf += roots * ipow4(k);
    *n_faces = nf;
    *n_leaves = roots * ipow4(level);
    *n_verts = 2 + vfac * ipow4(level);
    return LPM_OK;
}

// Builds the mesh and fills whichever outputs are not NULL.
static int mesh_build_into(int kind, int level, double radius, double* vert_xyz, double* face_xyz,
                           double* face_area, uint8_t* face_divided, int64_t* face_verts) {
    int64_t nv, nf, nl;
    int rc = lpm_mesh_counts(kind, level, &nv, &nf, &nl);
    if (rc != LPM_OK) return rc;
    try {
        const bool icos = kind == LPM_MESH_ICOS_TRI;
        MeshBuilder mb(icos ? 3 : 4, radius);
        mb.vx_.reserve(nv);
        mb.fdiv_.reserve(nf);
        mb.farea_.reserve(nf);
        mb.fe_.reserve(nf * (icos ? 3 : 4));
        const int nsv = icos ? 12 : 8;
        for (int i = 0; i < nsv; ++i) {
            const char* const* s = icos ? kIcosVerts[i] : kCubeVerts[i];
            V3 v{std::strtod(s[0], nullptr), std::strtod(s[1], nullptr), std::strtod(s[2], nullptr)};
            v.x *= radius; v.y *= radius; v.z *= radius;
            mb.add_vertex(v);
        }
        const int nse = icos ? 30 : 12;
        for (int i = 0; i < nse; ++i) {
            const int* e = icos ? kIcosEdges[i] : kCubeEdges[i];
            mb.add_edge(e[0], e[1], e[2], e[3]);
        }
        const int nsf = icos ? 20 : 6;
        for (int i = 0; i < nsf; ++i) {
            int64_t el[4];
            for (int j = 0; j < (icos ? 3 : 4); ++j) el[j] = icos ? kIcosFaces[i][j] : kCubeFaces[i][j];
            mb.add_face(el);
        }
        for (int64_t f = 0; f < mb.nfaces(); ++f) mb.compute_area(f);
        for (int k = 0; k < level; ++k) {
            const int64_t n = mb.nfaces();
            for (int64_t f = 0; f < n; ++f)
                if (!mb.divided(f)) mb.divide(f);
        }
        if ((int64_t)mb.vx_.size() != nv || mb.nfaces() != nf) return LPM_ERR_INTERNAL;
        for (int64_t i = 0; vert_xyz && i < nv; ++i) {
            vert_xyz[3 * i] = mb.vx_[i].x;
            vert_xyz[3 * i + 1] = mb.vx_[i].y;
            vert_xyz[3 * i + 2] = mb.vx_[i].z;
        }
        for (int64_t f = 0; f < nf; ++f) {
            if (face_xyz) {
                const V3 c = mb.centroid(f);
                face_xyz[3 * f] = c.x;
                face_xyz[3 * f + 1] = c.y;
                face_xyz[3 * f + 2] = c.z;
            }
            if (face_area) face_area[f] = mb.farea_[f];
            if (face_divided) face_divided[f] = mb.fdiv_[f];
            if (face_verts) mb.face_vertices(f, face_verts + f * (icos ? 3 : 4));
        }
    } catch (...) {
        return LPM_ERR_OOM;
    }
    return LPM_OK;
}

extern "C" int lpm_mesh_build(int kind, int level, double radius, double* vert_xyz, double* face_xyz,
                              double* face_area, uint8_t* face_divided) {
    if (!vert_xyz || !face_xyz || !face_area || !face_divided || !(radius > 0.0)) return LPM_ERR_ARG;
    return mesh_build_into(kind, level, radius, vert_xyz, face_xyz, face_area, face_divided, nullptr);
}

extern "C" int lpm_mesh_face_vertices(int kind, int level, int64_t* face_verts) {
    if (!face_verts) return LPM_ERR_ARG;
    return mesh_build_into(kind, level, 1.0, nullptr, nullptr, nullptr, nullptr, face_verts);
}
