// Lpm::TreeSum (declared by the reference's src/LpmTreeSum.h) on the GPU: replaces src/LpmTreeSum.cpp
// for the mesh path (src/LpmTreeSum.cpp:55-86,182-197,221-238).  No CPU tree is built: each meshSolve
// builds the octree, moments and interaction lists on the GPU (lpm_tree_sum_mesh) with the object's
// series order (|k| < order), leaf capacity and the caller's acceptance parameter; macCounter grows by
// the number of accepted far-field (batch, cluster) pairs.  computeMeshMoments and computeMoments are
// kept as calls but do no work: moments are formed inside each solve from the source field's current
// values.  The mesh constructor initialises the smoothing and shrink flags the reference leaves unset
// (src/LpmTreeSum.cpp:221-226).
//
// Acceptance parameter: meshSolve's mp_tol is the treecode's theta, a (target batch, cluster) pair being
// far when rho < theta (|x_b - c| - r_b) with c and rho the cluster's centre (mean source position) and
// radius, x_b and r_b the centre and radius of a batch of up to 128 targets.  The reference accepts per
// target when box.maxRadius / |box.centroid - x| < mp_tol (src/LpmTreeSum.cpp:22-24).
//
// Arithmetic: the near field is FP32 with FP64 accumulation; the far expansions are FP32, or FP64 when the
// environment variable LPM_B200_PRECISION is "f64" (the same variable selects the DirectSum arithmetic).
#include "LpmTreeSum.h"

#include "LpmB200Dropin.h"

#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace Lpm {

namespace {

int tree_precision_from_env() {
    const char* s = std::getenv("LPM_B200_PRECISION");
    return (s && std::strcmp(s, "f64") == 0) ? LPM_PREC_F64 : LPM_PREC_F32;
}

// Node count of the octree over xyz (n x 3, host) in the root box: lpm_tree_build_host, counted.  A build
// that cannot split a leaf below max_per_leaf within the supported depth (coincident points) throws.
index_type gpu_tree_node_count(const std::vector<double>& xyz, const double box[6], int max_per_leaf) {
    lpm_tree* tr = nullptr;
    const int rc = lpm_tree_build_host(b200::context(), xyz.data(), (int64_t)(xyz.size() / 3), box, max_per_leaf, 0,
                                       &tr);
    int64_t n_in = 0, n_nodes = 0, n_leaves = 0;
    int depth = 0;
    int rc2 = LPM_OK;
    if (tr) {
        rc2 = lpm_tree_counts(tr, &n_in, &n_nodes, &n_leaves, &depth);
        lpm_tree_destroy(tr);
    }
    b200::check(rc, "lpm_tree_build_host");
    b200::check(rc2, "lpm_tree_counts");
    return (index_type)n_nodes;
}

}  // namespace

TreeSum::TreeSum(const std::shared_ptr<Coords> crds, const int max_series_order, const int max_particles_per_box,
                 const scalar_type smoother, const bool do_shrink)
    : Tree(crds),
      _maxSeriesOrder(max_series_order),
      _maxParticlesPerNode(max_particles_per_box),
      _smooth(smoother),
      _shrink(do_shrink),
      sKern(NULL),
      vKern(NULL) {
    // The reference's meshfree constructor splits Tree(crds)'s root (box min - 1e-5 min .. max + 1e-5 max
    // per axis, src/LpmOctree.cpp:16-33) until no node holds more than max_particles_per_box points
    // (src/LpmTreeSum.cpp:208-219, 240-264) and counts the nodes.  The same tree is built on the GPU for
    // nNodes(); depth() stays 0 as there.  With do_shrink the reference shrinks every child box to its
    // points before splitting it further (Tree::shrinkBox), which changes the later splits: not restated,
    // so that case is refused rather than counted differently.
    if (do_shrink) throw std::invalid_argument("TreeSum: do_shrink is not supported by the GPU tree build");
    const index_type n = crds->n();
    std::vector<double> xyz;
    xyz.reserve(3 * (size_t)n);
    for (index_type i = 0; i < n; ++i) {
        const XyzVector v = crds->getVec(i);
        xyz.push_back(v.x);
        xyz.push_back(v.y);
        xyz.push_back(v.z);
    }
    const Box3d& rb = _root->box;
    const double box[6] = {rb.xmin, rb.xmax, rb.ymin, rb.ymax, rb.zmin, rb.zmax};
    _nnodes = gpu_tree_node_count(xyz, box, _maxParticlesPerNode);
}

TreeSum::TreeSum(const int max_series_order, const int max_particles_per_box, std::shared_ptr<MeshedParticles> pmesh,
                 const std::shared_ptr<VectorKernel> kernel, const std::string tgtFieldName,
                 const std::string srcFieldName)
    : Tree(),
      _maxSeriesOrder(max_series_order),
      _maxParticlesPerNode(max_particles_per_box),
      _smooth(0.0),
      _shrink(false),
      sKern(NULL),
      vKern(kernel.get()),
      _mesh(pmesh),
      _vertTgt(pmesh->getVertexFieldPtr(tgtFieldName)),
      _faceSrc(pmesh->getFaceFieldPtr(srcFieldName)),
      _faceTgt(pmesh->getFaceFieldPtr(tgtFieldName)) {
    // The reference's constructor builds the tree over the leaf-face centroids under Box3d(maxR) and counts
    // its nodes (nNodes()); it never computes a depth (depth() stays 0).  The same tree is built here on the
    // GPU for its node count.
    const Box3d rbox(pmesh->maxR());
    std::vector<double> xyz;
    xyz.reserve(3 * (size_t)pmesh->nFaces());
    for (index_type i = 0; i < pmesh->nFaces(); ++i) {
        if (pmesh->faceIsDivided(i)) continue;
        const XyzVector c = pmesh->getFaceCentroid(i);
        xyz.push_back(c.x);
        xyz.push_back(c.y);
        xyz.push_back(c.z);
    }
    const double box[6] = {rbox.xmin, rbox.xmax, rbox.ymin, rbox.ymax, rbox.zmin, rbox.zmax};
    _nnodes = gpu_tree_node_count(xyz, box, _maxParticlesPerNode);
}

void TreeSum::computeMoments(const std::shared_ptr<Field>) {}
void TreeSum::computeMeshMoments() {}

void TreeSum::meshSolve(const MPIReplicatedData& mpiVerts, const MPIReplicatedData& mpiFaces, const scalar_type mp_tol,
                        int& macCounter) {
    const int rank = mpiVerts.getRank();
    std::shared_ptr<MeshedParticles> pm = _mesh.lock();
    std::shared_ptr<Field> src = _faceSrc.lock(), vtgt = _vertTgt.lock(), ftgt = _faceTgt.lock();
    if (!pm || !src || !vtgt || !ftgt) throw std::runtime_error("TreeSum::meshSolve: mesh or field expired");
    if (!vKern) throw std::logic_error("invalid kernel");
    const lpm_kernel_desc kd = b200::describe(*vKern);
    const index_type nv = pm->nVertices(), nf = pm->nFaces();
    std::vector<double> vx(nv), vy(nv), vz(nv), fx(nf), fy(nf), fz(nf), area(nf), s(nf);
    std::vector<uint8_t> divided(nf);
    for (index_type i = 0; i < nv; ++i) {
        const XyzVector v = pm->getVertex(i);
        vx[i] = v.x;
        vy[i] = v.y;
        vz[i] = v.z;
    }
    for (index_type j = 0; j < nf; ++j) {
        divided[j] = pm->faceIsDivided(j) ? 1 : 0;
        if (divided[j]) continue;
        const XyzVector c = pm->getFaceCentroid(j);
        fx[j] = c.x;
        fy[j] = c.y;
        fz[j] = c.z;
        area[j] = pm->getFaceArea(j);
        s[j] = src->getScalar(j);
    }
    lpm_solver_desc sd{};
    sd.method = LPM_METHOD_TREE;
    sd.precision = tree_precision_from_env();
    sd.order = _maxSeriesOrder;
    sd.max_per_leaf = _maxParticlesPerNode;
    sd.theta = mp_tol;
    sd.order_policy = LPM_ORDER_FIXED;
    int64_t mac = 0;
    b200::check(lpm_tree_sum_mesh(b200::context(), &kd, &sd, nv, vx.data(), vy.data(), vz.data(), nf, fx.data(),
                                  fy.data(), fz.data(), area.data(), divided.data(), s.data(),
                                  mpiVerts.startIndex(rank), mpiVerts.endIndex(rank), mpiFaces.startIndex(rank),
                                  mpiFaces.endIndex(rank), vtgt->getPtrToData(0), vtgt->getPtrToData(1),
                                  vtgt->getPtrToData(2), ftgt->getPtrToData(0), ftgt->getPtrToData(1),
                                  ftgt->getPtrToData(2), &mac),
                "lpm_tree_sum_mesh");
    macCounter += (int)mac;
}

// One GPU computes every target of the calling rank; the slices of other ranks are theirs to compute.
void TreeSum::meshBroadcast(const MPIReplicatedData&, const MPIReplicatedData&) const {}

}  // namespace Lpm
