// Lpm::DirectSum (declared by the reference's src/LpmDirectSum.h) on the GPU: replaces
// src/LpmDirectSum.cpp.  The constructors bind the same fields as the reference's
// (src/LpmDirectSum.cpp:9-23) so that the class layout and ownership rules stay the reference's own;
// the solves gather the mesh data once per call and run lpm_direct_sum_mesh / lpm_direct_sum_meshfree.
// Arithmetic: FP64 (the reference's), or FP32 with FP64 accumulation when LPM_B200_PRECISION=f32.
#include "LpmDirectSum.h"

#include "LpmB200Dropin.h"

#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace Lpm {

std::unique_ptr<Logger> DirectSum::log(new Logger(OutputMessage::debugPriority, "DirectSum_log"));

DirectSum::DirectSum(std::shared_ptr<MeshedParticles> pmesh, const std::shared_ptr<ScalarKernel> kernel,
                     const std::string tgtFieldName, const std::string srcFieldName)
    : _kernel(kernel),
      useWeights(false),
      _mesh(pmesh->meshPtr()),
      _vertTgt(pmesh->getVertexFieldPtr(tgtFieldName)),
      _faceSrc(pmesh->getFaceFieldPtr(srcFieldName)),
      _faceTgt(pmesh->getFaceFieldPtr(tgtFieldName)) {}

DirectSum::DirectSum(std::shared_ptr<Particles> particles, const std::shared_ptr<ScalarKernel> kernel,
                     const std::string tgtFieldName, const std::string srcFieldName, const std::string srcWeightName)
    : _kernel(kernel),
      _srcWeights(particles->getFieldPtr(srcWeightName)),
      _srcLocs(particles->getCoordPtr(false)),
      _srcVals(particles->getFieldPtr(srcFieldName)),
      _tgtVals(particles->getFieldPtr(tgtFieldName)) {
    useWeights = !_srcWeights.expired();
}

DirectSum::DirectSum(std::shared_ptr<MeshedParticles> pmesh, const std::shared_ptr<VectorKernel> kernel,
                     const std::string tgtFieldName, const std::string srcFieldName)
    : _vecKernel(kernel),
      useWeights(false),
      _mesh(pmesh->meshPtr()),
      _vertTgt(pmesh->getVertexFieldPtr(tgtFieldName)),
      _faceSrc(pmesh->getFaceFieldPtr(srcFieldName)),
      _faceTgt(pmesh->getFaceFieldPtr(tgtFieldName)) {}

namespace {

int precision_from_env() {
    const char* s = std::getenv("LPM_B200_PRECISION");
    return (s && std::strcmp(s, "f32") == 0) ? LPM_PREC_F32 : LPM_PREC_F64;
}

struct MeshArrays {
    std::vector<double> vx, vy, vz, fx, fy, fz, area, src;
    std::vector<uint8_t> divided;
};

MeshArrays gather(const PolyMesh2d& mesh, const Field& src) {
    MeshArrays a;
    std::shared_ptr<Coords> verts = mesh.getPhysCoords();
    std::shared_ptr<Faces> faces = mesh.getFaces();
    const index_type nv = verts->n(), nf = faces->n();
    a.vx.resize(nv);
    a.vy.resize(nv);
    a.vz.resize(nv);
    for (index_type i = 0; i < nv; ++i) {
        const XyzVector v = verts->getVec(i);
        a.vx[i] = v.x;
        a.vy[i] = v.y;
        a.vz[i] = v.z;
    }
    a.fx.resize(nf);
    a.fy.resize(nf);
    a.fz.resize(nf);
    a.area.resize(nf);
    a.src.resize(nf);
    a.divided.resize(nf);
    for (index_type j = 0; j < nf; ++j) {
        a.divided[j] = faces->hasChildren(j) ? 1 : 0;
        if (a.divided[j]) continue;  // the solver reads leaf faces only
        const XyzVector c = faces->centroid(j);
        a.fx[j] = c.x;
        a.fy[j] = c.y;
        a.fz[j] = c.z;
        a.area[j] = faces->area(j);
        a.src[j] = src.getScalar(j);
    }
    return a;
}

}  // namespace

void DirectSum::meshSolve(const MPIReplicatedData& mpiVerts, const MPIReplicatedData& mpiFaces) const {
    const int rank = mpiVerts.getRank();
    std::shared_ptr<PolyMesh2d> mesh = _mesh.lock();
    std::shared_ptr<Field> src = _faceSrc.lock(), vtgt = _vertTgt.lock(), ftgt = _faceTgt.lock();
    if (!mesh || !src || !vtgt || !ftgt) throw std::runtime_error("DirectSum::meshSolve: mesh or field expired");
    lpm_kernel_desc kd;
    if (!_vecKernel.expired()) kd = b200::describe(*_vecKernel.lock());
    else if (!_kernel.expired()) kd = b200::describe(*_kernel.lock());
    else throw std::logic_error("invalid kernel");
    const bool vec = kd.kind == LPM_KERNEL_BIOT_SAVART_SPHERE;
    if (vec && (vtgt->nDim() < 3 || ftgt->nDim() < 3)) throw std::runtime_error("DirectSum: target field must be 3d");
    MeshArrays a = gather(*mesh, *src);
    const index_type nv = (index_type)a.vx.size(), nf = (index_type)a.fx.size();
    b200::check(lpm_direct_sum_mesh(b200::context(), &kd, precision_from_env(), nv, a.vx.data(), a.vy.data(),
                                    a.vz.data(), nf, a.fx.data(), a.fy.data(), a.fz.data(), a.area.data(),
                                    a.divided.data(), a.src.data(), mpiVerts.startIndex(rank),
                                    mpiVerts.endIndex(rank), mpiFaces.startIndex(rank), mpiFaces.endIndex(rank),
                                    vtgt->getPtrToData(0), vec ? vtgt->getPtrToData(1) : nullptr,
                                    vec ? vtgt->getPtrToData(2) : nullptr, ftgt->getPtrToData(0),
                                    vec ? ftgt->getPtrToData(1) : nullptr, vec ? ftgt->getPtrToData(2) : nullptr),
                "lpm_direct_sum_mesh");
}

void DirectSum::meshfreeSolve(const MPIReplicatedData& mpiParticles) const {
    const int rank = mpiParticles.getRank();
    std::shared_ptr<Coords> crd = _srcLocs.lock();
    std::shared_ptr<Field> src = _srcVals.lock(), tgt = _tgtVals.lock();
    std::shared_ptr<ScalarKernel> kernel = _kernel.lock();
    if (!kernel) throw std::logic_error("invalid kernel");
    if (!crd || !src || !tgt) throw std::runtime_error("DirectSum::meshfreeSolve: coords or field expired");
    const lpm_kernel_desc kd = b200::describe(*kernel);
    const index_type n = crd->n();
    std::vector<double> x(n), y(n), z(n), s(n), w;
    for (index_type i = 0; i < n; ++i) {
        const XyzVector v = crd->getVec(i);
        x[i] = v.x;
        y[i] = v.y;
        z[i] = v.z;
        s[i] = src->getScalar(i);
    }
    if (useWeights) {
        std::shared_ptr<Field> wt = _srcWeights.lock();
        w.resize(n);
        for (index_type i = 0; i < n; ++i) w[i] = wt->getScalar(i);
    }
    b200::check(lpm_direct_sum_meshfree(b200::context(), &kd, precision_from_env(), n, x.data(), y.data(), z.data(),
                                        s.data(), useWeights ? w.data() : nullptr, mpiParticles.startIndex(rank),
                                        mpiParticles.endIndex(rank), tgt->getPtrToData(0)),
                "lpm_direct_sum_meshfree");
}

// One GPU computes every target of the calling rank; the slices of other ranks are theirs to compute.
void DirectSum::meshBroadcast(const MPIReplicatedData&, const MPIReplicatedData&) const {}
void DirectSum::meshfreeBroadcast(const MPIReplicatedData&) const {}

}  // namespace Lpm
