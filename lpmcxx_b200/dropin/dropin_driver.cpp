/*
 * Driver of the drop-in classes: it uses only the reference's public API (MeshedParticles, Particles,
 * Field, MPIReplicatedData, DirectSum, TreeSum, BiotSavartSphere) plus PoissonGreensFn3d, with the
 * GPU implementations of DirectSum / TreeSum linked in place of the reference's.  Inputs (vorticity
 * or charges) are read from raw little-endian float64 files so that a test can feed the same values
 * the reference was run with; outputs are written the same way.
 *
 *   direct KIND LEVEL DELTA ZETA.bin OUTDIR          DirectSum(pmesh, BiotSavartSphere(DELTA)).meshSolve
 *   tree   KIND LEVEL ORDER LEAF THETA ZETA.bin OUTDIR TreeSum(ORDER, LEAF, pmesh, kernel).meshSolve(THETA)
 *   poisson N XYZQ.bin OUTDIR                          DirectSum(particles, PoissonGreensFn3d).meshfreeSolve
 *   ptree N XYZ.bin LEAF                               TreeSum(coords, 8, LEAF, 0): the meshfree constructor's
 *                                                      tree (prints its node count and depth)
 *   scalar KIND LEVEL KERNEL PARAM ZETA.bin OUTDIR     DirectSum(pmesh, ScalarKernel).meshSolve with the reference's
 *                                                      SphereGreensFn(PARAM) | PlanarGreensFnFreeBoundaries |
 *                                                      SecondOrderDelta3d(PARAM) | SphereDelta(PARAM)
 *                                                      (KERNEL = spheregreens|planarlog|delta3d|spheredelta)
 * KIND is icos|cube.  ZETA.bin holds one value per face (divided faces included, as the face field);
 * XYZQ.bin holds N x 4 (x, y, z, charge).  OUTDIR receives vert_vel.bin / face_vel.bin (n x 3),
 * vert_phi.bin / face_phi.bin (n) or potential.bin (N), and the driver prints one JSON line.
 */
#include "LpmB200Dropin.h"
#include "LpmDirectSum.h"
#include "LpmEuclideanCoords.h"
#include "LpmMPIReplicatedData.h"
#include "LpmMeshSeed.h"
#include "LpmMeshedParticles.h"
#include "LpmParticles.h"
#include "LpmTreeSum.h"

#include <mpi.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace Lpm;

static std::vector<double> read_f64(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<double> v;
    double buf[4096];
    size_t k;
    while ((k = std::fread(buf, sizeof(double), 4096, f)) > 0) v.insert(v.end(), buf, buf + k);
    std::fclose(f);
    return v;
}

static void write_f64(const std::string& path, const std::vector<double>& v) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
}

static std::unique_ptr<MeshSeed> seed_for(const std::string& kind) {
    if (kind == "icos") return std::unique_ptr<MeshSeed>(new IcosTriSphereSeed());
    if (kind == "cube") return std::unique_ptr<MeshSeed>(new CubedSphereSeed());
    throw std::invalid_argument("KIND must be icos or cube");
}

static std::vector<double> rows3(const std::shared_ptr<Field>& f, index_type n) {
    std::vector<double> out(3 * n);
    for (index_type i = 0; i < n; ++i) {
        const XyzVector v = f->get3dVector(i);
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
    return out;
}

static std::shared_ptr<MeshedParticles> mesh_with_zeta(const std::string& kind, int level, const std::string& zfile) {
    std::unique_ptr<MeshSeed> seed = seed_for(kind);
    auto pm = std::make_shared<MeshedParticles>(*seed, level, false, 1.0, 0);
    pm->createFaceField("vorticity", "1/time", 1);
    pm->createVertexField("velocity", "1/time", 3);
    pm->createFaceField("velocity", "1/time", 3);
    const std::vector<double> z = read_f64(zfile);
    if ((index_type)z.size() != pm->nFaces()) throw std::runtime_error("ZETA.bin must hold one value per face");
    std::shared_ptr<Field> fz = pm->getFaceFieldPtr("vorticity");
    for (index_type i = 0; i < pm->nFaces(); ++i) fz->replace(i, z[i]);
    return pm;
}

int main(int argc, char** argv) {
    MPI_Init(&argc, &argv);
    try {
        const std::string cmd = argc > 1 ? argv[1] : "";
        if (cmd == "direct" && argc == 7) {
            auto pm = mesh_with_zeta(argv[2], std::atoi(argv[3]), argv[5]);
            auto kernel = std::make_shared<BiotSavartSphere>(std::atof(argv[4]));
            MPIReplicatedData mv(pm->nVertices(), 0, 1), mf(pm->nFaces(), 0, 1);
            DirectSum ds(pm, kernel, "velocity", "vorticity");
            ds.meshSolve(mv, mf);
            ds.meshBroadcast(mv, mf);
            const std::string out = argv[6];
            write_f64(out + "/vert_vel.bin", rows3(pm->getVertexFieldPtr("velocity"), pm->nVertices()));
            write_f64(out + "/face_vel.bin", rows3(pm->getFaceFieldPtr("velocity"), pm->nFaces()));
            std::printf("{\"cmd\": \"direct\", \"n_verts\": %ld, \"n_faces\": %ld}\n", (long)pm->nVertices(),
                        (long)pm->nFaces());
        } else if (cmd == "tree" && argc == 9) {
            auto pm = mesh_with_zeta(argv[2], std::atoi(argv[3]), argv[7]);
            auto kernel = std::make_shared<BiotSavartSphere>();
            MPIReplicatedData mv(pm->nVertices(), 0, 1), mf(pm->nFaces(), 0, 1);
            TreeSum ts(std::atoi(argv[4]), std::atoi(argv[5]), pm, kernel, "velocity", "vorticity");
            ts.computeMeshMoments();
            int mac = 0;
            ts.meshSolve(mv, mf, std::atof(argv[6]), mac);
            const std::string out = argv[8];
            write_f64(out + "/vert_vel.bin", rows3(pm->getVertexFieldPtr("velocity"), pm->nVertices()));
            write_f64(out + "/face_vel.bin", rows3(pm->getFaceFieldPtr("velocity"), pm->nFaces()));
            std::printf("{\"cmd\": \"tree\", \"mac_count\": %d, \"n_nodes\": %ld, \"depth\": %d}\n", mac,
                        (long)ts.nNodes(), ts.depth());
        } else if (cmd == "scalar" && argc == 8) {
            auto pm = mesh_with_zeta(argv[2], std::atoi(argv[3]), argv[6]);
            pm->createVertexField("potential", "n/a", 1);
            pm->createFaceField("potential", "n/a", 1);
            const std::string kname = argv[4];
            const double param = std::atof(argv[5]);
            std::shared_ptr<ScalarKernel> kernel;
            if (kname == "spheregreens") kernel = std::make_shared<SphereGreensFn>(param);
            else if (kname == "planarlog") kernel = std::make_shared<PlanarGreensFnFreeBoundaries>();
            else if (kname == "delta3d") kernel = std::make_shared<SecondOrderDelta3d>(param);
            else if (kname == "spheredelta") kernel = std::make_shared<SphereDelta>(param);
            else throw std::invalid_argument("KERNEL must be spheregreens, planarlog, delta3d or spheredelta");
            MPIReplicatedData mv(pm->nVertices(), 0, 1), mf(pm->nFaces(), 0, 1);
            DirectSum solver(pm, kernel, "potential", "vorticity");
            solver.meshSolve(mv, mf);
            const std::string out = argv[7];
            std::vector<double> vp(pm->nVertices()), fp(pm->nFaces());
            for (index_type i = 0; i < pm->nVertices(); ++i) vp[i] = pm->getVertexFieldPtr("potential")->getScalar(i);
            for (index_type i = 0; i < pm->nFaces(); ++i) fp[i] = pm->getFaceFieldPtr("potential")->getScalar(i);
            write_f64(out + "/vert_phi.bin", vp);
            write_f64(out + "/face_phi.bin", fp);
            std::printf("{\"cmd\": \"scalar\", \"kernel\": \"%s\"}\n", kname.c_str());
        } else if (cmd == "poisson" && argc == 5) {
            const long n = std::atol(argv[2]);
            const std::vector<double> p = read_f64(argv[3]);
            if ((long)p.size() != 4 * n) throw std::runtime_error("XYZQ.bin must hold N x 4 values");
            auto crds = std::make_shared<EuclideanCoords>(n, CARTESIAN_3D_GEOMETRY);
            auto q = std::make_shared<Field>(n, 1, "charge", "n/a");
            auto phi = std::make_shared<Field>(n, 1, "potential", "n/a");
            for (long i = 0; i < n; ++i) {
                crds->insert(p[4 * i], p[4 * i + 1], p[4 * i + 2]);
                q->insert(p[4 * i + 3]);
                phi->insert(0.0);
            }
            auto parts = std::make_shared<Particles>(crds, nullptr, std::vector<std::shared_ptr<Field>>{q, phi}, 0);
            auto kernel = std::make_shared<PoissonGreensFn3d>();
            MPIReplicatedData mp(n, 0, 1);
            DirectSum ds(parts, kernel, "potential", "charge");
            ds.meshfreeSolve(mp);
            std::vector<double> out(n);
            for (long i = 0; i < n; ++i) out[i] = phi->getScalar(i);
            write_f64(std::string(argv[4]) + "/potential.bin", out);
            std::printf("{\"cmd\": \"poisson\", \"n\": %ld}\n", n);
        } else if (cmd == "ptree" && argc == 5) {
            const long n = std::atol(argv[2]);
            const std::vector<double> p = read_f64(argv[3]);
            if ((long)p.size() != 3 * n) throw std::runtime_error("XYZ.bin must hold N x 3 values");
            auto crds = std::make_shared<EuclideanCoords>(n, CARTESIAN_3D_GEOMETRY);
            for (long i = 0; i < n; ++i) crds->insert(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
            TreeSum ts(crds, 8, std::atoi(argv[4]), 0.0);
            std::printf("{\"cmd\": \"ptree\", \"n_nodes\": %ld, \"depth\": %d}\n", (long)ts.nNodes(), ts.depth());
        } else {
            std::fprintf(stderr, "usage: see the header of dropin_driver.cpp\n");
            MPI_Finalize();
            return 2;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        MPI_Finalize();
        return 1;
    }
    MPI_Finalize();
    return 0;
}
