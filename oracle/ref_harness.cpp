/*
 * Test-infrastructure driver that runs the UNMODIFIED lpmCxx reference (compiled from its
 * own sources by oracle/Makefile, linked against oracle/mpi_stub/mpi.h) and writes its
 * inputs and outputs as .npy files.  It is the oracle's pin: golden fixtures under
 * tests/golden/ are produced by it (tests/golden/make_golden.py), and the CPU baseline
 * of bench.py times its `direct` command.  Nothing in the product links or runs it.
 *
 * Commands (all write into OUTDIR, which must exist):
 *   mesh     KIND LEVEL OUTDIR                    PolyMesh2d ctor          (src/LpmPolyMesh2d.cpp:20-93)
 *   direct   KIND LEVEL ZETA DELTA OUTDIR          DirectSum::meshSolve     (src/LpmDirectSum.cpp:94-167)
 *   tree     KIND LEVEL MAXLEAF OUTDIR             TreeSum mesh ctor + tree (src/LpmTreeSum.cpp:221-238,266-290)
 *   treesum  KIND LEVEL ZETA P MAXLEAF THETA OUTDIR  TreeSum::computeMeshMoments + meshSolve
 *                                                  (src/LpmTreeSum.cpp:55-86,106-197)
 *   scalar   KIND LEVEL ZETA KERNEL PARAM OUTDIR   DirectSum::meshSolve, scalar branch (src/LpmDirectSum.cpp:29-93)
 *                                                  with the reference's ScalarKernel KERNEL: spheregreens (PARAM =
 *                                                  radius), planarlog, delta3d / spheredelta (PARAM = eps)
 *   vtk      KIND LEVEL ZETA LAG OUTDIR            MeshedParticles::writeToVtkFile (src/LpmMeshedParticles.cpp:131-153)
 *                                                  of a mesh (Lagrangian if LAG is 1) with the vorticity and its
 *                                                  DirectSum velocity as vertex and face fields -> OUTDIR/mesh.vtk;
 *                                                  VtkWriter::writePointsAndFieldsToCSV of the vertices with
 *                                                  (velocity, vorticity) -> OUTDIR/points.csv
 *   vtktime  KIND LEVEL OUTDIR                     times writeToVtkFile of the mesh with vorticity (rh) and a zero
 *                                                  velocity field (no solve) -> OUTDIR/mesh.vtk
 *   poisson  NPTS SEED OUTDIR                      DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:240-252)
 *   time_poisson NPTS SEED [REPS]                  the same on this rank's slice, timed (CPU baseline)
 *   sakajo   KIND LEVEL DEPTH OUTDIR              SakajoTree(4, DEPTH) over the leaf-face centroids
 *                                                 (src/LpmSakajo2009.cpp:25-63,74-79,201-213): its non-empty nodes
 *                                                  with a 1/(4 pi r) ScalarKernel subclass
 *   pointtree NPTS SEED MAXLEAF OUTDIR             TreeSum(coords,...) meshfree ctor (src/LpmTreeSum.cpp:208-219)
 * KIND is icos|cube.  ZETA is rh (2z - sphereHarmonic54, the Rossby-Haurwitz m=4 wave with
 * omega=K=1), harm (sphereHarmonic54) or gauss (4 pi exp(-16|x-x0|^2) minus its area-weighted
 * mean, x0 at lat 0.05, lon 3 pi/4).  The target slice follows the MPI stub's
 * LPM_STUB_RANK / LPM_STUB_SIZE (the reference's own MPIReplicatedData split).
 */
#include "LpmConfig.h"
#include "LpmTypeDefs.h"
#include "LpmXyzVector.h"
#include "LpmMeshSeed.h"
#include "LpmMeshedParticles.h"
#include "LpmAnalyticFunctions.h"
#include "LpmMPIReplicatedData.h"
#include "LpmDirectSum.h"
#include "LpmTreeSum.h"
#include "LpmSakajo2009.h"
#include "LpmSphericalCoords.h"
#include "LpmVtkFileIO.h"
#include <fstream>
#include "LpmEuclideanCoords.h"
#include "LpmParticles.h"
#include <mpi.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <string>
#include <vector>
#include <memory>
#include <new>
#include <stdexcept>
#include <chrono>
#include <iostream>

using namespace Lpm;

// ---------------------------------------------------------------- .npy writer
static void write_npy(const std::string& path, const char* descr, size_t elsize,
                      const std::vector<int64_t>& shape, const void* data) {
    std::string hdr = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (";
    size_t count = 1;
    for (size_t i = 0; i < shape.size(); ++i) {
        hdr += std::to_string(shape[i]);
        hdr += (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
        count *= (size_t)shape[i];
    }
    hdr += "), }";
    size_t total = 10 + hdr.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    hdr += std::string(pad, ' ');
    hdr += "\n";
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    fwrite(magic, 1, 8, f);
    uint16_t hl = (uint16_t)hdr.size();
    fwrite(&hl, 2, 1, f);
    fwrite(hdr.data(), 1, hdr.size(), f);
    if (count) fwrite(data, elsize, count, f);
    fclose(f);
}
static void npy_f64(const std::string& dir, const std::string& name, const std::vector<double>& v,
                    int64_t cols = 1) {
    std::vector<int64_t> shape = cols == 1 ? std::vector<int64_t>{(int64_t)v.size()}
                                           : std::vector<int64_t>{(int64_t)v.size() / cols, cols};
    write_npy(dir + "/" + name + ".npy", "<f8", 8, shape, v.data());
}
static void npy_i64(const std::string& dir, const std::string& name, const std::vector<int64_t>& v) {
    write_npy(dir + "/" + name + ".npy", "<i8", 8, {(int64_t)v.size()}, v.data());
}
static void npy_u8(const std::string& dir, const std::string& name, const std::vector<uint8_t>& v) {
    write_npy(dir + "/" + name + ".npy", "|u1", 1, {(int64_t)v.size()}, v.data());
}

// ---------------------------------------------------------------- inputs
static std::unique_ptr<MeshSeed> make_seed(const std::string& kind) {
    if (kind == "icos") return std::unique_ptr<MeshSeed>(new IcosTriSphereSeed());
    if (kind == "cube") return std::unique_ptr<MeshSeed>(new CubedSphereSeed());
    throw std::invalid_argument("KIND must be icos or cube");
}

class RHWave4 : public AnalyticFunction {  // 2 omega sin(phi) - 30 cos^4 sin cos(4 lambda), omega=K=1
  public:
    scalar_type evaluateScalar(const XyzVector& v) const override { return 2.0 * v.z - harm.evaluateScalar(v); }
    scalar_type evaluateScalar(const scalar_type x, const scalar_type y, const scalar_type z) const override {
        return evaluateScalar(XyzVector(x, y, z));
    }
    sphereHarmonic54 harm;
};

class GaussVortex : public AnalyticFunction {  // 4 pi exp(-16 |x - x0|^2)
  public:
    GaussVortex() {
        const double lat = 0.05, lon = 3.0 * PI / 4.0;
        x0 = XyzVector(std::cos(lat) * std::cos(lon), std::cos(lat) * std::sin(lon), std::sin(lat));
    }
    scalar_type evaluateScalar(const XyzVector& v) const override {
        const XyzVector d = v - x0;
        return 4.0 * PI * std::exp(-16.0 * d.magnitudeSquared());
    }
    scalar_type evaluateScalar(const scalar_type x, const scalar_type y, const scalar_type z) const override {
        return evaluateScalar(XyzVector(x, y, z));
    }
    XyzVector x0;
};

static void init_vorticity(MeshedParticles& pm, const std::string& zeta) {
    pm.createVertexField("vorticity", "1/time", 1);
    pm.createFaceField("vorticity", "1/time", 1);
    if (zeta == "rh") {
        RHWave4 f;
        pm.initializeVertexFieldWithFunction("vorticity", &f);
        pm.initializeFaceFieldWithFunction("vorticity", &f);
    } else if (zeta == "harm") {
        sphereHarmonic54 f;
        pm.initializeVertexFieldWithFunction("vorticity", &f);
        pm.initializeFaceFieldWithFunction("vorticity", &f);
    } else if (zeta == "gauss") {
        GaussVortex f;
        pm.initializeVertexFieldWithFunction("vorticity", &f);
        pm.initializeFaceFieldWithFunction("vorticity", &f);
        // subtract the area-weighted mean over leaf faces (total circulation zero)
        std::shared_ptr<Field> fz = pm.getFaceFieldPtr("vorticity");
        double num = 0.0, den = 0.0;
        for (index_type i = 0; i < pm.nFaces(); ++i) {
            if (!pm.faceIsDivided(i)) {
                num += fz->getScalar(i) * pm.getFaceArea(i);
                den += pm.getFaceArea(i);
            }
        }
        const double mean = num / den;
        for (index_type i = 0; i < pm.nFaces(); ++i)
            if (!pm.faceIsDivided(i)) fz->replace(i, fz->getScalar(i) - mean);
        std::shared_ptr<Field> vz = pm.getVertexFieldPtr("vorticity");
        for (index_type i = 0; i < pm.nVertices(); ++i) vz->replace(i, vz->getScalar(i) - mean);
    } else {
        throw std::invalid_argument("ZETA must be rh, harm or gauss");
    }
}

static void dump_mesh(MeshedParticles& pm, const std::string& out) {
    const index_type nv = pm.nVertices(), nf = pm.nFaces();
    std::vector<double> vxyz(3 * nv), fxyz(3 * nf), farea(nf);
    std::vector<uint8_t> divided(nf);
    for (index_type i = 0; i < nv; ++i) {
        const XyzVector v = pm.getVertex(i);
        vxyz[3 * i] = v.x; vxyz[3 * i + 1] = v.y; vxyz[3 * i + 2] = v.z;
    }
    for (index_type i = 0; i < nf; ++i) {
        const XyzVector c = pm.getFaceCentroid(i);
        fxyz[3 * i] = c.x; fxyz[3 * i + 1] = c.y; fxyz[3 * i + 2] = c.z;
        farea[i] = pm.getFaceArea(i);
        divided[i] = pm.faceIsDivided(i) ? 1 : 0;
    }
    npy_f64(out, "vert_xyz", vxyz, 3);
    npy_f64(out, "face_xyz", fxyz, 3);
    npy_f64(out, "face_area", farea);
    npy_u8(out, "face_divided", divided);
}

static std::vector<double> field3(const std::shared_ptr<Field>& f, index_type n) {
    std::vector<double> out(3 * n);
    for (index_type i = 0; i < n; ++i) {
        const XyzVector v = f->get3dVector(i);
        out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
    }
    return out;
}

// A TreeSum with access to its (protected) node tree.  Built on zero-filled storage:
// the mesh ctor leaves _smooth and _shrink uninitialised (src/LpmTreeSum.cpp:221-226,
// src/LpmTreeSum.h:86-87); zero storage gives the no-shrink, no-smoothing behaviour the
// ctor's callers expect, deterministically.
struct TreeProbe : public TreeSum {
    using TreeSum::TreeSum;
    void walk(const Node* node, int64_t parent, std::vector<int64_t>& level, std::vector<int64_t>& par,
              std::vector<int64_t>& nkids, std::vector<int64_t>& ncoords, std::vector<double>& box,
              std::vector<int64_t>& leaf_begin, std::vector<int64_t>& members) const {
        const int64_t me = (int64_t)level.size();
        level.push_back(node->level);
        par.push_back(parent);
        nkids.push_back((int64_t)node->kids.size());
        ncoords.push_back((int64_t)node->coordsContained.size());
        const Box3d& b = node->box;
        const double bb[8] = {b.xmin, b.xmax, b.ymin, b.ymax, b.zmin, b.zmax, b.maxRadius, 0.0};
        box.insert(box.end(), bb, bb + 8);
        if (node->kids.empty()) {
            leaf_begin.push_back((int64_t)members.size());
            for (index_type j : node->coordsContained) members.push_back((int64_t)j);
        }
        for (const auto& k : node->kids)
            walk(k.get(), me, level, par, nkids, ncoords, box, leaf_begin, members);
    }
    void dump(const std::string& out) const {
        std::vector<int64_t> level, par, nkids, ncoords, leaf_begin, members;
        std::vector<double> box;
        walk(_root.get(), -1, level, par, nkids, ncoords, box, leaf_begin, members);
        leaf_begin.push_back((int64_t)members.size());
        npy_i64(out, "node_level", level);
        npy_i64(out, "node_parent", par);
        npy_i64(out, "node_nkids", nkids);
        npy_i64(out, "node_ncoords", ncoords);
        npy_f64(out, "node_box", box, 8);
        npy_i64(out, "leaf_offsets", leaf_begin);
        npy_i64(out, "leaf_members", members);
    }
};

// SakajoTree's nodes after computeMoments: the non-empty ones (holding at least one point below them) in
// depth-first order with their level, parent, point count and box, and the leaf membership at full depth.
struct SakajoProbe : public SakajoTree {
    using SakajoTree::SakajoTree;
    int64_t count(const Node* node) const {
        int64_t c = (int64_t)node->coordsContained.size();
        for (const auto& k : node->kids) c += count(k.get());
        return c;
    }
    void walk(const Node* node, int64_t parent, std::vector<int64_t>& level, std::vector<int64_t>& par,
              std::vector<int64_t>& ncoords, std::vector<double>& box, std::vector<int64_t>& leaf_begin,
              std::vector<int64_t>& members) const {
        const int64_t c = count(node);
        if (c == 0) return;
        const int64_t me = (int64_t)level.size();
        level.push_back(node->level);
        par.push_back(parent);
        ncoords.push_back(c);
        const Box3d& b = node->box;
        const double bb[6] = {b.xmin, b.xmax, b.ymin, b.ymax, b.zmin, b.zmax};
        box.insert(box.end(), bb, bb + 6);
        if (!node->coordsContained.empty()) {
            leaf_begin.push_back((int64_t)members.size());
            for (index_type j : node->coordsContained) members.push_back((int64_t)j);
        }
        for (const auto& k : node->kids) walk(k.get(), me, level, par, ncoords, box, leaf_begin, members);
    }
    void dump(const std::string& out) const {
        std::vector<int64_t> level, par, ncoords, leaf_begin, members;
        std::vector<double> box;
        walk(_root.get(), -1, level, par, ncoords, box, leaf_begin, members);
        leaf_begin.push_back((int64_t)members.size());
        npy_i64(out, "node_level", level);
        npy_i64(out, "node_parent", par);
        npy_i64(out, "node_ncoords", ncoords);
        npy_f64(out, "node_box", box, 6);
        npy_i64(out, "leaf_offsets", leaf_begin);
        npy_i64(out, "leaf_members", members);
        npy_i64(out, "n_nodes_all", {(int64_t)_nnodes});
    }
};

template <typename... Args>
static TreeProbe* new_zeroed_probe(Args&&... args) {
    void* mem = ::operator new(sizeof(TreeProbe));
    std::memset(mem, 0, sizeof(TreeProbe));
    return new (mem) TreeProbe(std::forward<Args>(args)...);
}

// 1/(4 pi |x - y|) with the self term returning 0 (reported non-singular so that
// DirectSum::meshfreeSolve takes its correct-bound loop, src/LpmDirectSum.cpp:240-252).
class Poisson3dKernel : public ScalarKernel {
  public:
    scalar_type evaluate(const XyzVector& t, const XyzVector& s) const override {
        const XyzVector d = t - s;
        const scalar_type r = d.magnitude();
        return r > 0.0 ? 1.0 / (4.0 * PI * r) : 0.0;
    }
    bool isSingular() const override { return false; }
};

// splitmix64 -> uniform doubles in [-1, 1): the seeded generator of the 3D Poisson workload.
static uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double uniform_pm1(uint64_t& s) { return 2.0 * ((splitmix64(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0; }

static int usage() {
    fprintf(stderr, "usage: ref_harness mesh|direct|scalar|vtk|tree|treesum|poisson|time_poisson|sakajo|pointtree ...\n");
    return 2;
}

int main(int argc, char** argv) {
    MPI_Init(&argc, &argv);
    int rank = 0, size = 1;
    MPI_Comm_rank(MPI_COMM_WORLD, &rank);
    MPI_Comm_size(MPI_COMM_WORLD, &size);
    if (argc < 2) return usage();
    const std::string cmd = argv[1];
    try {
        if (cmd == "mesh" && argc == 5) {
            auto seed = make_seed(argv[2]);
            MeshedParticles pm(*seed, atoi(argv[3]), false, 1.0, rank);
            dump_mesh(pm, argv[4]);
        } else if (cmd == "direct" && argc == 7) {
            auto seed = make_seed(argv[2]);
            const std::string out = argv[6];
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, argv[4]);
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            std::shared_ptr<VectorKernel> kernel(new BiotSavartSphere(atof(argv[5])));
            MPIReplicatedData mv(pm->nVertices(), rank, size), mf(pm->nFaces(), rank, size);
            DirectSum solver(pm, kernel, "velocity", "vorticity");
            const auto t0 = std::chrono::steady_clock::now();
            solver.meshSolve(mv, mf);
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            solver.meshBroadcast(mv, mf);
            if (rank == 0) dump_mesh(*pm, out);
            std::vector<double> fz(pm->nFaces());
            for (index_type i = 0; i < pm->nFaces(); ++i) fz[i] = pm->getFaceFieldPtr("vorticity")->getScalar(i);
            const std::string tag = size > 1 ? "_r" + std::to_string(rank) : "";
            npy_f64(out, "face_zeta" + tag, fz);
            npy_f64(out, "vert_vel" + tag, field3(pm->getVertexFieldPtr("velocity"), pm->nVertices()), 3);
            npy_f64(out, "face_vel" + tag, field3(pm->getFaceFieldPtr("velocity"), pm->nFaces()), 3);
            npy_i64(out, "slice" + tag, {mv.startIndex(rank), mv.endIndex(rank), mf.startIndex(rank), mf.endIndex(rank)});
            printf("{\"cmd\": \"direct\", \"rank\": %d, \"size\": %d, \"seconds\": %.6f}\n", rank, size, secs);
        } else if (cmd == "time_direct" && (argc == 5 || argc == 6)) {
            // times DirectSum::meshSolve on this rank's slice only (no output files), REPS times: the
            // CPU baseline.  Prints one JSON line with the per-repetition seconds.
            auto seed = make_seed(argv[2]);
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, argv[4]);
            const int reps = argc == 6 ? atoi(argv[5]) : 1;
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            std::shared_ptr<VectorKernel> kernel(new BiotSavartSphere());
            MPIReplicatedData mv(pm->nVertices(), rank, size), mf(pm->nFaces(), rank, size);
            DirectSum solver(pm, kernel, "velocity", "vorticity");
            std::string secs = "[";
            for (int r = 0; r < reps; ++r) {
                const auto t0 = std::chrono::steady_clock::now();
                solver.meshSolve(mv, mf);
                const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                secs += (r ? ", " : "") + std::to_string(s);
            }
            secs += "]";
            long nft = 0;
            for (index_type i = mf.startIndex(rank); i <= mf.endIndex(rank); ++i) nft += pm->faceIsDivided(i) ? 0 : 1;
            printf("{\"cmd\": \"time_direct\", \"rank\": %d, \"size\": %d, \"seconds\": %s, \"vert_targets\": %ld, "
                   "\"face_targets\": %ld, \"sources\": %ld, \"n_verts\": %ld, \"n_leaves\": %ld}\n",
                   rank, size, secs.c_str(), (long)mv.msgSize(rank), nft, (long)pm->nLeafFaces(),
                   (long)pm->nVertices(), (long)pm->nLeafFaces());
        } else if (cmd == "tree" && argc == 6) {
            auto seed = make_seed(argv[2]);
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, "rh");
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            std::shared_ptr<VectorKernel> kernel(new BiotSavartSphere());
            TreeProbe* tree = new_zeroed_probe(8, atoi(argv[4]), pm, kernel, std::string("velocity"),
                                               std::string("vorticity"));
            tree->dump(argv[5]);
            npy_f64(argv[5], "maxr", {pm->maxR()});
            tree->~TreeProbe();
            ::operator delete(tree);
        } else if (cmd == "treesum" && argc == 9) {
            auto seed = make_seed(argv[2]);
            const std::string out = argv[8];
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, argv[4]);
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            std::shared_ptr<VectorKernel> kernel(new BiotSavartSphere());
            TreeProbe* tree = new_zeroed_probe(atoi(argv[5]), atoi(argv[6]), pm, kernel, std::string("velocity"),
                                               std::string("vorticity"));
            MPIReplicatedData mv(pm->nVertices(), rank, size), mf(pm->nFaces(), rank, size);
            const auto t0 = std::chrono::steady_clock::now();
            tree->computeMeshMoments();
            int mac = 0;
            tree->meshSolve(mv, mf, atof(argv[7]), mac);
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            tree->dump(out);
            std::vector<double> fz(pm->nFaces());
            for (index_type i = 0; i < pm->nFaces(); ++i) fz[i] = pm->getFaceFieldPtr("vorticity")->getScalar(i);
            npy_f64(out, "face_zeta", fz);
            npy_f64(out, "vert_vel", field3(pm->getVertexFieldPtr("velocity"), pm->nVertices()), 3);
            npy_f64(out, "face_vel", field3(pm->getFaceFieldPtr("velocity"), pm->nFaces()), 3);
            npy_i64(out, "mac_count", {(int64_t)mac});
            printf("{\"cmd\": \"treesum\", \"mac\": %d, \"seconds\": %.6f}\n", mac, secs);
            tree->~TreeProbe();
            ::operator delete(tree);
        } else if (cmd == "scalar" && argc == 8) {
            auto seed = make_seed(argv[2]);
            const std::string out = argv[7], kname = argv[5];
            const double param = atof(argv[6]);
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, argv[4]);
            pm->createVertexField("potential", "n/a", 1);
            pm->createFaceField("potential", "n/a", 1);
            std::shared_ptr<ScalarKernel> kernel;
            if (kname == "spheregreens") kernel.reset(new SphereGreensFn(param));
            else if (kname == "planarlog") kernel.reset(new PlanarGreensFnFreeBoundaries());
            else if (kname == "delta3d") kernel.reset(new SecondOrderDelta3d(param));
            else if (kname == "spheredelta") kernel.reset(new SphereDelta(param));
            else throw std::invalid_argument("KERNEL must be spheregreens, planarlog, delta3d or spheredelta");
            MPIReplicatedData mv(pm->nVertices(), rank, size), mf(pm->nFaces(), rank, size);
            DirectSum solver(pm, kernel, "potential", "vorticity");
            const auto t0 = std::chrono::steady_clock::now();
            solver.meshSolve(mv, mf);
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::vector<double> fz(pm->nFaces()), vp(pm->nVertices()), fp(pm->nFaces());
            for (index_type i = 0; i < pm->nFaces(); ++i) {
                fz[i] = pm->getFaceFieldPtr("vorticity")->getScalar(i);
                fp[i] = pm->getFaceFieldPtr("potential")->getScalar(i);
            }
            for (index_type i = 0; i < pm->nVertices(); ++i) vp[i] = pm->getVertexFieldPtr("potential")->getScalar(i);
            npy_f64(out, "face_zeta", fz);
            npy_f64(out, "vert_phi", vp);
            npy_f64(out, "face_phi", fp);
            printf("{\"cmd\": \"scalar\", \"kernel\": \"%s\", \"seconds\": %.6f}\n", kname.c_str(), secs);
        } else if (cmd == "vtk" && argc == 7) {
            auto seed = make_seed(argv[2]);
            const std::string out = argv[6];
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), atoi(argv[5]) != 0, 1.0, rank);
            init_vorticity(*pm, argv[4]);
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            std::shared_ptr<VectorKernel> kernel(new BiotSavartSphere());
            MPIReplicatedData mv(pm->nVertices(), rank, size), mf(pm->nFaces(), rank, size);
            DirectSum solver(pm, kernel, "velocity", "vorticity");
            solver.meshSolve(mv, mf);
            pm->writeToVtkFile(out + "/mesh.vtk", "lpm vtk test");
            {
                VtkWriter writer;
                std::ofstream fs(out + "/points.csv");
                writer.writePointsAndFieldsToCSV(fs, pm->getCoordPtr(false),
                                                 {pm->getVertexFieldPtr("velocity"), pm->getVertexFieldPtr("vorticity")});
            }
            std::vector<double> vz(pm->nVertices()), fz(pm->nFaces());
            for (index_type i = 0; i < pm->nVertices(); ++i) vz[i] = pm->getVertexFieldPtr("vorticity")->getScalar(i);
            for (index_type i = 0; i < pm->nFaces(); ++i) fz[i] = pm->getFaceFieldPtr("vorticity")->getScalar(i);
            npy_f64(out, "vert_zeta", vz);
            npy_f64(out, "face_zeta", fz);
            npy_f64(out, "vert_vel", field3(pm->getVertexFieldPtr("velocity"), pm->nVertices()), 3);
            npy_f64(out, "face_vel", field3(pm->getFaceFieldPtr("velocity"), pm->nFaces()), 3);
        } else if (cmd == "vtktime" && argc == 5) {
            auto seed = make_seed(argv[2]);
            const std::string out = argv[4];
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, "rh");
            pm->createVertexField("velocity", "length/time", 3);
            pm->createFaceField("velocity", "length/time", 3);
            const auto t0 = std::chrono::steady_clock::now();
            pm->writeToVtkFile(out + "/mesh.vtk", "lpm vtk test");
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            printf("{\"cmd\": \"vtktime\", \"seconds\": %.6f}\n", secs);
        } else if (cmd == "poisson" && argc == 5) {
            const index_type n = atol(argv[2]);
            uint64_t s = strtoull(argv[3], nullptr, 0);
            auto crds = std::make_shared<EuclideanCoords>(n, CARTESIAN_3D_GEOMETRY);
            auto q = std::make_shared<Field>(n, 1, "charge", "n/a");
            auto phi = std::make_shared<Field>(n, 1, "potential", "n/a");
            std::vector<double> xyz(3 * n), qv(n);
            for (index_type i = 0; i < n; ++i) {
                xyz[3 * i] = uniform_pm1(s); xyz[3 * i + 1] = uniform_pm1(s); xyz[3 * i + 2] = uniform_pm1(s);
                crds->insert(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
            }
            for (index_type i = 0; i < n; ++i) { qv[i] = uniform_pm1(s); q->insert(qv[i]); phi->insert(0.0); }
            auto parts = std::make_shared<Particles>(crds, nullptr,
                                                     std::vector<std::shared_ptr<Field>>{q, phi}, rank);
            std::shared_ptr<ScalarKernel> kernel(new Poisson3dKernel());
            DirectSum solver(parts, kernel, "potential", "charge");
            MPIReplicatedData mp(n, rank, size);
            const auto t0 = std::chrono::steady_clock::now();
            solver.meshfreeSolve(mp);
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::vector<double> pv(n);
            for (index_type i = 0; i < n; ++i) pv[i] = phi->getScalar(i);
            const std::string out = argv[4];
            npy_f64(out, "xyz", xyz, 3);
            npy_f64(out, "charge", qv);
            npy_f64(out, "potential", pv);
            printf("{\"cmd\": \"poisson\", \"seconds\": %.6f}\n", secs);
        } else if (cmd == "time_poisson" && (argc == 4 || argc == 5)) {
            // times DirectSum::meshfreeSolve (1/(4 pi r) kernel) on this rank's MPIReplicatedData slice of
            // the NPTS-point splitmix64 cube, REPS times (no output files): the 3D Poisson CPU baseline
            const index_type n = atol(argv[2]);
            uint64_t s = strtoull(argv[3], nullptr, 0);
            const int reps = argc == 5 ? atoi(argv[4]) : 1;
            auto crds = std::make_shared<EuclideanCoords>(n, CARTESIAN_3D_GEOMETRY);
            auto q = std::make_shared<Field>(n, 1, "charge", "n/a");
            auto phi = std::make_shared<Field>(n, 1, "potential", "n/a");
            for (index_type i = 0; i < n; ++i) {
                const double x = uniform_pm1(s), y = uniform_pm1(s), z = uniform_pm1(s);
                crds->insert(x, y, z);
                const double c = uniform_pm1(s);
                q->insert(c);
                phi->insert(0.0);
            }
            auto parts = std::make_shared<Particles>(crds, nullptr,
                                                     std::vector<std::shared_ptr<Field>>{q, phi}, rank);
            std::shared_ptr<ScalarKernel> kernel(new Poisson3dKernel());
            DirectSum solver(parts, kernel, "potential", "charge");
            MPIReplicatedData mp(n, rank, size);
            std::string secs = "[";
            for (int r = 0; r < reps; ++r) {
                const auto t0 = std::chrono::steady_clock::now();
                solver.meshfreeSolve(mp);
                const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                secs += (r ? ", " : "") + std::to_string(t);
            }
            secs += "]";
            printf("{\"cmd\": \"time_poisson\", \"rank\": %d, \"size\": %d, \"seconds\": %s, \"targets\": %ld, "
                   "\"sources\": %ld}\n", rank, size, secs.c_str(), (long)mp.msgSize(rank), (long)n);
        } else if (cmd == "sakajo" && argc == 6) {
            // SakajoTree(order 4, DEPTH, radius 1) over the leaf-face centroids of a mesh, computeMoments with
            // the RH circulation, then the non-empty nodes and the full-depth leaf membership
            auto seed = make_seed(argv[2]);
            auto pm = std::make_shared<MeshedParticles>(*seed, atoi(argv[3]), false, 1.0, rank);
            init_vorticity(*pm, "rh");
            auto sc = std::make_shared<SphericalCoords>(pm->nLeafFaces());
            auto circ = std::make_shared<Field>(pm->nLeafFaces(), 1, "circulation", "n/a");
            std::vector<double> xyz;
            for (index_type i = 0; i < pm->nFaces(); ++i) {
                if (pm->faceIsDivided(i)) continue;
                const XyzVector c = pm->getFaceCentroid(i);
                sc->insert(c.x, c.y, c.z);
                circ->insert(pm->getFaceFieldPtr("vorticity")->getScalar(i) * pm->getFaceArea(i));
                xyz.push_back(c.x); xyz.push_back(c.y); xyz.push_back(c.z);
            }
            SakajoProbe tree(4, atoi(argv[4]), 1.0, 0.0, rank);
            tree.computeMoments(sc, circ);
            tree.dump(argv[5]);
            npy_f64(argv[5], "xyz", xyz, 3);
        } else if (cmd == "pointtree" && argc == 6) {
            const index_type n = atol(argv[2]);
            uint64_t s = strtoull(argv[3], nullptr, 0);
            auto crds = std::make_shared<EuclideanCoords>(n, CARTESIAN_3D_GEOMETRY);
            std::vector<double> xyz(3 * n);
            for (index_type i = 0; i < n; ++i) {
                xyz[3 * i] = uniform_pm1(s); xyz[3 * i + 1] = uniform_pm1(s); xyz[3 * i + 2] = uniform_pm1(s);
                crds->insert(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
            }
            TreeProbe* tree = new_zeroed_probe(std::static_pointer_cast<Coords>(crds), 4, atoi(argv[4]), 0.0, false);
            const std::string out = argv[5];
            tree->dump(out);
            npy_f64(out, "xyz", xyz, 3);
            tree->~TreeProbe();
            ::operator delete(tree);
        } else {
            return usage();
        }
    } catch (const std::exception& e) {
        fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
    MPI_Finalize();
    return 0;
}
