"""Regenerate the golden fixtures in this directory from the UNMODIFIED lpmCxx reference.

    make -C oracle ref && python tests/golden/make_golden.py

The reference is compiled from its own sources by oracle/Makefile (target `ref`) against the
single-rank MPI stub in oracle/mpi_stub/; oracle/ref_harness.cpp drives its public API and dumps
.npy files, which this script packs into small .npz fixtures.  The fixtures are committed; the
reference tree itself is not needed to run the tests.

Fixtures
  mesh_{icos,cube}3.npz      PolyMesh2d(seed, 3): vertices, centroids, areas, divided mask
  direct_icos4_rh.npz        DirectSum::meshSolve, BiotSavartSphere(), icos level 4, RH m=4 wave
  direct_cube3_gauss_d05.npz DirectSum::meshSolve, BiotSavartSphere(0.05) (non-singular branch),
                             cube level 3, Gaussian vortex
  direct_icos3_rh_r2.npz     MPIReplicatedData rank 1 of 3: only that rank's target slice is written
  poisson_2000.npz           DirectSum::meshfreeSolve with a 1/(4 pi r) ScalarKernel, 2000 points
  scalar_icos3_harm.npz      DirectSum::meshSolve, scalar branch, with the reference's SphereGreensFn(1),
                             PlanarGreensFnFreeBoundaries, SecondOrderDelta3d(0.1) and SphereDelta(0.1);
                             icos level 3, zeta = sphereHarmonic54
  tree_icos8_m512.npz        TreeSum's mesh constructor at the treecode's full size (icos level 8, 512 per
                             leaf): node levels, parents, counts, boxes, leaf offsets and a digest of each
                             leaf's members (oracle.leaf_hashes) instead of the 1.3M member indices
  sakajo_icos4_d3.npz,       SakajoTree(4, depth) over the leaf-face centroids (icos level 4 depth 3, cube level 4
  sakajo_cube4_d2.npz        depth 2): its non-empty nodes and full-depth leaf membership, and the points
  vtk_icos2_rh.npz,          MeshedParticles::writeToVtkFile (non-Lagrangian icos level 2 / Lagrangian cube
  vtk_cube2_gauss_lag.npz    level 2) with vorticity and DirectSum velocity fields, and
                             VtkWriter::writePointsAndFieldsToCSV of the vertices: the files' bytes and the
                             field values written
`python make_golden.py scalar vtk tree8 sakajo` remakes only the named groups.
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402


def harness(*args, env=None) -> Path:
    out = Path(tempfile.mkdtemp(prefix="lpm_golden_"))
    oracle.run_ref_harness(*args, out, env=env)
    return out


def load(d: Path, *names) -> dict:
    return {n: np.load(d / f"{n}.npy") for n in names}


SCALAR_KERNELS = (("spheregreens", 1.0), ("planarlog", 0.0), ("delta3d", 0.1), ("spheredelta", 0.1))


def scalar_fixture() -> None:
    z = {}
    for name, param in SCALAR_KERNELS:
        d = harness("scalar", "icos", 3, "harm", name, param)
        z["face_zeta"] = np.load(d / "face_zeta.npy")
        z[f"{name}_vert_phi"] = np.load(d / "vert_phi.npy")
        z[f"{name}_face_phi"] = np.load(d / "face_phi.npy")
        z[f"{name}_param"] = np.array(param)
    np.savez_compressed(HERE / "scalar_icos3_harm.npz", **z)


def vtk_fixtures() -> None:
    for kind, level, zeta, lag, name in (("icos", 2, "rh", 0, "vtk_icos2_rh"), ("cube", 2, "gauss", 1, "vtk_cube2_gauss_lag")):
        d = harness("vtk", kind, level, zeta, lag)
        z = load(d, "vert_zeta", "face_zeta", "vert_vel", "face_vel")
        z["vtk"] = np.frombuffer((d / "mesh.vtk").read_bytes(), dtype=np.uint8)
        z["csv"] = np.frombuffer((d / "points.csv").read_bytes(), dtype=np.uint8)
        np.savez_compressed(HERE / f"{name}.npz", **z)


def tree8_fixture() -> None:
    d = harness("tree", "icos", 8, 512)
    z = load(d, "node_level", "node_parent", "node_nkids", "node_ncoords", "node_box", "leaf_offsets",
             "leaf_members", "maxr")
    np.savez_compressed(HERE / "tree_icos8_m512.npz", maxr=z["maxr"], node_level=z["node_level"].astype(np.int8),
                        node_parent=z["node_parent"].astype(np.int32), node_nkids=z["node_nkids"].astype(np.int8),
                        node_ncoords=z["node_ncoords"].astype(np.int32), node_box=z["node_box"][:, :6],
                        leaf_offsets=z["leaf_offsets"].astype(np.int32),
                        leaf_hash=oracle.leaf_hashes(z["leaf_members"], z["leaf_offsets"]))


def sakajo_fixture() -> None:
    for kind, level, depth in (("icos", 4, 3), ("cube", 4, 2)):
        d = harness("sakajo", kind, level, depth)
        z = load(d, "node_level", "node_parent", "node_ncoords", "node_box", "leaf_offsets", "leaf_members",
                 "n_nodes_all", "xyz")
        np.savez_compressed(HERE / f"sakajo_{kind}{level}_d{depth}.npz", **z)


def main() -> None:
    groups = {"scalar": scalar_fixture, "vtk": vtk_fixtures, "tree8": tree8_fixture, "sakajo": sakajo_fixture}
    if sys.argv[1:]:
        for g in sys.argv[1:]:
            groups[g]()
        return
    scalar_fixture()
    vtk_fixtures()
    tree8_fixture()
    sakajo_fixture()
    for kind in ("icos", "cube"):
        d = harness("mesh", kind, 3)
        np.savez_compressed(HERE / f"mesh_{kind}3.npz",
                            **load(d, "vert_xyz", "face_xyz", "face_area", "face_divided"))

    d = harness("direct", "icos", 4, "rh", 0.0)
    np.savez_compressed(HERE / "direct_icos4_rh.npz", **load(d, "face_zeta", "vert_vel", "face_vel"),
                        face_xyz_sum=np.load(d / "face_xyz.npy").sum(axis=0))

    d = harness("direct", "cube", 3, "gauss", 0.05)
    np.savez_compressed(HERE / "direct_cube3_gauss_d05.npz", **load(d, "face_zeta", "vert_vel", "face_vel"))

    d = harness("direct", "icos", 3, "rh", 0.0, env={"LPM_STUB_RANK": "1", "LPM_STUB_SIZE": "3"})
    np.savez_compressed(HERE / "direct_icos3_rh_r2.npz", face_zeta=np.load(d / "face_zeta_r1.npy"),
                        vert_vel=np.load(d / "vert_vel_r1.npy"), face_vel=np.load(d / "face_vel_r1.npy"),
                        slice=np.load(d / "slice_r1.npy"))

    d = harness("poisson", 2000, "0x2B")
    np.savez_compressed(HERE / "poisson_2000.npz", **load(d, "xyz", "charge", "potential"))

    # octrees: TreeSum's mesh constructor (leaf-face centroids, Box3d(maxR) root) and its meshfree
    # constructor (Tree(coords) root with relative padding)
    for kind, level, max_leaf in (("icos", 4, 64), ("icos", 5, 100), ("cube", 4, 32)):
        d = harness("tree", kind, level, max_leaf)
        z = load(d, "node_level", "node_parent", "node_nkids", "node_ncoords", "node_box", "leaf_offsets",
                 "leaf_members", "maxr")
        z["leaf_members"] = z["leaf_members"].astype(np.int32)
        np.savez_compressed(HERE / f"tree_{kind}{level}_m{max_leaf}.npz", **z)
    d = harness("pointtree", 8000, "0x5EED", 10)
    z = load(d, "node_level", "node_parent", "node_nkids", "node_ncoords", "node_box", "leaf_offsets",
             "leaf_members", "xyz")
    np.savez_compressed(HERE / "pointtree_8000_m10.npz", **z)

    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
