"""Octree: leaf membership and node structure bit-exact against the reference's TreeSum trees
(golden fixtures made by the unmodified reference); the oracle on CPU, the CUDA build on GPU."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import oracle
from conftest import golden

MESH_TREES = [("icos", 4, 64), ("icos", 5, 100), ("cube", 4, 32)]


def mesh_points(kind, level):
    m = L.build_mesh(kind, level)
    leaf_faces = np.nonzero(m.leaf)[0]
    return m, leaf_faces, oracle.pack4(m.face_xyz[leaf_faces])


def ref_box(g):
    # reference dumps the box as xmin,xmax,ymin,ymax,zmin,zmax,maxRadius,0
    return g["node_box"][:, :6]


def check_against_reference(g, members, offsets, nodes, to_ref_index):
    assert np.array_equal(offsets, g["leaf_offsets"])
    assert np.array_equal(to_ref_index(members), g["leaf_members"].astype(np.int64))
    assert np.array_equal(nodes["node_level"], g["node_level"])
    assert np.array_equal(nodes["node_parent"], g["node_parent"])
    assert np.array_equal(nodes["node_count"], g["node_ncoords"])
    assert np.array_equal(nodes["node_box"], ref_box(g))


@pytest.mark.parametrize("kind,level,max_leaf", MESH_TREES)
def test_oracle_tree_matches_reference(kind, level, max_leaf):
    g = golden(f"tree_{kind}{level}_m{max_leaf}.npz")
    m, leaf_faces, pts = mesh_points(kind, level)
    box = oracle.mesh_root_box(m.vert_xyz)
    assert box[1] == g["maxr"][0] + 1e-5
    t = oracle.tree_build(pts, box, max_leaf)
    assert t["flags"] == 0
    check_against_reference(g, t["members"], t["leaf_offsets"], t, lambda idx: leaf_faces[idx])


def test_oracle_pointtree_matches_reference():
    g = golden("pointtree_8000_m10.npz")
    xyz = g["xyz"]
    t = oracle.tree_build(oracle.pack4(xyz), oracle.coords_root_box(xyz), 10)
    check_against_reference(g, t["members"], t["leaf_offsets"], t, lambda idx: idx)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,level,max_leaf", MESH_TREES)
def test_gpu_tree_matches_reference(ctx, kind, level, max_leaf):
    torch = ctx.use_torch_stream()
    g = golden(f"tree_{kind}{level}_m{max_leaf}.npz")
    m, leaf_faces, pts = mesh_points(kind, level)
    tree = L.Tree(ctx, torch.tensor(pts, device="cuda"), oracle.mesh_root_box(m.vert_xyz), max_leaf)
    members, offsets = tree.leaf_membership()
    check_against_reference(g, members, offsets, tree.nodes(), lambda idx: leaf_faces[idx])
    tree.close()


@pytest.mark.gpu
def test_gpu_pointtree_matches_reference(ctx):
    # meshfree TreeSum root: Tree(coords)'s relative padding drops the points at negative minima
    torch = ctx.use_torch_stream()
    g = golden("pointtree_8000_m10.npz")
    xyz = g["xyz"]
    tree = L.Tree(ctx, torch.tensor(oracle.pack4(xyz), device="cuda"), oracle.coords_root_box(xyz), 10)
    members, offsets = tree.leaf_membership()
    check_against_reference(g, members, offsets, tree.nodes(), lambda idx: idx)
    assert tree.counts()["n_in_tree"] < xyz.shape[0]


@pytest.mark.gpu
@pytest.mark.parametrize("n,max_leaf,seed", [(1, 1, 0), (9, 1, 1), (50000, 7, 2), (200000, 512, 3)])
def test_gpu_tree_matches_oracle_random(ctx, n, max_leaf, seed):
    torch = ctx.use_torch_stream()
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 3))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    pts = oracle.pack4(x)
    box = oracle.mesh_root_box(x)
    ref = oracle.tree_build(pts, box, max_leaf)
    tree = L.Tree(ctx, torch.tensor(pts, device="cuda"), box, max_leaf)
    members, offsets = tree.leaf_membership()
    assert np.array_equal(members, ref["members"])
    assert np.array_equal(offsets, ref["leaf_offsets"])
    nodes = tree.nodes()
    for k in ("node_level", "node_parent", "node_count", "node_box"):
        assert np.array_equal(nodes[k], ref[k])


@pytest.mark.gpu
def test_gpu_tree_duplicate_points_hit_depth_limit(ctx):
    # more coincident points than a leaf holds can never be separated: the build reports it
    torch = ctx.use_torch_stream()
    pts = oracle.pack4(np.tile([[0.1, 0.2, 0.3]], (20, 1)))
    tree = L.Tree(ctx, torch.tensor(pts, device="cuda"), [-1, 1, -1, 1, -1, 1], 4, max_depth=6,
                  allow_overflow=True)
    assert tree.overflow
    assert tree.counts()["depth"] == 6
    with pytest.raises(L.LpmError):
        L.Tree(ctx, torch.tensor(pts, device="cuda"), [-1, 1, -1, 1, -1, 1], 4, max_depth=6)
