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


def check_against_digest(g, members, offsets, nodes, to_ref_index):
    """Large trees: the fixture holds per-leaf digests of the member lists (oracle.leaf_hashes)."""
    assert np.array_equal(offsets, g["leaf_offsets"])
    assert np.array_equal(oracle.leaf_hashes(to_ref_index(members), offsets), g["leaf_hash"])
    assert np.array_equal(nodes["node_level"], g["node_level"])
    assert np.array_equal(nodes["node_parent"], g["node_parent"])
    assert np.array_equal(nodes["node_count"], g["node_ncoords"])
    assert np.array_equal(nodes["node_box"], g["node_box"])


def test_oracle_tree_icos8_m512_matches_reference():
    # the treecode's full-size configuration: 1,310,720 leaf faces, 512 per leaf
    g = golden("tree_icos8_m512.npz")
    m, leaf_faces, pts = mesh_points("icos", 8)
    box = oracle.mesh_root_box(m.vert_xyz)
    assert box[1] == g["maxr"][0] + 1e-5
    t = oracle.tree_build(pts, box, 512)
    assert t["flags"] == 0
    check_against_digest(g, t["members"], t["leaf_offsets"], t, lambda idx: leaf_faces[idx])


@pytest.mark.gpu
def test_gpu_treecode_source_tree_is_reference_tree_icos8(ctx):
    """The octree the treecode builds inside its RK4 step (root Box3d(maxR) of the vertex particles,
    computed on the device) has the reference TreeSum's leaves at icos L8 / 512 per leaf."""
    import lpmcxx_b200.workloads as W

    torch = ctx.use_torch_stream()
    g = golden("tree_icos8_m512.npz")
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", 8)
    leaf_faces = np.nonzero(mesh.leaf)[0]
    assert n_src == leaf_faces.size
    rk = L.RK4(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 8, 512, 0.7), n_src, p.shape[0])
    assert rk.get_param("root_first") == n_src
    rk.set_state(torch.tensor(p, device="cuda"))
    u = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
    rk.velocity(u)
    tree = rk.source_tree()
    members, offsets = tree.leaf_membership()
    assert tree.counts()["n_in_tree"] == n_src
    check_against_digest(g, members, offsets, tree.nodes(), lambda idx: leaf_faces[idx])
    tree.close()
    rk.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,level,max_leaf", MESH_TREES)
def test_gpu_treesum_source_tree_matches_reference(ctx, kind, level, max_leaf):
    """A TreeSum evaluation over the mesh (targets: leaf faces, then vertices) with the root taken from
    the vertex targets builds the reference's tree."""
    torch = ctx.use_torch_stream()
    g = golden(f"tree_{kind}{level}_m{max_leaf}.npz")
    m, leaf_faces, pts = mesh_points(kind, level)
    tgt = np.concatenate([pts, oracle.pack4(m.vert_xyz)])
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 6, max_leaf, 0.5), pts.shape[0],
                   tgt.shape[0])
    ts.set_param("root_first", pts.shape[0])
    out = torch.empty((3, tgt.shape[0]), dtype=torch.float64, device="cuda")
    ts.eval(torch.tensor(pts, device="cuda"), torch.tensor(tgt, device="cuda"), out)
    tree = ts.source_tree()
    members, offsets = tree.leaf_membership()
    check_against_reference(g, members, offsets, tree.nodes(), lambda idx: leaf_faces[idx])
    tree.close()
    ts.close()


SAKAJO = [("icos", 4, 3), ("cube", 4, 2)]


@pytest.mark.parametrize("kind,level,depth", SAKAJO)
def test_oracle_sakajo_tree_matches_reference(kind, level, depth):
    g = golden(f"sakajo_{kind}{level}_d{depth}.npz")
    t = oracle.sakajo_tree(g["xyz"], depth)
    assert np.array_equal(t["node_level"], g["node_level"])
    assert np.array_equal(t["node_parent"], g["node_parent"])
    assert np.array_equal(t["node_count"], g["node_ncoords"])
    assert np.array_equal(t["node_box"], g["node_box"])
    assert np.array_equal(t["leaf_offsets"], g["leaf_offsets"])
    assert np.array_equal(t["members"], g["leaf_members"])


@pytest.mark.gpu
@pytest.mark.parametrize("kind,level,depth", SAKAJO)
def test_gpu_sakajo_tree_matches_reference(ctx, kind, level, depth):
    """The treecode's source tree in Sakajo mode (sakajo_depth = L) is the reference SakajoTree's: every
    non-empty node (depth-first: level, parent, point count, box) and the full-depth leaves' members."""
    torch = ctx.use_torch_stream()
    g = golden(f"sakajo_{kind}{level}_d{depth}.npz")
    pts = oracle.pack4(g["xyz"], np.ones(g["xyz"].shape[0]))
    d = torch.tensor(pts, device="cuda")
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 6, 1, 0.5, sakajo_depth=depth),
                   pts.shape[0], pts.shape[0])
    assert ts.get_param("sakajo_depth") == depth
    out = torch.empty((3, pts.shape[0]), dtype=torch.float64, device="cuda")
    ts.eval(d, d, out)
    tree = ts.source_tree()
    nodes = tree.nodes()
    assert np.array_equal(nodes["node_level"], g["node_level"])
    assert np.array_equal(nodes["node_parent"], g["node_parent"])
    assert np.array_equal(nodes["node_count"], g["node_ncoords"])
    assert np.array_equal(nodes["node_box"], g["node_box"])
    members, offsets = tree.leaf_membership()
    assert np.array_equal(offsets, g["leaf_offsets"])
    assert np.array_equal(members, g["leaf_members"])
    tree.close()
    ts.close()
