"""Mesh generator (the step before the hot path) against the reference's PolyMesh2d.  CPU only."""
import numpy as np
import pytest

import lpmcxx_b200 as L
from conftest import golden


@pytest.mark.parametrize("kind", ["icos", "cube"])
def test_mesh_bit_exact_vs_reference(kind):
    g = golden(f"mesh_{kind}3.npz")
    m = L.build_mesh(kind, 3)
    for name in ("vert_xyz", "face_xyz", "face_area", "face_divided"):
        assert np.array_equal(getattr(m, name), g[name]), name


@pytest.mark.parametrize("kind,level", [("icos", 0), ("icos", 5), ("cube", 0), ("cube", 5)])
def test_mesh_counts_and_area(kind, level):
    # face/vertex counts of src/LpmMeshSeed.cpp:233-268; leaf areas sum to 4 pi
    m = L.build_mesh(kind, level)
    roots, vf = (20, 10) if kind == "icos" else (6, 6)
    assert m.leaf.sum() == roots * 4 ** level
    assert m.n_verts == 2 + vf * 4 ** level
    assert m.n_faces == sum(roots * 4 ** k for k in range(level + 1))
    assert abs(m.face_area[m.leaf].sum() - 4 * np.pi) < 1e-11
    assert np.all(m.face_area[~m.leaf] == 0)
    assert np.allclose(np.linalg.norm(m.vert_xyz, axis=1), 1.0, atol=1e-15)


def test_mesh_bad_args():
    with pytest.raises(L.LpmError):
        L.mesh_counts("icos", -1)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,level", [("icos", 0), ("icos", 1), ("icos", 4), ("icos", 6), ("cube", 0), ("cube", 1),
                                        ("cube", 4), ("cube", 6)])
def test_gpu_mesh_refinement_matches_host_generator(ctx, kind, level):
    """The device refinement (lpm_mesh_build_dev) gives the host generator's mesh: vertex coordinates,
    centroids, divided mask and connectivity bit for bit; areas within 1e-13 relative (CUDA's atan2 / tan
    against the host's libm, amplified by L'Huilier's formula: 11 ulp measured at icos L4), summing to 4 pi."""
    ctx.use_torch_stream()
    d = L.build_mesh_dev(ctx, kind, level, face_verts=True)
    m = L.build_mesh(kind, level)
    assert np.array_equal(d["vert_xyz"].cpu().numpy(), m.vert_xyz)
    assert np.array_equal(d["face_xyz"].cpu().numpy(), m.face_xyz)
    assert np.array_equal(d["face_divided"].cpu().numpy(), m.face_divided)
    k = L.LPM_MESH_ICOS_TRI if kind == "icos" else L.LPM_MESH_CUBED_SPHERE
    fv = np.zeros((m.n_faces, 3 if kind == "icos" else 4), np.int64)
    L.check(L.lib().lpm_mesh_face_vertices(k, level, fv.ctypes.data), "lpm_mesh_face_vertices")
    assert np.array_equal(d["face_verts"].cpu().numpy(), fv)
    area = d["face_area"].cpu().numpy()
    assert np.all(area[~m.leaf] == 0.0)
    assert (np.abs(area[m.leaf] - m.face_area[m.leaf]) / m.face_area[m.leaf]).max() < 1e-13
    assert abs(area.sum() - 4 * np.pi) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["icos", "cube"])
def test_gpu_mesh_refinement_matches_reference(ctx, kind):
    """Against the reference's own PolyMesh2d (golden fixture, level 3)."""
    ctx.use_torch_stream()
    g = golden(f"mesh_{kind}3.npz")
    d = L.build_mesh_dev(ctx, kind, 3)
    for name in ("vert_xyz", "face_xyz", "face_divided"):
        assert np.array_equal(d[name].cpu().numpy(), g[name]), name
    leaf = g["face_divided"] == 0
    a = d["face_area"].cpu().numpy()[leaf]
    assert (np.abs(a - g["face_area"][leaf]) / g["face_area"][leaf]).max() < 1e-13


@pytest.mark.gpu
def test_gpu_mesh_particles_match_workload(ctx):
    """lpm_mesh_particles_dev packs the RK4 state of workloads.particles from device arrays."""
    import lpmcxx_b200.workloads as W

    torch = ctx.use_torch_stream()
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", 5)
    zeta = np.zeros(mesh.n_faces)
    zeta[mesh.leaf] = p[:n_src, 3] / mesh.face_area[mesh.leaf]
    d = L.build_mesh_dev(ctx, "icos", 5)
    state = L.mesh_particles_dev(ctx, "icos", 5, d, torch.tensor(zeta, device="cuda")).cpu().numpy()
    assert np.array_equal(state[:, :3], p[:, :3])
    assert np.allclose(state[:, 3], p[:, 3], rtol=1e-14, atol=0.0)
