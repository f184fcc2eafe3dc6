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
