"""Field output in the reference's file formats against files the reference itself wrote
(MeshedParticles::writeToVtkFile and VtkWriter::writePointsAndFieldsToCSV through the unmodified reference,
tests/golden/make_golden.py): the library's files must match them byte for byte.  Host arrays need no
GPU; the device-tensor case is marked gpu."""
import numpy as np
import pytest

import lpmcxx_b200 as L
from conftest import golden
from lpmcxx_b200.fieldio import mesh_face_vertices, write_csv, write_vtk

CASES = (("icos", 2, "vtk_icos2_rh.npz", False), ("cube", 2, "vtk_cube2_gauss_lag.npz", True))


def fields_of(g, mesh, to=lambda a: a):
    vert = [("velocity", "length/time", to(g["vert_vel"].T.copy())), ("vorticity", "1/time", to(g["vert_zeta"]))]
    face = [("faceArea", "length^2", to(mesh.face_area)), ("velocity", "length/time", to(g["face_vel"].T.copy())),
            ("vorticity", "1/time", to(g["face_zeta"]))]
    return vert, face


@pytest.mark.parametrize("kind,level,name,lag", CASES)
def test_vtk_bytes_match_reference(tmp_path, kind, level, name, lag):
    g = golden(name)
    m = L.build_mesh(kind, level)
    vert, face = fields_of(g, m)
    out = tmp_path / "mesh.vtk"
    write_vtk(out, m, vert_fields=vert, face_fields=face, title="lpm vtk test",
              lagrangian=m.vert_xyz if lag else None)
    assert out.read_bytes() == g["vtk"].tobytes()


@pytest.mark.parametrize("kind,level,name,lag", CASES)
def test_csv_bytes_match_reference(tmp_path, kind, level, name, lag):
    g = golden(name)
    m = L.build_mesh(kind, level)
    out = tmp_path / "points.csv"
    write_csv(out, m.vert_xyz, [("velocity", "length/time", g["vert_vel"].T.copy()),
                                ("vorticity", "1/time", g["vert_zeta"])])
    assert out.read_bytes() == g["csv"].tobytes()


def test_face_vertices_give_the_centroids():
    for kind in ("icos", "cube"):
        m = L.build_mesh(kind, 3)
        fv = mesh_face_vertices(kind, 3)
        assert fv.shape == (m.n_faces, 3 if kind == "icos" else 4)
        assert fv.min() >= 0 and fv.max() < m.n_verts
        c = m.vert_xyz[fv].mean(axis=1)
        c /= np.linalg.norm(c, axis=1, keepdims=True)
        assert np.abs(c - m.face_xyz).max() < 1e-14


def test_state_layout_and_bad_fields(tmp_path):
    # (n, 4) particle states (the RK4 layout) write the same POINTS as (n, 3) coordinates
    m = L.build_mesh("icos", 1)
    st = np.concatenate([m.vert_xyz, np.ones((m.n_verts, 1))], axis=1)
    write_vtk(tmp_path / "a.vtk", m)
    write_vtk(tmp_path / "b.vtk", m, xyz=st)
    assert (tmp_path / "a.vtk").read_bytes() == (tmp_path / "b.vtk").read_bytes()
    with pytest.raises(ValueError):
        write_vtk(tmp_path / "c.vtk", m, vert_fields=[("x", "u", np.zeros(m.n_verts + 1))])
    with pytest.raises(L.LpmError):
        write_vtk(tmp_path / "no_such_dir" / "d.vtk", m)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,level,name,lag", CASES)
def test_vtk_from_device_tensors(tmp_path, kind, level, name, lag):
    torch = pytest.importorskip("torch")
    g = golden(name)
    m = L.build_mesh(kind, level)
    vert, face = fields_of(g, m, to=lambda a: torch.tensor(a, device="cuda"))
    xyz = torch.tensor(np.concatenate([m.vert_xyz, np.zeros((m.n_verts, 1))], axis=1), device="cuda")
    out = tmp_path / "mesh.vtk"
    write_vtk(out, m, vert_fields=vert, face_fields=face, title="lpm vtk test", xyz=xyz,
              lagrangian=xyz if lag else None)
    assert out.read_bytes() == g["vtk"].tobytes()
