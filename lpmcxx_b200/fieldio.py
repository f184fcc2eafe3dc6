"""Field output in the reference's file formats: legacy ASCII VTK POLYDATA (MeshedParticles::writeToVtkFile,
src/LpmMeshedParticles.cpp:131-153) and points-and-fields CSV (VtkWriter::writePointsAndFieldsToCSV,
src/LpmVtkFileIO.cpp:117-193), written by the library's host code from host arrays or device tensors.

    vo, fo = ctx.direct_sum_mesh(L.biot_savart_kernel(), L.LPM_PREC_F64, mesh, zeta)
    write_vtk("out.vtk", mesh, vert_fields=[("velocity", "length/time", vo)],
              face_fields=[("faceArea", "length^2", mesh.face_area), ("velocity", "length/time", fo)])

A field is (name, units, data) with data of shape (n,) or (ndim, n) (component-major, the layout of the
library's outputs), a numpy array or a CUDA tensor (read on the device by the writer).  Fields are
written in the order given; MeshedParticles writes them in name order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, lib, ptr


def mesh_face_vertices(kind: str, level: int) -> np.ndarray:
    """(n_faces, 3|4) vertex indices of every face in Faces::vertexIndices order."""
    from . import MESH_KINDS, mesh_counts

    _, nf, _ = mesh_counts(kind, level)
    out = np.empty((nf, 3 if kind == "icos" else 4), dtype=np.int64)
    check(lib().lpm_mesh_face_vertices(MESH_KINDS[kind], level, ptr(out)), "lpm_mesh_face_vertices")
    return out


def _field_descs(fields, n: int):
    keep, descs = [], []
    for name, units, data in fields:
        on_dev = hasattr(data, "is_cuda") and bool(data.is_cuda)
        if hasattr(data, "detach"):
            import torch

            data = data.detach().to(torch.float64).contiguous()
            if not on_dev:
                data = data.numpy()
        else:
            data = np.ascontiguousarray(data, dtype=np.float64)
        shape = tuple(data.shape)
        if len(shape) == 1:
            ndim = 1
        elif len(shape) == 2 and 1 <= shape[0] <= 3:
            ndim = shape[0]
        else:
            raise ValueError(f"field {name}: shape must be (n,) or (ndim, n), got {shape}")
        if shape[-1] != n:
            raise ValueError(f"field {name}: {shape[-1]} items, expected {n}")
        keep.append(data)
        descs.append(_capi.FieldDesc(name.encode(), units.encode(), ndim, 1 if on_dev else 0, ptr(data)))
    arr = (_capi.FieldDesc * max(len(descs), 1))(*descs)
    return arr, len(descs), keep


def _coords(xyz):
    """(pointer, stride, on_device, keep-alive) of an (n, 3) or (n, 4) array or tensor."""
    on_dev = hasattr(xyz, "is_cuda") and bool(xyz.is_cuda)
    if hasattr(xyz, "detach"):
        import torch

        xyz = xyz.detach().to(torch.float64).contiguous()
        if not on_dev:
            xyz = xyz.numpy()
    else:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    if xyz.ndim != 2 or xyz.shape[1] not in (3, 4):
        raise ValueError("coordinates must be (n, 3) or (n, 4)")
    return ptr(xyz), xyz.shape[1], 1 if on_dev else 0, xyz


def write_vtk(path: str, mesh, vert_fields=(), face_fields=(), title: str = "", lagrangian=None, xyz=None,
              face_verts=None) -> None:
    """Write mesh (a SphereMesh) and fields as MeshedParticles::writeToVtkFile does.  xyz replaces the
    mesh's vertex positions (e.g. the advected particles, (n, 3|4), host or device); lagrangian, if
    given, is written as the "lagrangian_coords" point data (same layout and residency as xyz)."""
    nv, nf = mesh.n_verts, mesh.n_faces
    fv = face_verts if face_verts is not None else mesh_face_vertices(mesh.kind, mesh.level)
    fv = np.ascontiguousarray(fv, dtype=np.int64)
    xp, stride, on_dev, keep_x = _coords(mesh.vert_xyz if xyz is None else xyz)
    lp = None
    if lagrangian is not None:
        lp, lstride, lon, keep_l = _coords(lagrangian)
        if lstride != stride or lon != on_dev:
            raise ValueError("lagrangian coordinates must have the layout and residency of xyz")
    va, nva, keep_v = _field_descs(vert_fields, nv)
    fa, nfa, keep_f = _field_descs(face_fields, nf)
    div = np.ascontiguousarray(mesh.face_divided, dtype=np.uint8)
    check(lib().lpm_write_vtk(str(path).encode(), title.encode(), nv, xp, stride, on_dev, lp, nf, fv.shape[1],
                              ptr(fv), ptr(div), nva, va, nfa, fa), "lpm_write_vtk")


def write_csv(path: str, xyz, fields=()) -> None:
    """Points and fields as VtkWriter::writePointsAndFieldsToCSV lays them out ("%g" values)."""
    xp, stride, on_dev, keep_x = _coords(xyz)
    n = keep_x.shape[0]
    fa, nfa, keep_f = _field_descs(fields, n)
    check(lib().lpm_write_csv(str(path).encode(), n, xp, stride, on_dev, nfa, fa), "lpm_write_csv")


__all__ = ["write_vtk", "write_csv", "mesh_face_vertices"]
