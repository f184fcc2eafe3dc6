"""lpmcxx_b200 -- B200-native (sm_100a) DirectSum / TreeSum hot path of lpmCxx.

Python-side convenience layer over the C ABI in include/lpm_b200.h (liblpm_b200.so).  The
reference-facing C++ drop-in classes live in lpmcxx_b200/host/; this module is what tests and
bench.py use.  Every compute call goes to the CUDA library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import (LPM_KERNEL_BIOT_SAVART_SPHERE, LPM_KERNEL_DELTA_3D, LPM_KERNEL_PLANAR_LOG,
                    LPM_KERNEL_POISSON_3D, LPM_KERNEL_SPHERE_DELTA, LPM_KERNEL_SPHERE_GREENS, LPM_MESH_CUBED_SPHERE,
                    LPM_MESH_ICOS_TRI, LPM_PREC_F32, LPM_PREC_F64, KernelDesc, LpmError, check, lib, ptr)

__all__ = [
    "Context", "SphereMesh", "build_mesh", "mesh_counts", "biot_savart_kernel", "poisson_kernel",
    "sphere_greens_kernel", "planar_log_kernel", "delta3d_kernel", "sphere_delta_kernel", "LpmError",
    "LPM_MESH_ICOS_TRI", "LPM_MESH_CUBED_SPHERE", "LPM_PREC_F64", "LPM_PREC_F32",
]

MESH_KINDS = {"icos": LPM_MESH_ICOS_TRI, "cube": LPM_MESH_CUBED_SPHERE}


def biot_savart_kernel(radius: float = 1.0, delta: float = 0.0) -> KernelDesc:
    """BiotSavartSphere(delta, sphRadius) (src/LpmVectorKernel.h:19-39)."""
    return KernelDesc(LPM_KERNEL_BIOT_SAVART_SPHERE, 0, float(radius), float(delta))


def poisson_kernel() -> KernelDesc:
    """1/(4 pi |x - y|), zero at x == y."""
    return KernelDesc(LPM_KERNEL_POISSON_3D, 0, 1.0, 0.0)


def sphere_greens_kernel(radius: float = 1.0) -> KernelDesc:
    """SphereGreensFn(r): -log(r^2 - x.y) / (4 pi r) (src/LpmScalarKernel.h:31-45); singular."""
    return KernelDesc(LPM_KERNEL_SPHERE_GREENS, 0, float(radius), 0.0)


def planar_log_kernel() -> KernelDesc:
    """PlanarGreensFnFreeBoundaries: log(|x - y|^2) / (4 pi) (src/LpmScalarKernel.h:19-29); singular."""
    return KernelDesc(LPM_KERNEL_PLANAR_LOG, 0, 1.0, 0.0)


def delta3d_kernel(eps: float) -> KernelDesc:
    """SecondOrderDelta3d(eps): 3 exp(-(|x - y|/eps)^3) / (4 pi eps^3) (src/LpmScalarKernel.h:47-62)."""
    return KernelDesc(LPM_KERNEL_DELTA_3D, 0, 1.0, float(eps))


def sphere_delta_kernel(eps: float) -> KernelDesc:
    """SphereDelta(eps) (src/LpmScalarKernel.h:64-78)."""
    return KernelDesc(LPM_KERNEL_SPHERE_DELTA, 0, 1.0, float(eps))


@dataclass
class SphereMesh:
    """Arrays of a refined sphere mesh in the reference's index order."""
    kind: str
    level: int
    vert_xyz: np.ndarray      # (n_verts, 3)
    face_xyz: np.ndarray      # (n_faces, 3) centroids
    face_area: np.ndarray     # (n_faces,) zero for divided faces
    face_divided: np.ndarray  # (n_faces,) uint8

    @property
    def leaf(self) -> np.ndarray:
        return self.face_divided == 0

    @property
    def n_verts(self) -> int:
        return self.vert_xyz.shape[0]

    @property
    def n_faces(self) -> int:
        return self.face_xyz.shape[0]


def mesh_counts(kind: str, level: int) -> tuple[int, int, int]:
    nv, nf, nl = C.c_int64(), C.c_int64(), C.c_int64()
    check(lib().lpm_mesh_counts(MESH_KINDS[kind], level, C.byref(nv), C.byref(nf), C.byref(nl)), "lpm_mesh_counts")
    return nv.value, nf.value, nl.value


def build_mesh(kind: str, level: int, radius: float = 1.0) -> SphereMesh:
    """PolyMesh2d(seed, level) (src/LpmPolyMesh2d.cpp:20-93), generated by the library's host code."""
    nv, nf, _ = mesh_counts(kind, level)
    v = np.empty((nv, 3)); f = np.empty((nf, 3)); a = np.empty(nf); d = np.empty(nf, dtype=np.uint8)
    check(lib().lpm_mesh_build(MESH_KINDS[kind], level, radius, ptr(v), ptr(f), ptr(a), ptr(d)), "lpm_mesh_build")
    return SphereMesh(kind, level, v, f, a, d)


def build_mesh_dev(ctx, kind: str, level: int, radius: float = 1.0, face_verts: bool = False) -> dict:
    """The mesh of build_mesh refined on the GPU (lpm_mesh_build_dev): CUDA tensors vert_xyz, face_xyz,
    face_area, face_divided (and face_verts)."""
    import torch

    k = _capi.LPM_MESH_ICOS_TRI if kind == "icos" else _capi.LPM_MESH_CUBED_SPHERE
    nv, nf, _ = mesh_counts(kind, level)
    ns = 3 if kind == "icos" else 4
    out = {"vert_xyz": torch.empty((nv, 3), dtype=torch.float64, device="cuda"),
           "face_xyz": torch.empty((nf, 3), dtype=torch.float64, device="cuda"),
           "face_area": torch.empty(nf, dtype=torch.float64, device="cuda"),
           "face_divided": torch.empty(nf, dtype=torch.uint8, device="cuda")}
    if face_verts:
        out["face_verts"] = torch.empty((nf, ns), dtype=torch.int64, device="cuda")
    check(lib().lpm_mesh_build_dev(ctx.h, k, level, radius, ptr(out["vert_xyz"]), ptr(out["face_xyz"]),
                                   ptr(out["face_area"]), ptr(out["face_divided"]), ptr(out.get("face_verts"))),
          "lpm_mesh_build_dev")
    return out


def mesh_particles_dev(ctx, kind: str, level: int, mesh: dict, face_src):
    """RK4 particles of a device mesh: (n_leaves + n_verts, 4) CUDA tensor, leaf centroids with face_src x
    area, then the vertices with strength 0."""
    import torch

    k = _capi.LPM_MESH_ICOS_TRI if kind == "icos" else _capi.LPM_MESH_CUBED_SPHERE
    nv, nf, nl = mesh_counts(kind, level)
    state = torch.empty((nl + nv, 4), dtype=torch.float64, device="cuda")
    check(lib().lpm_mesh_particles_dev(ctx.h, k, level, ptr(mesh["vert_xyz"]), ptr(mesh["face_xyz"]),
                                       ptr(mesh["face_area"]), ptr(face_src), ptr(state)), "lpm_mesh_particles_dev")
    return state


class Context:
    """One device + stream + scratch buffers (lpm_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().lpm_ctx_create(device, C.byref(h)), "lpm_ctx_create")
        self.h = h
        self.device = device

    def close(self) -> None:
        if self.h:
            lib().lpm_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None) -> None:
        """Run on this cudaStream_t handle (0/None = the legacy default stream, as torch's default)."""
        check(lib().lpm_ctx_set_stream(self.h, stream_handle or None), "lpm_ctx_set_stream")

    def use_torch_stream(self):
        """Run on torch's current stream; returns the torch module."""
        import torch

        self.set_stream(torch.cuda.current_stream().cuda_stream)
        return torch

    def use_own_stream(self) -> None:
        check(lib().lpm_ctx_set_stream(self.h, lib().lpm_ctx_own_stream(self.h)), "lpm_ctx_set_stream")

    def synchronize(self) -> None:
        check(lib().lpm_ctx_synchronize(self.h), "lpm_ctx_synchronize")

    @property
    def launch_count(self) -> int:
        return lib().lpm_ctx_launch_count(self.h)

    def set_param(self, name: str, value: float) -> None:
        """Context parameter (lpm_ctx_set_param): "direct_targets" (2, 4 or 8)."""
        check(lib().lpm_ctx_set_param(self.h, name.encode(), float(value)), "lpm_ctx_set_param")

    def get_param(self, name: str) -> float:
        v = C.c_double()
        check(lib().lpm_ctx_get_param(self.h, name.encode(), C.byref(v)), "lpm_ctx_get_param")
        return v.value

    def set_profiling(self, on: bool) -> None:
        check(lib().lpm_ctx_set_profiling(self.h, 1 if on else 0), "lpm_ctx_set_profiling")

    def profile_report(self) -> dict:
        """Per-kernel {name: {"ms": total, "launches": n}} since profiling was switched on (then cleared)."""
        import json

        buf = C.create_string_buffer(1 << 16)
        check(lib().lpm_ctx_profile_report(self.h, buf, len(buf)), "lpm_ctx_profile_report")
        return json.loads(buf.value.decode())

    def fma_peak_tflops(self, precision: int) -> float:
        t = C.c_double()
        check(lib().lpm_fma_peak(self.h, precision, C.byref(t)), "lpm_fma_peak")
        return t.value

    # ---- direct sums
    def direct_sum_dev(self, kernel: KernelDesc, precision: int, src, tgt, out, n_coincident: int = 0) -> None:
        """Device tensors: src (n_src,4) f64, tgt (n_tgt,4) f64, out ({3|1}, n_tgt) f64.  Targets
        0..n_coincident-1 sit on sources 0..n_coincident-1."""
        check(lib().lpm_direct_sum_dev(self.h, C.byref(kernel), precision, ptr(src), src.shape[0], ptr(tgt),
                                       tgt.shape[0], n_coincident, ptr(out)), "lpm_direct_sum_dev")

    def direct_sum_mesh(self, kernel: KernelDesc, precision: int, mesh: SphereMesh, face_src: np.ndarray,
                        vert_range=None, face_range=None, vert_out=None, face_out=None):
        """DirectSum::meshSolve on host arrays; returns (vert_out (c,nv), face_out (c,nf)) with c = 3 for
        the Biot-Savart kernel and 1 for the scalar kernels."""
        nv, nf = mesh.n_verts, mesh.n_faces
        comps = 3 if kernel.kind == LPM_KERNEL_BIOT_SAVART_SPHERE else 1
        vb, ve = vert_range if vert_range is not None else (0, nv - 1)
        fb, fe = face_range if face_range is not None else (0, nf - 1)
        vx, vy, vz = (np.ascontiguousarray(mesh.vert_xyz[:, c]) for c in range(3))
        fx, fy, fz = (np.ascontiguousarray(mesh.face_xyz[:, c]) for c in range(3))
        vo = np.zeros((comps, nv)) if vert_out is None else vert_out
        fo = np.zeros((comps, nf)) if face_out is None else face_out
        src = np.ascontiguousarray(face_src, dtype=np.float64)
        rest = lambda a, c: ptr(a[c]) if comps == 3 else None  # noqa: E731
        check(lib().lpm_direct_sum_mesh(self.h, C.byref(kernel), precision, nv, ptr(vx), ptr(vy), ptr(vz), nf,
                                        ptr(fx), ptr(fy), ptr(fz), ptr(mesh.face_area), ptr(mesh.face_divided),
                                        ptr(src), vb, ve, fb, fe, ptr(vo[0]), rest(vo, 1), rest(vo, 2),
                                        ptr(fo[0]), rest(fo, 1), rest(fo, 2)), "lpm_direct_sum_mesh")
        return vo, fo

    def direct_sum_meshfree(self, kernel: KernelDesc, precision: int, xyz: np.ndarray, src: np.ndarray,
                            weights: np.ndarray | None = None, rng=None, out=None) -> np.ndarray:
        n = xyz.shape[0]
        b, e = rng if rng is not None else (0, n - 1)
        x, y, z = (np.ascontiguousarray(xyz[:, c]) for c in range(3))
        o = np.zeros(n) if out is None else out
        s = np.ascontiguousarray(src, dtype=np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        check(lib().lpm_direct_sum_meshfree(self.h, C.byref(kernel), precision, n, ptr(x), ptr(y), ptr(z), ptr(s),
                                            ptr(w), b, e, ptr(o)), "lpm_direct_sum_meshfree")
        return o


def direct_solver(precision: int = LPM_PREC_F64) -> _capi.SolverDesc:
    return _capi.SolverDesc(_capi.LPM_METHOD_DIRECT, precision, 0, 0, 0.0, 0, 0, 0.0)


def tree_solver(precision: int = LPM_PREC_F32, order: int = 8, max_per_leaf: int = 512, theta: float = 0.7,
                learned: bool = False, tolerance: float = 0.0, sakajo_depth: int = 0) -> _capi.SolverDesc:
    """Treecode descriptor.  sakajo_depth = L > 0 selects the Sakajo (2009) fixed-depth tree (3L bisections
    along z, x, y in turn) instead of the octree split at max_per_leaf."""
    return _capi.SolverDesc(_capi.LPM_METHOD_TREE, precision, order, max_per_leaf, theta,
                            _capi.LPM_ORDER_LEARNED if learned else _capi.LPM_ORDER_FIXED, sakajo_depth, tolerance)


class RK4:
    """Device-resident RK4 integrator of sphere particles (lpm_rk4).  The first n_src particles carry
    strengths (sources); state is (n, 4) float64 (x, y, z, w)."""

    def __init__(self, ctx: Context, kernel: KernelDesc, solver: _capi.SolverDesc, n_src: int, n_pts: int):
        h = C.c_void_p()
        check(lib().lpm_rk4_create(ctx.h, C.byref(kernel), C.byref(solver), n_src, n_pts, C.byref(h)),
              "lpm_rk4_create")
        self.h, self.ctx, self.n_src, self.n = h, ctx, n_src, n_pts

    def close(self) -> None:
        if self.h:
            lib().lpm_rk4_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state) -> None:
        """From a CUDA tensor (device copy, enqueued) or a host array / CPU tensor (synchronous)."""
        if getattr(state, "is_cuda", False):
            check(lib().lpm_rk4_set_state_dev(self.h, ptr(state)), "lpm_rk4_set_state_dev")
        else:
            s = state if hasattr(state, "data_ptr") else np.ascontiguousarray(state, dtype=np.float64)
            check(lib().lpm_rk4_set_state(self.h, ptr(s)), "lpm_rk4_set_state")

    def get_state(self, out=None):
        """Into a CUDA tensor (enqueued), a CPU tensor / host array (synchronous), or a new array."""
        if out is not None and getattr(out, "is_cuda", False):
            check(lib().lpm_rk4_get_state_dev(self.h, ptr(out)), "lpm_rk4_get_state_dev")
            return out
        o = np.empty((self.n, 4)) if out is None else out
        check(lib().lpm_rk4_get_state(self.h, ptr(o)), "lpm_rk4_get_state")
        return o

    def checkpoint_write(self, path, step: int = 0, t: float = 0.0, dt: float = 0.0) -> None:
        """lpm_rk4_checkpoint_write: the state, with the caller's step count, time and time step, to a file."""
        check(lib().lpm_rk4_checkpoint_write(self.h, str(path).encode(), int(step), float(t), float(dt)),
              "lpm_rk4_checkpoint_write")

    def checkpoint_read(self, path) -> tuple:
        """lpm_rk4_checkpoint_read: restores the state; returns the stored (step, t, dt)."""
        s, t, dt = C.c_int64(), C.c_double(), C.c_double()
        check(lib().lpm_rk4_checkpoint_read(self.h, str(path).encode(), C.byref(s), C.byref(t), C.byref(dt)),
              "lpm_rk4_checkpoint_read")
        return s.value, t.value, dt.value

    def step(self, dt: float, nsteps: int = 1, use_graph: bool = False) -> None:
        check(lib().lpm_rk4_step(self.h, dt, nsteps, 1 if use_graph else 0), "lpm_rk4_step")

    def velocity(self, out) -> None:
        """Velocity (3, n) at the current state into a device tensor."""
        check(lib().lpm_rk4_velocity_dev(self.h, ptr(out)), "lpm_rk4_velocity_dev")

    def tree_stats(self) -> dict:
        o = np.zeros(10, np.int64)
        check(lib().lpm_rk4_tree_stats(self.h, ptr(o)), "lpm_rk4_tree_stats")
        return dict(zip(TreeSum.STAT_KEYS, (int(v) for v in o)))

    def set_param(self, name: str, value: float) -> None:
        check(lib().lpm_rk4_set_param(self.h, name.encode(), float(value)), "lpm_rk4_set_param")

    def get_param(self, name: str) -> float:
        v = C.c_double()
        check(lib().lpm_rk4_get_param(self.h, name.encode(), C.byref(v)), "lpm_rk4_get_param")
        return v.value

    def source_tree(self) -> "Tree":
        """The treecode's source octree of the last velocity evaluation (a read-only view)."""
        h = C.c_void_p()
        check(lib().lpm_rk4_source_tree(self.h, C.byref(h)), "lpm_rk4_source_tree")
        return Tree._view(h)

    def set_mlp(self, params) -> None:
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        check(lib().lpm_rk4_set_mlp(self.h, ptr(p)), "lpm_rk4_set_mlp")


class _RK4View(RK4):
    """An ensemble instance: an RK4 whose lifetime the ensemble owns."""

    def __init__(self, ctx, h, n_src, n_pts):
        self.h, self.ctx, self.n_src, self.n = h, ctx, n_src, n_pts

    def close(self) -> None:
        self.h = None


class Ensemble:
    """lpm_ensemble: independent RK4 problems of uneven sizes, advanced together by one CUDA graph per
    step spread over `lanes` streams, the far and near fields of all instances in fused persistent launches
    (set_param("fused", 0): per lane).  `instance(i)` gives an RK4 handle for states."""

    def __init__(self, ctx: Context, kernel: KernelDesc, solver, n_src, n_pts, lanes: int = 8):
        """solver: one SolverDesc for every instance, or a sequence of them (one per instance)."""
        n_src = np.ascontiguousarray(n_src, dtype=np.int64)
        n_pts = np.ascontiguousarray(n_pts, dtype=np.int64)
        h = C.c_void_p()
        if isinstance(solver, _capi.SolverDesc):
            check(lib().lpm_ensemble_create(ctx.h, C.byref(kernel), C.byref(solver), len(n_src), ptr(n_src),
                                            ptr(n_pts), lanes, C.byref(h)), "lpm_ensemble_create")
        else:
            arr = (_capi.SolverDesc * len(solver))(*solver)
            check(lib().lpm_ensemble_create_each(ctx.h, C.byref(kernel), arr, len(n_src), ptr(n_src), ptr(n_pts),
                                                 lanes, C.byref(h)), "lpm_ensemble_create_each")
        self.h, self.ctx = h, ctx
        self.n_src, self.n_pts = n_src, n_pts

    def close(self) -> None:
        if self.h:
            lib().lpm_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.n_src)

    def instance(self, i: int) -> RK4:
        r = C.c_void_p()
        check(lib().lpm_ensemble_instance(self.h, i, C.byref(r)), "lpm_ensemble_instance")
        return _RK4View(self.ctx, r, int(self.n_src[i]), int(self.n_pts[i]))

    def lane_of(self, i: int) -> int:
        v = C.c_int()
        check(lib().lpm_ensemble_lane_of(self.h, i, C.byref(v)), "lpm_ensemble_lane_of")
        return v.value

    def set_mlp(self, params) -> None:
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        check(lib().lpm_ensemble_set_mlp(self.h, ptr(p)), "lpm_ensemble_set_mlp")

    def set_param(self, name: str, value: float) -> None:
        """lpm_ensemble_set_param: one run-time treecode parameter for every instance, or the ensemble's own
        "fused" (1: far and near fields of all instances in fused persistent launches; 0: per lane)."""
        check(lib().lpm_ensemble_set_param(self.h, name.encode(), float(value)), "lpm_ensemble_set_param")

    def get_param(self, name: str) -> float:
        """lpm_ensemble_get_param ("fused")."""
        v = C.c_double()
        check(lib().lpm_ensemble_get_param(self.h, name.encode(), C.byref(v)), "lpm_ensemble_get_param")
        return v.value

    def step(self, dt: float, nsteps: int = 1, use_graph: bool = True) -> None:
        check(lib().lpm_ensemble_step(self.h, dt, nsteps, 1 if use_graph else 0), "lpm_ensemble_step")

    def checkpoint_write(self, path, step: int = 0, t: float = 0.0, dt: float = 0.0) -> None:
        """lpm_ensemble_checkpoint_write: every instance's state in one file."""
        check(lib().lpm_ensemble_checkpoint_write(self.h, str(path).encode(), int(step), float(t), float(dt)),
              "lpm_ensemble_checkpoint_write")

    def checkpoint_read(self, path) -> tuple:
        """lpm_ensemble_checkpoint_read: restores every instance's state; returns the stored (step, t, dt)."""
        s, t, dt = C.c_int64(), C.c_double(), C.c_double()
        check(lib().lpm_ensemble_checkpoint_read(self.h, str(path).encode(), C.byref(s), C.byref(t), C.byref(dt)),
              "lpm_ensemble_checkpoint_read")
        return s.value, t.value, dt.value


class Tree:
    """Device octree (lpm_tree) over a (n, 4) float64 CUDA tensor of points."""

    def __init__(self, ctx: Context, pts, box, max_per_leaf: int, max_depth: int = 0, allow_overflow: bool = False):
        h = C.c_void_p()
        b = np.ascontiguousarray(box, dtype=np.float64)
        rc = lib().lpm_tree_build(ctx.h, ptr(pts), pts.shape[0], ptr(b), max_per_leaf, max_depth, C.byref(h))
        self.h = h
        if rc != _capi.LPM_OK and not (allow_overflow and rc == _capi.LPM_ERR_CAPACITY and h):
            if h:
                lib().lpm_tree_destroy(h)
                self.h = None
            check(rc, "lpm_tree_build")
        self.overflow = rc == _capi.LPM_ERR_CAPACITY

    @classmethod
    def _view(cls, h) -> "Tree":
        t = cls.__new__(cls)
        t.h, t.overflow = h, False
        return t

    def close(self):
        if self.h:
            lib().lpm_tree_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def counts(self) -> dict:
        a, b, c, d = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
        check(lib().lpm_tree_counts(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), "lpm_tree_counts")
        return {"n_in_tree": a.value, "n_nodes": b.value, "n_leaves": c.value, "depth": d.value}

    def leaf_membership(self):
        c = self.counts()
        members = np.zeros(max(c["n_in_tree"], 1), np.int64)
        offs = np.zeros(c["n_leaves"] + 1, np.int64)
        check(lib().lpm_tree_leaf_membership(self.h, ptr(members), ptr(offs)), "lpm_tree_leaf_membership")
        return members[:c["n_in_tree"]], offs

    def nodes(self) -> dict:
        m = self.counts()["n_nodes"]
        lv, par, cnt = (np.zeros(m, np.int64) for _ in range(3))
        box = np.zeros((m, 6))
        check(lib().lpm_tree_nodes(self.h, ptr(lv), ptr(par), ptr(cnt), ptr(box)), "lpm_tree_nodes")
        return {"node_level": lv, "node_parent": par, "node_count": cnt, "node_box": box}


class TreeSum:
    """Device-resident treecode solver (lpm_treesum) for fixed source / target counts."""

    STAT_KEYS = ("nodes", "leaves", "depth", "far_pairs", "near_runs", "batches", "overflow", "far_evals",
                 "near_pairs", "far_terms")

    def __init__(self, ctx: Context, kernel: KernelDesc, solver: _capi.SolverDesc, n_src: int, n_tgt: int):
        h = C.c_void_p()
        check(lib().lpm_treesum_create(ctx.h, C.byref(kernel), C.byref(solver), n_src, n_tgt, C.byref(h)),
              "lpm_treesum_create")
        self.h, self.ctx, self.n_src, self.n_tgt = h, ctx, n_src, n_tgt

    def close(self):
        if self.h:
            lib().lpm_treesum_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def eval(self, src, tgt, out) -> None:
        """src (n_src,4), tgt (n_tgt,4), out (3,n_tgt): float64 CUDA tensors."""
        check(lib().lpm_treesum_eval_dev(self.h, ptr(src), ptr(tgt), ptr(out)), "lpm_treesum_eval_dev")

    def stats(self) -> dict:
        o = np.zeros(10, np.int64)
        check(lib().lpm_treesum_stats(self.h, ptr(o)), "lpm_treesum_stats")
        return dict(zip(self.STAT_KEYS, (int(v) for v in o)))

    def set_param(self, name: str, value: float) -> None:
        """Run-time parameter (lpm_treesum_set_param): "theta", "f64_from", "eps", "batch_level",
        "order_bias", "root_maxr" or "root_first"."""
        check(lib().lpm_treesum_set_param(self.h, name.encode(), float(value)), "lpm_treesum_set_param")

    def source_tree(self) -> "Tree":
        """The source octree of the last evaluation (a read-only view, valid until the next one)."""
        h = C.c_void_p()
        check(lib().lpm_treesum_source_tree(self.h, C.byref(h)), "lpm_treesum_source_tree")
        return Tree._view(h)

    def get_param(self, name: str) -> float:
        """Current run-time parameter: as set_param, plus "batch_level_max" and "order"."""
        v = C.c_double()
        check(lib().lpm_treesum_get_param(self.h, name.encode(), C.byref(v)), "lpm_treesum_get_param")
        return v.value

    def set_mlp(self, params) -> None:
        """Load the order selector (MLP_PARAMS floats), or None for the fixed-order fallback."""
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        check(lib().lpm_treesum_set_mlp(self.h, ptr(p)), "lpm_treesum_set_mlp")

    def sample_labels(self, src, tgt, stride: int, max_pairs: int, with_errors: bool = False):
        """(features (n, 8), labels (n,), errors (n, 11) or None) of accepted pairs of one evaluation:
        every stride-th, or (stride <= 0) max_pairs spread over all of them."""
        f = np.zeros((max_pairs, 8), np.float32)
        lab = np.zeros(max_pairs, np.int32)
        err = np.zeros((max_pairs, 11), np.float32) if with_errors else None
        n = C.c_int64()
        check(lib().lpm_treesum_sample_labels(self.h, ptr(src), ptr(tgt), stride, max_pairs, ptr(f), ptr(lab),
                                              ptr(err), C.byref(n)), "lpm_treesum_sample_labels")
        k = n.value
        return f[:k], lab[:k], (err[:k] if err is not None else None)


def tree_sum_mesh(ctx: Context, kernel: KernelDesc, solver: _capi.SolverDesc, mesh: SphereMesh, face_src,
                  vert_range=None, face_range=None, vert_out=None, face_out=None):
    """TreeSum::meshSolve on host arrays; returns (vert_out (3,nv), face_out (3,nf), mac_count)."""
    nv, nf = mesh.n_verts, mesh.n_faces
    vb, ve = vert_range if vert_range is not None else (0, nv - 1)
    fb, fe = face_range if face_range is not None else (0, nf - 1)
    vx, vy, vz = (np.ascontiguousarray(mesh.vert_xyz[:, c]) for c in range(3))
    fx, fy, fz = (np.ascontiguousarray(mesh.face_xyz[:, c]) for c in range(3))
    vo = np.zeros((3, nv)) if vert_out is None else vert_out
    fo = np.zeros((3, nf)) if face_out is None else face_out
    src = np.ascontiguousarray(face_src, dtype=np.float64)
    mac = C.c_int64()
    check(lib().lpm_tree_sum_mesh(ctx.h, C.byref(kernel), C.byref(solver), nv, ptr(vx), ptr(vy), ptr(vz), nf,
                                  ptr(fx), ptr(fy), ptr(fz), ptr(mesh.face_area), ptr(mesh.face_divided), ptr(src),
                                  vb, ve, fb, fe, ptr(vo[0]), ptr(vo[1]), ptr(vo[2]), ptr(fo[0]), ptr(fo[1]),
                                  ptr(fo[2]), C.byref(mac)), "lpm_tree_sum_mesh")
    return vo, fo, mac.value


# ---- order-selection MLP (training and inference run in the library's CUDA kernels)
MLP_PARAMS = _capi.LPM_MLP_PARAMS
MLP_TRAINABLE = _capi.LPM_MLP_TRAINABLE


def mlp_init(feats: np.ndarray, seed: int = 0) -> np.ndarray:
    """Initial parameters: scaled Gaussian weights, zero biases, standardisation from `feats`."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_PARAMS, np.float32)
    o = 0
    for fan_out, fan_in in ((64, 8), (64, 64), (12, 64)):
        p[o:o + fan_out * fan_in] = rng.normal(0.0, 1.0 / np.sqrt(fan_in), fan_out * fan_in)
        o += fan_out * fan_in + fan_out
    mean = feats.mean(axis=0)
    std = feats.std(axis=0)
    p[o:o + 8] = mean
    p[o + 8:o + 16] = 1.0 / np.where(std > 1e-6, std, 1.0)
    return p


def mlp_train(ctx: Context, feats, labels, params, epochs: int = 20, minibatch: int = 512, lr: float = 2e-3,
              seed: int = 0):
    """Train `params` in place on the GPU; returns the per-epoch mean loss."""
    f = np.ascontiguousarray(feats, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    if params.dtype != np.float32 or not params.flags.c_contiguous:
        raise TypeError("params must be a contiguous float32 array")
    loss = np.zeros(max(epochs, 1), np.float32)
    check(lib().lpm_mlp_train(ctx.h, ptr(f), ptr(lab), f.shape[0], epochs, minibatch, lr, seed, ptr(params),
                              ptr(loss)), "lpm_mlp_train")
    return loss[:epochs]


def mlp_grad(ctx: Context, params, feats, labels):
    """(gradient of the mean loss (MLP_TRAINABLE,), mean loss) computed by the training kernels."""
    f = np.ascontiguousarray(feats, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    g = np.zeros(MLP_TRAINABLE, np.float32)
    loss = C.c_float()
    check(lib().lpm_mlp_grad(ctx.h, ptr(np.ascontiguousarray(params, np.float32)), ptr(f), ptr(lab), f.shape[0],
                             ptr(g), C.byref(loss)), "lpm_mlp_grad")
    return g, loss.value


def mlp_predict(ctx: Context, params, feats) -> np.ndarray:
    """Classes from the BF16 inference path the treecode uses."""
    f = np.ascontiguousarray(feats, dtype=np.float32)
    cls = np.zeros(f.shape[0], np.int32)
    check(lib().lpm_mlp_predict(ctx.h, ptr(np.ascontiguousarray(params, np.float32)), ptr(f), f.shape[0], ptr(cls)),
          "lpm_mlp_predict")
    return cls
