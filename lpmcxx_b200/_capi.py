"""ctypes binding of the C ABI declared in include/lpm_b200.h.

The library is loaded from the package directory (built in-tree by lpmcxx_b200/build.py).  A
missing library is an error: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# LPM_B200_LIB selects another build of the library (e.g. one compiled with different tuning constants)
LIB_PATH = Path(os.environ.get("LPM_B200_LIB", str(Path(__file__).resolve().parent / "liblpm_b200.so")))

LPM_OK = 0
LPM_ERR_ARG = 1
LPM_ERR_KERNEL = 2
LPM_ERR_OOM = 3
LPM_ERR_CUDA = 4
LPM_ERR_CAPACITY = 6
LPM_ERR_INTERNAL = 7
LPM_ERR_NO_DEVICE = 8

LPM_MESH_ICOS_TRI = 1
LPM_MESH_CUBED_SPHERE = 2
LPM_KERNEL_BIOT_SAVART_SPHERE = 1
LPM_KERNEL_POISSON_3D = 2
LPM_KERNEL_SPHERE_GREENS = 3
LPM_KERNEL_PLANAR_LOG = 4
LPM_KERNEL_DELTA_3D = 5
LPM_KERNEL_SPHERE_DELTA = 6
LPM_PREC_F64 = 0
LPM_PREC_F32 = 1


class KernelDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("radius", C.c_double), ("delta", C.c_double)]


LPM_METHOD_DIRECT = 0
LPM_METHOD_TREE = 1
LPM_ORDER_FIXED = 0
LPM_ORDER_LEARNED = 1
LPM_MLP_PARAMS = 5532
LPM_MLP_TRAINABLE = 5516


class FieldDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("units", C.c_char_p), ("ndim", C.c_int32), ("on_device", C.c_int32),
                ("data", C.c_void_p)]


class SolverDesc(C.Structure):
    _fields_ = [("method", C.c_int32), ("precision", C.c_int32), ("order", C.c_int32), ("max_per_leaf", C.c_int32),
                ("theta", C.c_double), ("order_policy", C.c_int32), ("sakajo_depth", C.c_int32),
                ("tolerance", C.c_double)]


class LpmError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


P = C.c_void_p
I64 = C.c_int64
D = C.c_double
PD = C.POINTER(C.c_double)

# (name, restype, argtypes): every entry point declared in include/lpm_b200.h
SIGNATURES = {
    "lpm_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "lpm_ctx_destroy": (C.c_int, [P]),
    "lpm_ctx_set_stream": (C.c_int, [P, P]),
    "lpm_ctx_own_stream": (P, [P]),
    "lpm_ctx_synchronize": (C.c_int, [P]),
    "lpm_last_error": (C.c_char_p, []),
    "lpm_ctx_launch_count": (C.c_int64, [P]),
    "lpm_fma_peak": (C.c_int, [P, C.c_int, C.POINTER(D)]),
    "lpm_ctx_set_profiling": (C.c_int, [P, C.c_int]),
    "lpm_ctx_set_param": (C.c_int, [P, C.c_char_p, C.c_double]),
    "lpm_ctx_get_param": (C.c_int, [P, C.c_char_p, P]),
    "lpm_ctx_profile_report": (C.c_int, [P, C.c_char_p, C.c_size_t]),
    "lpm_mesh_counts": (C.c_int, [C.c_int, C.c_int, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    "lpm_mesh_build": (C.c_int, [C.c_int, C.c_int, D, P, P, P, P]),
    "lpm_mesh_face_vertices": (C.c_int, [C.c_int, C.c_int, P]),
    "lpm_mesh_build_dev": (C.c_int, [P, C.c_int, C.c_int, D, P, P, P, P, P]),
    "lpm_mesh_particles_dev": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P]),
    "lpm_write_vtk": (C.c_int, [C.c_char_p, C.c_char_p, I64, P, C.c_int32, C.c_int32, P, I64, C.c_int32, P, P,
                                C.c_int32, C.POINTER(FieldDesc), C.c_int32, C.POINTER(FieldDesc)]),
    "lpm_write_csv": (C.c_int, [C.c_char_p, I64, P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(FieldDesc)]),
    "lpm_direct_sum_dev": (C.c_int, [P, C.POINTER(KernelDesc), C.c_int, P, I64, P, I64, I64, P]),
    "lpm_direct_sum_f32_noalloc": (C.c_int, [C.POINTER(KernelDesc), P, I64, P, I64, I64, P, P]),
    "lpm_direct_sum_mesh": (C.c_int, [P, C.POINTER(KernelDesc), C.c_int, I64, P, P, P, I64, P, P, P, P, P, P,
                                      I64, I64, I64, I64, P, P, P, P, P, P]),
    "lpm_direct_sum_meshfree": (C.c_int, [P, C.POINTER(KernelDesc), C.c_int, I64, P, P, P, P, P, I64, I64, P]),
    "lpm_tree_build": (C.c_int, [P, P, I64, P, C.c_int, C.c_int, C.POINTER(P)]),
    "lpm_tree_build_host": (C.c_int, [P, P, I64, P, C.c_int, C.c_int, C.POINTER(P)]),
    "lpm_tree_destroy": (C.c_int, [P]),
    "lpm_tree_counts": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(C.c_int)]),
    "lpm_tree_leaf_membership": (C.c_int, [P, P, P]),
    "lpm_tree_nodes": (C.c_int, [P, P, P, P, P]),
    "lpm_treesum_create": (C.c_int, [P, C.POINTER(KernelDesc), C.POINTER(SolverDesc), I64, I64, C.POINTER(P)]),
    "lpm_treesum_destroy": (C.c_int, [P]),
    "lpm_treesum_eval_dev": (C.c_int, [P, P, P, P]),
    "lpm_treesum_stats": (C.c_int, [P, P]),
    "lpm_treesum_set_param": (C.c_int, [P, C.c_char_p, C.c_double]),
    "lpm_treesum_get_param": (C.c_int, [P, C.c_char_p, P]),
    "lpm_treesum_source_tree": (C.c_int, [P, C.POINTER(P)]),
    "lpm_treesum_set_mlp": (C.c_int, [P, P]),
    "lpm_treesum_sample_labels": (C.c_int, [P, P, P, C.c_int64, C.c_int64, P, P, P, P]),
    "lpm_mlp_train": (C.c_int, [P, P, P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, P, P]),
    "lpm_mlp_grad": (C.c_int, [P, P, P, P, C.c_int64, P, P]),
    "lpm_mlp_predict": (C.c_int, [P, P, P, C.c_int64, P]),
    "lpm_tree_sum_mesh": (C.c_int, [P, C.POINTER(KernelDesc), C.POINTER(SolverDesc), I64, P, P, P, I64, P, P, P, P, P,
                                    P, I64, I64, I64, I64, P, P, P, P, P, P, C.POINTER(I64)]),
    "lpm_rk4_create": (C.c_int, [P, C.POINTER(KernelDesc), C.POINTER(SolverDesc), I64, I64, C.POINTER(P)]),
    "lpm_rk4_destroy": (C.c_int, [P]),
    "lpm_rk4_set_state_dev": (C.c_int, [P, P]),
    "lpm_rk4_get_state_dev": (C.c_int, [P, P]),
    "lpm_rk4_set_state": (C.c_int, [P, P]),
    "lpm_rk4_get_state": (C.c_int, [P, P]),
    "lpm_rk4_step": (C.c_int, [P, D, C.c_int, C.c_int]),
    "lpm_rk4_velocity_dev": (C.c_int, [P, P]),
    "lpm_rk4_tree_stats": (C.c_int, [P, P]),
    "lpm_rk4_set_param": (C.c_int, [P, C.c_char_p, C.c_double]),
    "lpm_rk4_get_param": (C.c_int, [P, C.c_char_p, P]),
    "lpm_rk4_source_tree": (C.c_int, [P, C.POINTER(P)]),
    "lpm_rk4_set_mlp": (C.c_int, [P, P]),
    "lpm_ensemble_create": (C.c_int, [P, P, P, C.c_int, P, P, C.c_int, P]),
    "lpm_ensemble_create_each": (C.c_int, [P, P, P, C.c_int, P, P, C.c_int, P]),
    "lpm_ensemble_destroy": (C.c_int, [P]),
    "lpm_ensemble_instance": (C.c_int, [P, C.c_int, P]),
    "lpm_ensemble_lane_of": (C.c_int, [P, C.c_int, P]),
    "lpm_ensemble_set_mlp": (C.c_int, [P, P]),
    "lpm_ensemble_set_param": (C.c_int, [P, C.c_char_p, C.c_double]),
    "lpm_ensemble_get_param": (C.c_int, [P, C.c_char_p, P]),
    "lpm_ensemble_step": (C.c_int, [P, C.c_double, C.c_int, C.c_int]),
    "lpm_rk4_checkpoint_write": (C.c_int, [P, C.c_char_p, C.c_int64, C.c_double, C.c_double]),
    "lpm_rk4_checkpoint_read": (C.c_int, [P, C.c_char_p, P, P, P]),
    "lpm_ensemble_checkpoint_write": (C.c_int, [P, C.c_char_p, C.c_int64, C.c_double, C.c_double]),
    "lpm_ensemble_checkpoint_read": (C.c_int, [P, C.c_char_p, P, P, P]),
    "lpm_debug_fail_allocations": (C.c_int, [C.c_int64]),
}

_lib = None


def lib() -> C.CDLL:
    """Load liblpm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lpmcxx_b200.build`")
        h = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(code: int, where: str) -> None:
    if code != LPM_OK:
        msg = lib().lpm_last_error()
        raise LpmError(code, where, msg.decode() if msg else "")


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
