"""The allocation-free FP32 direct sum (lpm_direct_sum_f32_noalloc) through the C ABI.

It serves callers that cannot allocate device memory at call time (hosts whose own pool allocator owns
the whole device, real-time loops that may not block in the allocator): its FP32 copies live in a fixed
file-scope device array instead of
context scratch.  Its output must match the regular FP32 entry point's within the FP32 tolerance of the
other GPU tests, on two calls in a row (the second reuses the array the first one filled).  This file is
collected last so a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.workloads as W
from lpmcxx_b200 import _capi
from conftest import rel_l2

pytestmark = pytest.mark.gpu

F32_TOL = 5e-6


def test_no_alloc_matches_regular_entry_point(ctx):
    torch = ctx.use_torch_stream()
    stream = torch.cuda.current_stream().cuda_stream or None
    k = L.biot_savart_kernel()
    for level in (4, 5):  # two calls in a row with different sizes
        mesh, p, n_src = W.gaussian_vortex_mesh("icos", level)
        d = torch.tensor(p, device="cuda")
        ref = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
        ctx.direct_sum_dev(k, L.LPM_PREC_F32, d[:n_src], d, ref, n_coincident=n_src)
        out = torch.full_like(ref, float("nan"))
        rc = _capi.lib().lpm_direct_sum_f32_noalloc(C.byref(k), d.data_ptr(), n_src, d.data_ptr(), p.shape[0], n_src,
                                                    out.data_ptr(), stream)
        _capi.check(rc, "lpm_direct_sum_f32_noalloc")
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < F32_TOL


def test_no_alloc_rejects_oversized_calls(ctx):
    torch = ctx.use_torch_stream()
    k = L.biot_savart_kernel()
    n = 300_000  # 600,000 points > 524,288
    d = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    rc = _capi.lib().lpm_direct_sum_f32_noalloc(C.byref(k), d.data_ptr(), n, d.data_ptr(), n, 0, out.data_ptr(),
                                                None)
    assert rc == _capi.LPM_ERR_CAPACITY
    assert b"static scratch" in _capi.lib().lpm_last_error()


@pytest.mark.parametrize("kernel", [L.sphere_greens_kernel(), L.planar_log_kernel(), L.delta3d_kernel(0.1),
                                    L.sphere_delta_kernel(0.1)], ids=["sphere_greens", "planar_log", "delta3d",
                                                                      "sphere_delta"])
def test_no_alloc_rejects_scalar_kernels_before_any_launch(ctx, kernel):
    """The scalar kernels have no FP32 direct sum: the call fails with the regular entry point's message before
    the capacity check and before it writes the shared array or the output (which keeps its NaNs)."""
    torch = ctx.use_torch_stream()
    n = 300_000  # also over capacity: the kind check comes first
    d = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    out = torch.full((1, n), float("nan"), dtype=torch.float64, device="cuda")
    rc = _capi.lib().lpm_direct_sum_f32_noalloc(C.byref(kernel), d.data_ptr(), n, d.data_ptr(), n, 0,
                                                out.data_ptr(), None)
    assert rc == _capi.LPM_ERR_KERNEL
    assert b"FP32 direct sum takes the Biot-Savart and 3D Poisson kernels" in _capi.lib().lpm_last_error()
    torch.cuda.synchronize()
    assert torch.isnan(out).all()
