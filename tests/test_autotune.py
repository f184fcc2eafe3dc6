"""Autotuner: the chosen setting meets the tolerance against the FP64 direct sum and is the fastest
candidate that does."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.learned  # noqa: F401  (L.learned: the shipped selector weights)
import lpmcxx_b200.workloads as W
from lpmcxx_b200.autotune import apply_tuned, autotune, default_grid, tuned_solver


def test_default_grids():
    leaves, thetas, knobs = default_grid(True, L.LPM_KERNEL_BIOT_SAVART_SPHERE)
    assert all(0 < t < 1 for t in thetas) and all(k > 0 for k in knobs) and min(leaves) >= 1
    _, _, orders = default_grid(False, L.LPM_KERNEL_POISSON_3D)
    assert all(isinstance(o, int) for o in orders)


def check(res, tol):
    ok = [c for c in res.tried if c.rel_err <= 0.8 * tol]
    assert res.best is not None and res.best in ok
    assert res.best.ms == min(c.ms for c in ok)


@pytest.mark.gpu
def test_autotune_learned_sphere(ctx):
    torch = ctx.use_torch_stream()
    _, p, n_src = W.gaussian_vortex_mesh("icos", 6)
    d = torch.tensor(p, device="cuda")
    tol = 1e-6
    res = autotune(ctx, L.biot_savart_kernel(), d[:n_src], d, tol, learned=True,
                   grid=((128, 256), (0.5, 0.6), (1e-8, 3e-8, 3e-7)), sample=2048, order_biases=(0, 2))
    check(res, tol)
    assert {c.bias for c in res.tried} == {0, 2}
    # the near-field tile shape is searched too: every shape was timed on the best setting, and the pick is
    # the fastest qualifying one among them
    shapes = {(c.near_targets, c.near_tile, c.near_split) for c in res.tried}
    assert shapes == {(t, s, g) for t in (2, 4) for s in (256, 512, 1024) for g in (1, 2)}
    # the tuned descriptor reproduces the accuracy on all targets
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), tuned_solver(res), n_src, p.shape[0])
    ts.set_mlp(L.learned.load()[0])
    apply_tuned(res, ts)
    assert (ts.get_param("near_targets"), ts.get_param("near_tile"), ts.get_param("near_split")) == \
        (res.best.near_targets, res.best.near_tile, res.best.near_split)
    out = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
    ts.eval(d[:n_src], d, out)
    ts.close()
    ref = torch.empty_like(out)
    ctx.direct_sum_dev(L.biot_savart_kernel(), L.LPM_PREC_F64, d[:n_src], d, ref)
    assert float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref)) < tol


@pytest.mark.gpu
def test_autotune_meets_tolerance_on_every_workload(ctx):
    """With `also`, the pick is timed on the first workload but meets the tolerance on every one: checked here
    against the FP64 direct sum on all targets of each of four ensemble members (icos L5, different vortices),
    and the reported error is the largest over the members."""
    torch = ctx.use_torch_stream()
    inst = W.ensemble_instances(levels=(5,), per_level=4)
    ds = [torch.tensor(p, device="cuda") for _, p, _ in inst]
    n_src = inst[0][2]
    tol = 1e-6
    res = autotune(ctx, L.biot_savart_kernel(), ds[0][:n_src], ds[0], tol, learned=True,
                   grid=((128, 256), (0.5, 0.6, 0.7), (3e-7, 1e-6)), sample=2048, order_biases=(2,),
                   also=[(d[:n_src], d) for d in ds[1:]])
    check(res, tol)
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), tuned_solver(res), n_src, ds[0].shape[0])
    ts.set_mlp(L.learned.load()[0])
    apply_tuned(res, ts)
    errs = []
    for d in ds:
        out = torch.empty((3, d.shape[0]), dtype=torch.float64, device="cuda")
        ts.eval(d[:n_src], d, out)
        ref = torch.empty_like(out)
        ctx.direct_sum_dev(L.biot_savart_kernel(), L.LPM_PREC_F64, d[:n_src], d, ref)
        errs.append(float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref)))
    ts.close()
    assert max(errs) < tol
    assert res.best.rel_err >= 0.5 * max(errs)  # the largest over the members, on 2048 sampled targets each


def test_autotune_rejects_larger_extra_workload():
    torch = pytest.importorskip("torch")
    small = torch.zeros((10, 4), dtype=torch.float64)
    big = torch.zeros((20, 4), dtype=torch.float64)
    with pytest.raises(ValueError, match="larger than the first"):
        autotune(None, L.biot_savart_kernel(), small, small, 1e-6, learned=False, also=[(big, big)])


@pytest.mark.gpu
def test_autotune_fixed_poisson(ctx):
    torch = ctx.use_torch_stream()
    p = W.poisson_cube(60_000)
    d = torch.tensor(p, device="cuda")
    tol = 1e-4
    res = autotune(ctx, L.poisson_kernel(), d, d, tol, learned=False, grid=((128, 256), (0.5, 0.7), (4, 6)),
                   batch_levels=(0,), sample=2048)
    check(res, tol)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["biot_savart", "poisson"])
def test_autotune_direct_tile_shape(ctx, kernel):
    """The FP32 direct sum's tile shape (2, 4 or 8 targets per thread) is tuned at run time: every shape is timed,
    the fastest is kept on the context, and the shapes' sums agree to FP32 rounding."""
    from lpmcxx_b200.autotune import autotune_direct

    torch = ctx.use_torch_stream()
    if kernel == "biot_savart":
        _, p, n_src = W.gaussian_vortex_mesh("icos", 6)
        kern, nc = L.biot_savart_kernel(), n_src
    else:
        p = W.poisson_cube(100_000)
        n_src, kern, nc = p.shape[0], L.poisson_kernel(), p.shape[0]
    d = torch.tensor(p, device="cuda")
    res = autotune_direct(ctx, kern, d[:n_src], d, n_coincident=nc)
    assert set(res["ms"]) == {2, 4, 8}
    assert res["direct_targets"] == min(res["ms"], key=res["ms"].get)
    assert ctx.get_param("direct_targets") == res["direct_targets"]
    assert res["max_rel_deviation"] < 1e-6
    ctx.set_param("direct_targets", 4)
    with pytest.raises(L.LpmError):
        ctx.set_param("direct_targets", 3)
