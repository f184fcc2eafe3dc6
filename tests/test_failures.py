"""Failure paths, injected on the host: non-finite input, a device allocation that fails (through the
library's injection point, lpm_debug_fail_allocations), and a capacity overflow inside a captured RK4 replay.
Each reports its status code, and the context stays usable afterwards.  No GPU fault is caused."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.workloads as W


@pytest.mark.gpu
def test_nan_source_is_reported(ctx):
    """A non-finite source coordinate makes the treecode's root box non-finite: the evaluation fails with
    LPM_ERR_ARG (no result is written from an incomplete tree), and the next valid evaluation succeeds."""
    torch = ctx.use_torch_stream()
    _, p, n_src = W.gaussian_vortex_mesh("icos", 4)
    bad = p.copy()
    bad[7, 0] = np.nan
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 8, 64, 0.5), n_src, p.shape[0])
    out = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
    d_bad = torch.tensor(bad, device="cuda")
    with pytest.raises(L.LpmError) as e:
        ts.eval(d_bad[:n_src], d_bad, out)
    assert e.value.code == L._capi.LPM_ERR_ARG
    d = torch.tensor(p, device="cuda")
    ts.eval(d[:n_src], d, out)
    assert torch.isfinite(out).all()
    ts.close()


@pytest.mark.gpu
def test_injected_allocation_failure_reports_oom_and_recovers(ctx):
    """Every device allocation of solver creation and of the first evaluation, failed in turn: the entry
    point that made it returns LPM_ERR_OOM (nothing leaks into later calls), and with the injection off the
    same calls succeed and agree with an undisturbed run."""
    torch = ctx.use_torch_stream()
    _, p, n_src = W.gaussian_vortex_mesh("icos", 4)
    d = torch.tensor(p, device="cuda")
    solver = L.tree_solver(L.LPM_PREC_F32, 8, 64, 0.5)
    want = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
    ts.eval(d[:n_src], d, want)
    ts.close()
    failed = 0
    lib = L.lib()
    try:
        for k in range(60):
            lib.lpm_debug_fail_allocations(k)
            try:
                ts = L.TreeSum(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
                out = torch.empty_like(want)
                ts.eval(d[:n_src], d, out)
                ts.close()
            except L.LpmError as e:
                assert e.code == L._capi.LPM_ERR_OOM, (k, e)
                failed += 1
                continue
            break  # k passed every allocation of creation and evaluation
    finally:
        lib.lpm_debug_fail_allocations(-1)
    assert failed > 5
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
    out = torch.empty_like(want)
    ts.eval(d[:n_src], d, out)
    ts.close()
    assert torch.equal(out, want)


@pytest.mark.gpu
def test_capacity_overflow_in_captured_replay_is_reported_and_recovers(ctx):
    """An RK4 step graph captured while every particle sits in one octree cell (a step of 1e-12 moves them by
    1e-7, inside the cell) holds interaction lists sized for that state; replayed on the spread-out mesh it needs
    ~8x more near-field entries than it holds: the step reports LPM_ERR_CAPACITY instead of returning wrong
    velocities.  An uncaptured step then regrows the lists, and the next graph step with the same dt captures a
    new graph (the old one holds the freed lists' addresses) whose result equals the uncaptured step's."""
    _, p, n_src = W.gaussian_vortex_mesh("icos", 5)
    tiny = p.copy()
    x0 = np.array([0.0, 0.0, 1.0])
    tiny[:, :3] = x0 + 1e-9 * (p[:, :3] - x0)
    tiny[:, :3] /= np.linalg.norm(tiny[:, :3], axis=1, keepdims=True)
    dt = 1e-12
    rk = L.RK4(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 4, 1, 0.3), n_src, p.shape[0])
    rk.set_state(tiny)
    rk.step(dt, 2, use_graph=True)  # one uncaptured step sizes the lists, then one graph replay
    rk.set_state(p)
    with pytest.raises(L.LpmError) as e:
        rk.step(dt, 1, use_graph=True)
    assert e.value.code == L._capi.LPM_ERR_CAPACITY
    rk.set_state(p)
    rk.step(dt, 1, use_graph=False)  # regrows the lists
    want = rk.get_state()
    rk.set_state(p)
    rk.step(dt, 1, use_graph=True)  # same dt: captured again because the lists moved
    got = rk.get_state()
    rk.close()
    assert np.array_equal(got, want)
