"""Ensembles: instances of uneven sizes advanced together by one CUDA graph per step over several
streams give exactly the states each instance reaches on its own."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.learned  # noqa: F401  (L.learned: the shipped selector weights)
import lpmcxx_b200.workloads as W


def test_ensemble_workload_shapes():
    inst = W.ensemble_instances(levels=(2, 3), per_level=2)
    assert [lvl for lvl, _, _ in inst] == [2, 2, 3, 3]
    for lvl, p, n_src in inst:
        assert n_src == 20 * 4 ** lvl and p.shape == (n_src + 2 + 10 * 4 ** lvl, 4)
        assert abs((p[:n_src, 3]).sum()) < 1e-10 * np.abs(p[:n_src, 3]).sum()  # zero net circulation
    # seeded: different instances, same call same data
    again = W.ensemble_instances(levels=(2, 3), per_level=2)
    assert all(np.array_equal(a[1], b[1]) for a, b in zip(inst, again))
    assert not np.array_equal(inst[0][1], inst[1][1])


@pytest.mark.gpu
@pytest.mark.parametrize("learned", [False, True])
def test_ensemble_matches_single_instances(ctx, learned):
    inst = W.ensemble_instances(levels=(3, 4, 5), per_level=2)
    solver = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=learned, tolerance=2e-8)
    params = L.learned.load()[0] if learned else None
    ens = L.Ensemble(ctx, L.biot_savart_kernel(), solver, [n for _, _, n in inst], [p.shape[0] for _, p, _ in inst],
                     lanes=3)
    if learned:
        ens.set_mlp(params)
    for i, (_, p, _) in enumerate(inst):
        ens.instance(i).set_state(p)
    assert sorted({ens.lane_of(i) for i in range(len(inst))}) == [0, 1, 2]
    ens.step(0.01, 3, use_graph=True)
    got = [ens.instance(i).get_state() for i in range(len(inst))]
    ens.close()
    for i, (_, p, n_src) in enumerate(inst):
        rk = L.RK4(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
        if learned:
            rk.set_mlp(params)
        rk.set_state(p)
        rk.step(0.01, 3, use_graph=False)
        want = rk.get_state()
        rk.close()
        assert np.array_equal(got[i], want), i


@pytest.mark.gpu
def test_ensemble_instances_track_fp64_direct_rk4(ctx):
    """Every instance of a learned-treecode ensemble (the ensemble workload's RH wave + seeded Gaussian, icos
    L3..L5, headline selector setting) stays within the treecode's error budget of the FP64 direct-sum RK4
    run of the same instance: after 3 graph-replayed steps of dt 0.01 the displacement X_3 - X_0 differs from
    the FP64 direct sum's by at most 5e-6 relative (L2 over the instance), and the velocity at the final
    state by at most 2e-6 relative."""
    import torch

    inst = W.ensemble_instances(levels=(3, 4, 5), per_level=2, seed=77)
    solver = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=True, tolerance=5e-7)
    ens = L.Ensemble(ctx, L.biot_savart_kernel(), solver, [n for _, _, n in inst], [p.shape[0] for _, p, _ in inst],
                     lanes=3)
    ens.set_mlp(L.learned.load()[0])
    ens.set_param("order_bias", 2)
    for i, (_, p, _) in enumerate(inst):
        ens.instance(i).set_state(p)
    ens.step(0.01, 3, use_graph=True)
    torch.cuda.synchronize()
    for i, (_, p, n_src) in enumerate(inst):
        rki = ens.instance(i)
        got = rki.get_state()
        u_tree = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
        rki.velocity(u_tree)
        torch.cuda.synchronize()
        rk = L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(L.LPM_PREC_F64), n_src, p.shape[0])
        rk.set_state(p)
        rk.step(0.01, 3, use_graph=False)
        want = rk.get_state()
        rk.set_state(got)
        u64 = torch.empty_like(u_tree)
        rk.velocity(u64)
        torch.cuda.synchronize()
        rk.close()
        disp_err = np.linalg.norm(got[:, :3] - want[:, :3]) / np.linalg.norm(want[:, :3] - p[:, :3])
        vel_err = float(torch.linalg.norm(u_tree - u64) / torch.linalg.norm(u64))
        assert disp_err < 5e-6, (i, disp_err)
        assert vel_err < 2e-6, (i, vel_err)
        assert np.array_equal(got[:, 3], p[:, 3])  # strengths are carried unchanged


@pytest.mark.gpu
def test_ensemble_set_param_between_graph_steps_takes_effect(ctx):
    """Changing an instance's parameter after the ensemble's step graph exists drops that graph: the next
    steps use the new value, as an uncaptured run of the same instances does."""
    inst = W.ensemble_instances(levels=(3, 4), per_level=1, seed=5)
    solver = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=True, tolerance=5e-7)
    params = L.learned.load()[0]
    ens = L.Ensemble(ctx, L.biot_savart_kernel(), solver, [n for _, _, n in inst], [p.shape[0] for _, p, _ in inst],
                     lanes=2)
    ens.set_mlp(params)
    for i, (_, p, _) in enumerate(inst):
        ens.instance(i).set_state(p)
    ens.step(0.01, 2, use_graph=True)   # warm-up step + one graph replay
    ens.instance(1).set_param("order_bias", 3)
    ens.instance(0).set_param("theta", 0.4)
    ens.step(0.01, 2, use_graph=True)
    got = [ens.instance(i).get_state() for i in range(len(inst))]
    ens.close()
    for i, (_, p, n_src) in enumerate(inst):
        rk = L.RK4(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
        rk.set_mlp(params)
        rk.set_state(p)
        rk.step(0.01, 2, use_graph=False)
        rk.set_param("order_bias" if i == 1 else "theta", 3 if i == 1 else 0.4)
        rk.step(0.01, 2, use_graph=False)
        want = rk.get_state()
        rk.close()
        assert np.array_equal(got[i], want), i


@pytest.mark.gpu
def test_fused_ensemble_equals_lane_mode(ctx):
    """The fused step (far field of all instances as one persistent launch per Taylor order, near field as one
    per near tile shape) gives bitwise the states of the lane mode, where every instance launches its own far
    and near kernels, on a mixed ensemble: learned-order instances (one with FP64 orders >= 6, whose orders 6..11
    keep their own launches; one with another near tile shape), fixed orders 8 and 12 (order 12 is above the
    fused FP32 kernels) and an FP32 direct-sum instance; with the lanes in 1, 2 (the default) or 3 groups that
    step independently, each with its own fused launches."""
    inst = W.ensemble_instances(levels=(3, 4, 5), per_level=2, seed=11)
    learned = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=True, tolerance=5e-7)
    solvers = [learned, L.tree_solver(L.LPM_PREC_F32, 8, 64, 0.6), learned, L.direct_solver(L.LPM_PREC_F32),
               learned, L.tree_solver(L.LPM_PREC_F32, 12, 128, 0.5)]
    params = L.learned.load()[0]

    def run(fused: bool, use_graph: bool, nsteps: int, groups: int = 2):
        ens = L.Ensemble(ctx, L.biot_savart_kernel(), solvers, [n for _, _, n in inst],
                         [p.shape[0] for _, p, _ in inst], lanes=3)
        assert ens.get_param("fused") == 1.0 and ens.get_param("fused_groups") == 2.0  # the defaults
        ens.set_param("fused", 1 if fused else 0)
        ens.set_param("fused_groups", groups)
        assert ens.get_param("fused") == (1.0 if fused else 0.0)
        for i in (0, 2, 4):
            ens.instance(i).set_mlp(params)
        ens.instance(2).set_param("f64_from", 6)
        ens.instance(4).set_param("near_targets", 4)
        ens.instance(4).set_param("near_tile", 512)
        ens.instance(4).set_param("near_split", 1)
        for i, (_, p, _) in enumerate(inst):
            ens.instance(i).set_state(p)
        ens.step(0.01, nsteps, use_graph=use_graph)
        out = [ens.instance(i).get_state() for i in range(len(inst))]
        ens.close()
        return out

    lanes = run(False, True, 3)
    for use_graph, nsteps, groups in ((True, 3, 2), (True, 3, 1), (True, 3, 3), (False, 2, 2)):
        fused = run(True, use_graph, nsteps, groups)
        ref = lanes if nsteps == 3 else run(False, False, 2)
        for i in range(len(inst)):
            assert np.array_equal(fused[i], ref[i]), (use_graph, groups, i)
    e = L.Ensemble(ctx, L.biot_savart_kernel(), learned, [inst[0][2]], [inst[0][1].shape[0]], lanes=1)
    try:
        for name, value in (("fused", 2), ("fused_groups", 0), ("fused_groups", 65), ("fused_groups", 1.5)):
            with pytest.raises(L.LpmError):
                e.set_param(name, value)
        with pytest.raises(L.LpmError):
            e.get_param("no_such_parameter")
        assert e.get_param("fused") == 1.0 and e.get_param("fused_groups") == 2.0  # unchanged by the refusals
    finally:
        e.close()


@pytest.mark.gpu
def test_fused_ensemble_edge_instances(ctx):
    """Fused steps with instances that take no part in the fused launches: a one-instance ensemble, and an
    ensemble holding an instance whose particles carry no sources (its velocity is zero, so it stays put up to
    the re-projection's rounding) next to a treecode instance; both give the lane mode's states bitwise."""
    inst = W.ensemble_instances(levels=(3, 4), per_level=1, seed=21)
    solver = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=True, tolerance=5e-7)
    params = L.learned.load()[0]
    passive = inst[0][1].copy()
    cases = [([inst[1]], [inst[1][2]]), ([inst[1], (3, passive, 0)], [inst[1][2], 0])]
    for members, n_src in cases:
        got = {}
        for fused in (1, 0):
            ens = L.Ensemble(ctx, L.biot_savart_kernel(), solver, n_src, [p.shape[0] for _, p, _ in members],
                             lanes=2)
            ens.set_param("fused", fused)
            ens.set_mlp(params)
            for i, (_, p, _) in enumerate(members):
                ens.instance(i).set_state(p)
            ens.step(0.01, 3, use_graph=True)
            got[fused] = [ens.instance(i).get_state() for i in range(len(members))]
            ens.close()
        for i in range(len(members)):
            assert np.array_equal(got[1][i], got[0][i]), (len(members), i)
        if len(members) == 2:  # zero velocity: only the re-projection onto the sphere touches the positions
            assert np.allclose(got[1][1], passive, rtol=0, atol=1e-14)
