"""Ensembles: instances of uneven sizes advanced together by one CUDA graph per step over several
streams give exactly the states each instance reaches on its own."""
import numpy as np
import pytest

import lpmcxx_b200 as L
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
