"""Checkpoint / resume of RK4 runs and ensembles: a run resumed from a checkpoint steps bitwise as the run that
wrote it; damaged, truncated, missing or mismatched files are refused and leave every state as it was."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.learned  # noqa: F401  (L.learned: the shipped selector weights)
import lpmcxx_b200.workloads as W


def _solver():
    return L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.5, learned=True, tolerance=5e-7)


@pytest.mark.gpu
def test_rk4_checkpoint_resume_is_bitwise(ctx, tmp_path):
    (_, p, n_src), = W.ensemble_instances(levels=(4,), per_level=1, seed=3)
    params = L.learned.load()[0]

    def make(ns=n_src):
        rk = L.RK4(ctx, L.biot_savart_kernel(), _solver(), ns, p.shape[0])
        rk.set_mlp(params)
        return rk

    a = make()
    a.set_state(p)
    a.step(0.01, 4, use_graph=True)
    want = a.get_state()
    a.close()
    b = make()
    b.set_state(p)
    b.step(0.01, 2, use_graph=True)
    path = tmp_path / "run.ckpt"
    b.checkpoint_write(path, step=2, t=0.02, dt=0.01)
    mid = b.get_state()
    b.close()
    c = make()
    assert c.checkpoint_read(path) == (2, 0.02, 0.01)
    assert np.array_equal(c.get_state(), mid)
    c.step(0.01, 2, use_graph=True)
    assert np.array_equal(c.get_state(), want)
    raw = path.read_bytes()
    bad = bytearray(raw)
    bad[100] ^= 1  # a bit of the particle data
    (tmp_path / "bad.ckpt").write_bytes(bytes(bad))
    (tmp_path / "short.ckpt").write_bytes(raw[:-9])
    (tmp_path / "long.ckpt").write_bytes(raw + b"\0")
    before = c.get_state()
    for name in ("bad.ckpt", "short.ckpt", "long.ckpt", "missing.ckpt"):
        with pytest.raises(L.LpmError):
            c.checkpoint_read(tmp_path / name)
        assert np.array_equal(c.get_state(), before), name
    c.close()
    other = make(n_src - 20)  # other source count
    with pytest.raises(L.LpmError):
        other.checkpoint_read(path)
    other.close()


@pytest.mark.gpu
def test_ensemble_checkpoint_resume_is_bitwise(ctx, tmp_path):
    inst = W.ensemble_instances(levels=(3, 4), per_level=1, seed=9)
    params = L.learned.load()[0]

    def make():
        ens = L.Ensemble(ctx, L.biot_savart_kernel(), _solver(), [n for _, _, n in inst],
                         [p.shape[0] for _, p, _ in inst], lanes=2)
        ens.set_mlp(params)
        return ens

    a = make()
    for i, (_, p, _) in enumerate(inst):
        a.instance(i).set_state(p)
    a.step(0.01, 3)
    want = [a.instance(i).get_state() for i in range(len(inst))]
    a.close()
    b = make()
    for i, (_, p, _) in enumerate(inst):
        b.instance(i).set_state(p)
    b.step(0.01, 1)
    path = tmp_path / "ens.ckpt"
    b.checkpoint_write(path, step=1, t=0.01, dt=0.01)
    b.close()
    c = make()
    assert c.checkpoint_read(path) == (1, 0.01, 0.01)
    c.step(0.01, 2)
    for i in range(len(inst)):
        assert np.array_equal(c.instance(i).get_state(), want[i]), i
    c.close()
    rk = L.RK4(ctx, L.biot_savart_kernel(), _solver(), inst[0][2], inst[0][1].shape[0])
    with pytest.raises(L.LpmError):  # two instances in the file, one RK4
        rk.checkpoint_read(path)
    rk.close()
