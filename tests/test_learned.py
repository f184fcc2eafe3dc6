"""Learned Taylor-order selector: MLP kernels against the FP64 numpy oracle, the labels the treecode
generates, and the learned treecode against the FP64 direct sum (its judge) and the fixed-order
treecode (its fallback)."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.workloads as W
from lpmcxx_b200 import learned
from oracle import mlp as OM


def random_problem(n, seed):
    rng = np.random.default_rng(seed)
    f = (rng.normal(size=(n, 8)) * rng.uniform(0.5, 3.0, 8) + rng.normal(size=8)).astype(np.float32)
    lab = rng.integers(0, 12, n).astype(np.int32)
    return f, lab


# ------------------------------------------------------------------ CPU: the oracle itself
def test_oracle_gradient_matches_finite_differences():
    f, lab = random_problem(40, 0)
    p = L.mlp_init(f, 1).astype(np.float64)
    _, g = OM.loss_and_grad(p, f, lab)
    rng = np.random.default_rng(2)
    h = 1e-6
    for i in rng.choice(OM.N_TRAINABLE, 40, replace=False):
        pp = p.copy()
        pp[i] += h
        lp = OM.loss_and_grad(pp, f, lab)[0]
        pp[i] -= 2 * h
        lm = OM.loss_and_grad(pp, f, lab)[0]
        assert abs((lp - lm) / (2 * h) - g[i]) < 1e-7 + 1e-6 * abs(g[i])


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0, 1.0 + 2 ** -8 + 2 ** -20], np.float32)
    r = OM.round_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie at 1 + 2^-8 rounds to even
    assert r[2] == np.float32(1.0078125)
    assert r[5] == np.float32(1.0078125)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_layout_constants_agree():
    assert L.MLP_PARAMS == OM.N_PARAMS and L.MLP_TRAINABLE == OM.N_TRAINABLE


def test_shipped_selector_file():
    params, meta = learned.load()
    assert params is not None, "lpmcxx_b200/data/order_mlp.npz is missing"
    assert params.shape == (L.MLP_PARAMS,) and np.all(np.isfinite(params))
    assert meta["fields"] == 20 and meta["level"] == 8 and meta["pairs"] >= 400_000


# ------------------------------------------------------------------ GPU: training and inference kernels
@pytest.mark.gpu
def test_gradient_matches_oracle(ctx):
    f, lab = random_problem(3000, 3)  # 47 blocks of 64 samples, the last one partial
    p = L.mlp_init(f, 4)
    g, loss = L.mlp_grad(ctx, p, f, lab)
    lo, go = OM.loss_and_grad(p.astype(np.float64), f, lab)
    assert abs(loss - lo) < 1e-5 * lo
    assert np.linalg.norm(g - go) < 2e-5 * np.linalg.norm(go)


@pytest.mark.gpu
def test_bf16_inference_matches_oracle(ctx):
    f, lab = random_problem(20000, 5)
    p = L.mlp_init(f, 6)
    p[:L.MLP_TRAINABLE] *= 3.0  # spread the logits
    got = L.mlp_predict(ctx, p, f)
    want, margin = OM.predict_bf16(p, f)
    clear = margin > 1e-3  # FP32 accumulation may flip near-ties only
    assert clear.mean() > 0.95
    assert np.array_equal(got[clear], want[clear])


@pytest.mark.gpu
def test_training_fits_and_is_deterministic(ctx):
    rng = np.random.default_rng(7)
    f = rng.normal(size=(8192, 8)).astype(np.float32)
    proj = rng.normal(size=(8, 12))
    lab = (f @ proj).argmax(axis=1).astype(np.int32)
    p1 = L.mlp_init(f, 8)
    p2 = p1.copy()
    loss1 = L.mlp_train(ctx, f, lab, p1, epochs=15, minibatch=256, lr=3e-3, seed=9)
    loss2 = L.mlp_train(ctx, f, lab, p2, epochs=15, minibatch=256, lr=3e-3, seed=9)
    assert np.array_equal(p1, p2) and np.array_equal(loss1, loss2)
    assert loss1[-1] < 0.3 * loss1[0]
    assert (L.mlp_predict(ctx, p1, f) == lab).mean() > 0.9
    assert np.array_equal(p1[L.MLP_TRAINABLE:], L.mlp_init(f, 8)[L.MLP_TRAINABLE:])  # standardisation kept


# ------------------------------------------------------------------ GPU: labels from the treecode
def field(level, seed=None):
    if seed is None:
        return W.gaussian_vortex_mesh("icos", level)
    mesh = L.build_mesh("icos", level)
    p, n_src = learned.seeded_vortex_particles(mesh, seed)
    return mesh, p, n_src


@pytest.mark.gpu
def test_labels_follow_the_per_order_errors(ctx):
    torch = ctx.use_torch_stream()
    _, p, n_src = field(6, seed=3)
    d = torch.tensor(p, device="cuda")
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 8, 128, 0.6, learned=True,
                                                              tolerance=2e-8), n_src, p.shape[0])
    f, lab, err = ts.sample_labels(d[:n_src], d, 0, 3000, with_errors=True)
    f2, lab2, _ = ts.sample_labels(d[:n_src], d, 0, 3000)
    ts.close()
    assert 1000 < f.shape[0] <= 3000 and np.all(np.isfinite(f))
    assert np.array_equal(f, f2) and np.array_equal(lab, lab2)  # deterministic
    ok = err <= 1.0
    first = np.where(ok.any(axis=1), ok.argmax(axis=1), 11)
    assert np.array_equal(lab, first)
    # the series converges: higher orders are more accurate on the whole
    med = np.median(err, axis=0)
    assert med[10] < 1e-3 * med[0]
    assert len(np.unique(lab)) >= 5


# ------------------------------------------------------------------ GPU: the learned treecode
def eval_tree(ctx, torch, d, n_src, solver, params=None, prm=()):
    n = d.shape[0]
    ts = L.TreeSum(ctx, L.biot_savart_kernel(), solver, n_src, n)
    if params is not None:
        ts.set_mlp(params)
    for k, v in prm:
        ts.set_param(k, v)
    u = torch.empty((3, n), dtype=torch.float64, device="cuda")
    ts.eval(d[:n_src], d, u)
    st = ts.stats()
    ts.close()
    return u, st


def far_near_work(st):
    """Algorithmic flops of one evaluation: 8 per far coefficient, ~40 per far setup, 17 per near pair."""
    return 8.0 * st["far_terms"] + 40.0 * st["far_evals"] + 17.0 * st["near_pairs"]


@pytest.mark.gpu
def test_learned_fallback_is_the_fixed_order(ctx):
    torch = ctx.use_torch_stream()
    _, p, n_src = field(6)
    d = torch.tensor(p, device="cuda")
    u_fix, st_fix = eval_tree(ctx, torch, d, n_src, L.tree_solver(L.LPM_PREC_F32, 8, 128, 0.5))
    u_fb, st_fb = eval_tree(ctx, torch, d, n_src, L.tree_solver(L.LPM_PREC_F32, 8, 128, 0.5, learned=True))
    assert st_fb["far_evals"] == st_fix["far_evals"] and st_fb["near_pairs"] == st_fix["near_pairs"]
    assert float(torch.linalg.norm(u_fb - u_fix) / torch.linalg.norm(u_fix)) < 1e-12


@pytest.mark.gpu
def test_learned_order_meets_tolerance_with_less_work(ctx):
    """On a field outside the training set (the bench's vortex), at level 7: the learned treecode stays
    within rel L2 1e-6 of the FP64 direct sum and does less work than the fixed order-10 treecode of the
    same accuracy class."""
    params, _ = learned.load()
    torch = ctx.use_torch_stream()
    _, p, n_src = field(7)
    n = p.shape[0]
    d = torch.tensor(p, device="cuda")
    u64 = torch.empty((3, n), dtype=torch.float64, device="cuda")
    ctx.direct_sum_dev(L.biot_savart_kernel(), L.LPM_PREC_F64, d[:n_src], d, u64)
    u_l, st_l = eval_tree(ctx, torch, d, n_src, L.tree_solver(L.LPM_PREC_F32, 10, 256, 0.6, learned=True,
                                                              tolerance=learned.DEFAULT_EPS), params)
    u_f, st_f = eval_tree(ctx, torch, d, n_src, L.tree_solver(L.LPM_PREC_F32, 10, 256, 0.5))
    err_l = float(torch.linalg.norm(u_l - u64) / torch.linalg.norm(u64))
    err_f = float(torch.linalg.norm(u_f - u64) / torch.linalg.norm(u64))
    assert err_f < 1e-6
    assert err_l < 1e-6
    assert far_near_work(st_l) < 0.8 * far_near_work(st_f)


@pytest.mark.gpu
def test_learned_rk4_graph_matches_uncaptured(ctx):
    params, _ = learned.load()
    torch = ctx.use_torch_stream()
    _, p, n_src = field(5)
    d = torch.tensor(p, device="cuda")
    solver = L.tree_solver(L.LPM_PREC_F32, 10, 128, 0.6, learned=True)
    out = []
    for use_graph in (False, True):
        rk = L.RK4(ctx, L.biot_savart_kernel(), solver, n_src, p.shape[0])
        rk.set_mlp(params)
        rk.set_state(d)
        rk.step(0.01, 3, use_graph=use_graph)
        out.append(rk.get_state())
        rk.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.gpu
def test_order_bias_raises_orders_and_accuracy(ctx):
    """order_bias adds orders to every selector choice: more far-field terms, smaller error; values outside
    0..3 are rejected."""
    params, _ = learned.load()
    torch = ctx.use_torch_stream()
    _, p, n_src = field(6)
    n = p.shape[0]
    d = torch.tensor(p, device="cuda")
    u64 = torch.empty((3, n), dtype=torch.float64, device="cuda")
    ctx.direct_sum_dev(L.biot_savart_kernel(), L.LPM_PREC_F64, d[:n_src], d, u64, n_coincident=n_src)
    res = {}
    for bias in (0, 2):
        ts = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 10, 256, 0.5, learned=True,
                                                                  tolerance=1e-7), n_src, n)
        ts.set_mlp(params)
        ts.set_param("order_bias", bias)
        assert ts.get_param("order_bias") == bias
        u = torch.empty((3, n), dtype=torch.float64, device="cuda")
        ts.eval(d[:n_src], d, u)
        torch.cuda.synchronize()
        res[bias] = (float(torch.linalg.norm(u - u64) / torch.linalg.norm(u64)), ts.stats()["far_terms"])
        for bad in (-1, 4, 1.5):
            with pytest.raises(L.LpmError):
                ts.set_param("order_bias", bad)
        ts.close()
    assert res[2][1] > res[0][1]
    assert res[2][0] < res[0][0]
    # the bias belongs to the learned selector: a fixed-order solver refuses it
    fixed = L.TreeSum(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F32, 10, 256, 0.5), n_src, n)
    with pytest.raises(L.LpmError):
        fixed.set_param("order_bias", 1)
    fixed.close()
