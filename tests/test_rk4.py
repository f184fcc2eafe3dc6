"""RK4 stage loop: the CPU oracle's semantics (CPU) and the CUDA integrator against it (GPU)."""
import numpy as np
import pytest

import lpmcxx_b200 as L
import lpmcxx_b200.workloads as W
import oracle


def test_oracle_rk4_solid_body_rotation():
    # zeta = 2z is solid-body rotation u = (-y, x, 0): after t = 0.1 every particle has turned by
    # 0.1 rad about z, up to the O(h^2) discretisation error of the direct sum at icos level 4
    mesh = L.build_mesh("icos", 4)
    p, n_src = W.particles(mesh, 2.0 * mesh.face_xyz[:, 2])
    out = oracle.rk4_direct(p, n_src, dt=0.01, nsteps=10)
    c, s = np.cos(0.1), np.sin(0.1)
    rot = p[:, :3] @ np.array([[c, s, 0], [-s, c, 0], [0, 0, 1]])
    assert np.abs(out[:, :3] - rot).max() < 2e-3
    assert np.allclose(np.linalg.norm(out[:, :3], axis=1), 1.0, atol=1e-15)
    assert np.array_equal(out[:, 3], p[:, 3])


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_rk4_direct_f64_matches_oracle(ctx, use_graph):
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", 3)
    ref = oracle.rk4_direct(p, n_src, dt=0.01, nsteps=3)
    rk = L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(L.LPM_PREC_F64), n_src, p.shape[0])
    rk.set_state(p)
    rk.step(0.01, 3, use_graph=use_graph)
    got = rk.get_state()
    rk.close()
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-12
    assert np.array_equal(got[:, 3], p[:, 3])


@pytest.mark.gpu
def test_rk4_direct_f32_close_to_oracle(ctx):
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", 4)
    ref = oracle.rk4_direct(p, n_src, dt=0.005, nsteps=4)
    rk = L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(L.LPM_PREC_F32), n_src, p.shape[0])
    rk.set_state(p)
    rk.step(0.005, 2, use_graph=False)
    rk.step(0.005, 2, use_graph=True)
    got = rk.get_state()
    rk.close()
    # FP32 velocities (rel. error ~1e-6) integrated over 4 steps of 0.005
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-7
    assert np.allclose(np.linalg.norm(got[:, :3], axis=1), 1.0, atol=1e-14)


@pytest.mark.gpu
def test_rk4_velocity_matches_direct_sum(ctx):
    torch = ctx.use_torch_stream()
    mesh, p, n_src = W.gaussian_vortex_mesh("cube", 3)
    rk = L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(L.LPM_PREC_F64), n_src, p.shape[0])
    rk.set_state(p)
    u = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
    rk.velocity(u)
    ctx.synchronize()
    ref = oracle.bs_direct(p[:n_src], p)
    assert np.abs(u.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-12
    rk.close()


@pytest.mark.gpu
def test_rk4_bad_args(ctx):
    with pytest.raises(L.LpmError):
        L.RK4(ctx, L.poisson_kernel(), L.direct_solver(), 1, 2)
    with pytest.raises(L.LpmError):
        L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(), 5, 2)


@pytest.mark.gpu
def test_config1_cube_l8_ten_steps_fp32_vs_fp64(ctx):
    """The at-scale direct-sum configuration: cubed sphere refined 8 levels (393,216 face sources, 393,218
    vertices), Gaussian vortex, 10 RK4 steps of dt = 0.005 with the FP64 and the FP32 (FP64-accumulated) direct
    sums: the FP32 trajectory's displacement stays within 1e-6 relative of the FP64 one, and every particle stays
    on the sphere."""
    torch = ctx.use_torch_stream()
    _, p, n_src = W.gaussian_vortex_mesh("cube", 8)
    assert n_src == 393_216 and p.shape[0] - n_src == 393_218
    final = {}
    for prec in (L.LPM_PREC_F64, L.LPM_PREC_F32):
        rk = L.RK4(ctx, L.biot_savart_kernel(), L.direct_solver(prec), n_src, p.shape[0])
        rk.set_state(torch.tensor(p, device="cuda"))
        rk.step(0.005, 10, use_graph=True)
        final[prec] = rk.get_state()
        rk.close()
    d64 = final[L.LPM_PREC_F64][:, :3] - p[:, :3]
    d32 = final[L.LPM_PREC_F32][:, :3] - p[:, :3]
    assert np.linalg.norm(d32 - d64) / np.linalg.norm(d64) < 1e-6
    for s in final.values():
        assert np.abs(np.linalg.norm(s[:, :3], axis=1) - 1.0).max() < 1e-14
