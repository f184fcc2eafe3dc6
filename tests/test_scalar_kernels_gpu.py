"""The reference's ScalarKernel family (SphereGreensFn, PlanarGreensFnFreeBoundaries, SecondOrderDelta3d,
SphereDelta; src/LpmScalarKernel.h:19-78) as FP64 GPU direct sums through the C ABI.

Tolerance: 1e-12 relative (L-infinity, relative to the largest value) against the reference's own
DirectSum::meshSolve outputs (tests/golden/scalar_icos3_harm.npz) and against the oracle's restatement
for the meshfree and device-pointer entry points.
"""
import numpy as np
import pytest

import lpmcxx_b200 as L
import oracle
from conftest import golden, rel_linf

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
CASES = (("spheregreens", L.sphere_greens_kernel, 3, True), ("planarlog", lambda p: L.planar_log_kernel(), 4, True),
         ("delta3d", L.delta3d_kernel, 5, False), ("spheredelta", L.sphere_delta_kernel, 6, False))


@pytest.mark.parametrize("name,make,kind,singular", CASES)
def test_scalar_mesh_matches_reference(ctx, name, make, kind, singular):
    g = golden("scalar_icos3_harm.npz")
    m = L.build_mesh("icos", 3)
    kern = make(float(g[f"{name}_param"]))
    vo, fo = ctx.direct_sum_mesh(kern, L.LPM_PREC_F64, m, g["face_zeta"])
    assert vo.shape == (1, m.n_verts) and fo.shape == (1, m.n_faces)
    leaf = m.leaf
    got = np.concatenate([fo[0][leaf], vo[0]])
    ref = np.concatenate([g[f"{name}_face_phi"][leaf], g[f"{name}_vert_phi"]])
    assert rel_linf(got, ref) < F64_TOL, name
    assert np.all(fo[0][~leaf] == 0.0)  # divided faces untouched


def test_scalar_mesh_target_slice(ctx):
    g = golden("scalar_icos3_harm.npz")
    m = L.build_mesh("icos", 3)
    vo, fo = ctx.direct_sum_mesh(L.sphere_greens_kernel(), L.LPM_PREC_F64, m, g["face_zeta"],
                                 vert_range=(10, 200), face_range=(300, 900))
    leaf = m.leaf
    sel = np.zeros(m.n_faces, bool)
    sel[300:901] = True
    assert rel_linf(vo[0][10:201], g["spheregreens_vert_phi"][10:201]) < F64_TOL
    assert rel_linf(fo[0][sel & leaf], g["spheregreens_face_phi"][sel & leaf]) < F64_TOL
    assert np.all(vo[0][:10] == 0) and np.all(vo[0][201:] == 0) and np.all(fo[0][~(sel & leaf)] == 0)


@pytest.mark.parametrize("name,make,kind,singular", CASES)
def test_scalar_meshfree_vs_oracle(ctx, name, make, kind, singular):
    rng = np.random.default_rng(7)
    n = 3001
    xyz = rng.normal(size=(n, 3))
    xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
    q, w = rng.uniform(-1, 1, n), rng.uniform(0.5, 1.5, n)
    param = {3: 1.0, 4: 0.0, 5: 0.2, 6: 0.2}[kind]  # sphere radius or delta width
    got = ctx.direct_sum_meshfree(make(param), L.LPM_PREC_F64, xyz, q, weights=w, rng=(17, 2500))
    src = oracle.pack4(xyz, q * w)
    self_idx = np.arange(17, 2501) if singular else None
    ref = oracle.scalar_direct(kind, param, src, src[17:2501], self_idx)
    assert rel_linf(got[17:2501], ref) < F64_TOL
    assert np.all(got[:17] == 0) and np.all(got[2501:] == 0)


def test_scalar_dev_api_coincident(ctx):
    torch = pytest.importorskip("torch")
    ctx.use_torch_stream()
    rng = np.random.default_rng(3)
    xyz = rng.normal(size=(1500, 3))
    xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
    src = oracle.pack4(xyz, rng.uniform(-1, 1, 1500))
    tgt = np.concatenate([src[:700, :], oracle.pack4(rng.normal(size=(300, 3)) * 0.5)])
    out = torch.empty((1, tgt.shape[0]), dtype=torch.float64, device="cuda")
    ctx.direct_sum_dev(L.planar_log_kernel(), L.LPM_PREC_F64, torch.tensor(src, device="cuda"),
                       torch.tensor(tgt, device="cuda"), out, n_coincident=700)
    self_idx = np.full(tgt.shape[0], -1, np.int64)
    self_idx[:700] = np.arange(700)
    ref = oracle.scalar_direct(4, 0.0, src, tgt, self_idx)
    assert rel_linf(out.cpu().numpy()[0], ref) < F64_TOL


def test_poisson_on_mesh(ctx):
    g = golden("scalar_icos3_harm.npz")
    m = L.build_mesh("icos", 3)
    vo, fo = ctx.direct_sum_mesh(L.poisson_kernel(), L.LPM_PREC_F64, m, g["face_zeta"])
    leaf = m.leaf
    src = oracle.pack4(m.face_xyz[leaf], g["face_zeta"][leaf] * m.face_area[leaf])
    tgt = np.concatenate([oracle.pack4(m.face_xyz[leaf]), oracle.pack4(m.vert_xyz)])
    ref = oracle.poisson_direct(src, tgt)
    assert rel_linf(np.concatenate([fo[0][leaf], vo[0]]), ref) < F64_TOL


def test_scalar_kernel_rejections(ctx):
    m = L.build_mesh("icos", 1)
    zeta = np.ones(m.n_faces)
    for kern, prec, code in ((L.sphere_greens_kernel(), L.LPM_PREC_F32, L._capi.LPM_ERR_KERNEL),
                             (L.delta3d_kernel(0.0), L.LPM_PREC_F64, L._capi.LPM_ERR_ARG),
                             (L.sphere_greens_kernel(-1.0), L.LPM_PREC_F64, L._capi.LPM_ERR_ARG)):
        with pytest.raises(L.LpmError) as e:
            ctx.direct_sum_mesh(kern, prec, m, zeta)
        assert e.value.code == code
    with pytest.raises(L.LpmError) as e:  # the treecode takes Biot-Savart and 3D Poisson only
        L.TreeSum(ctx, L.sphere_greens_kernel(), L.tree_solver(L.LPM_PREC_F32, 6, 64, 0.5), 100, 100)
    assert e.value.code == L._capi.LPM_ERR_KERNEL
