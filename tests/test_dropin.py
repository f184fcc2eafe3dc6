"""The drop-in C++ classes: the reference's Lpm::DirectSum / Lpm::TreeSum API (its own headers and
callers) with the GPU implementations linked in place of src/LpmDirectSum.cpp / src/LpmTreeSum.cpp,
checked against fixtures produced by the unmodified reference."""
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import golden, rel_l2, rel_linf

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "lpmcxx_b200" / "dropin" / "_build" / "dropin_driver"
needs_driver = pytest.mark.skipif(not DRIVER.exists(), reason="drop-in driver not built (make -C lpmcxx_b200/dropin)")


def run(*args):
    env = dict(os.environ)
    env["LPM_MESH_SEED_DIR"] = str(DRIVER.parent / "meshSeeds")
    r = subprocess.run([str(DRIVER), *map(str, args)], capture_output=True, text=True, env=env, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return r.stdout


@needs_driver
def test_driver_loads_library_and_reports_usage():
    r = subprocess.run([str(DRIVER)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


def direct_case(kind, level, delta, name):
    g = golden(name)
    with tempfile.TemporaryDirectory() as d:
        g["face_zeta"].astype("<f8").tofile(f"{d}/zeta.bin")
        run("direct", kind, level, delta, f"{d}/zeta.bin", d)
        vv = np.fromfile(f"{d}/vert_vel.bin").reshape(-1, 3)
        fv = np.fromfile(f"{d}/face_vel.bin").reshape(-1, 3)
    return g, vv, fv


@pytest.mark.gpu
@needs_driver
def test_dropin_direct_sum_matches_reference_icos4():
    g, vv, fv = direct_case("icos", 4, 0.0, "direct_icos4_rh.npz")
    assert rel_linf(vv, g["vert_vel"]) < 1e-12
    assert rel_linf(fv, g["face_vel"]) < 1e-12


@pytest.mark.gpu
@needs_driver
def test_dropin_direct_sum_nonsingular_kernel_cube3():
    # BiotSavartSphere(0.05): delta recovered through the kernel's public interface
    g, vv, fv = direct_case("cube", 3, 0.05, "direct_cube3_gauss_d05.npz")
    assert rel_linf(vv, g["vert_vel"]) < 1e-12
    assert rel_linf(fv, g["face_vel"]) < 1e-12


@pytest.mark.gpu
@needs_driver
@pytest.mark.parametrize("name", ["spheregreens", "planarlog", "delta3d", "spheredelta"])
def test_dropin_scalar_kernels_match_reference(name):
    # the reference's own ScalarKernel objects through the drop-in DirectSum::meshSolve (scalar branch);
    # their protected parameters are recovered through the public interface
    g = golden("scalar_icos3_harm.npz")
    with tempfile.TemporaryDirectory() as d:
        g["face_zeta"].astype("<f8").tofile(f"{d}/zeta.bin")
        run("scalar", "icos", 3, name, float(g[f"{name}_param"]), f"{d}/zeta.bin", d)
        vp = np.fromfile(f"{d}/vert_phi.bin")
        fp = np.fromfile(f"{d}/face_phi.bin")
    assert rel_linf(vp, g[f"{name}_vert_phi"]) < 1e-12
    assert rel_linf(fp, g[f"{name}_face_phi"]) < 1e-12


@pytest.mark.gpu
@needs_driver
def test_dropin_meshfree_poisson_matches_reference():
    g = golden("poisson_2000.npz")
    n = g["xyz"].shape[0]
    with tempfile.TemporaryDirectory() as d:
        np.concatenate([g["xyz"], g["charge"][:, None]], axis=1).astype("<f8").tofile(f"{d}/p.bin")
        run("poisson", n, f"{d}/p.bin", d)
        phi = np.fromfile(f"{d}/potential.bin")
    assert rel_linf(phi, g["potential"]) < 1e-12


@pytest.mark.gpu
@needs_driver
def test_dropin_treesum_against_reference_direct_sum():
    g = golden("direct_icos4_rh.npz")
    with tempfile.TemporaryDirectory() as d:
        g["face_zeta"].astype("<f8").tofile(f"{d}/zeta.bin")
        out = run("tree", "icos", 4, 6, 32, 0.5, f"{d}/zeta.bin", d)
        vv = np.fromfile(f"{d}/vert_vel.bin").reshape(-1, 3)
        fv = np.fromfile(f"{d}/face_vel.bin").reshape(-1, 3)
    assert json.loads(out.strip().splitlines()[-1])["mac_count"] > 0
    leaf = np.any(g["face_vel"] != 0, axis=1)
    # order 6 (|k| < 6) at theta 0.5: the accuracy class of the host-API treecode test
    assert rel_l2(vv, g["vert_vel"]) < 2e-3
    assert rel_l2(fv[leaf], g["face_vel"][leaf]) < 2e-3


@pytest.mark.gpu
@needs_driver
def test_dropin_treesum_node_count_matches_reference_tree():
    # the reference's mesh constructor counts the nodes of its tree (nNodes()) and leaves depth() at 0
    ref = golden("tree_icos4_m64.npz")
    g = golden("direct_icos4_rh.npz")
    with tempfile.TemporaryDirectory() as d:
        g["face_zeta"].astype("<f8").tofile(f"{d}/zeta.bin")
        out = json.loads(run("tree", "icos", 4, 6, 64, 0.5, f"{d}/zeta.bin", d).strip().splitlines()[-1])
    assert out["n_nodes"] == ref["node_level"].shape[0]
    assert out["depth"] == 0


@pytest.mark.gpu
@needs_driver
def test_dropin_meshfree_treesum_node_count_matches_reference_tree():
    """TreeSum(coords, ...) builds the reference's meshfree tree (Tree(coords) root, split while a node holds
    more than the leaf capacity): its nNodes() is the reference tree's node count."""
    ref = golden("pointtree_8000_m10.npz")
    xyz = ref["xyz"]
    with tempfile.TemporaryDirectory() as d:
        xyz.astype("<f8").tofile(f"{d}/xyz.bin")
        out = json.loads(run("ptree", xyz.shape[0], f"{d}/xyz.bin", 10).strip().splitlines()[-1])
    assert out["n_nodes"] == ref["node_level"].shape[0]
    assert out["depth"] == 0


@pytest.mark.gpu
@needs_driver
def test_dropin_treesum_fp64_far_field_switch(ctx):
    """LPM_B200_PRECISION=f64 evaluates the drop-in TreeSum's far expansions in FP64: its output is the host
    API's FP64-far-field treecode (lpm_tree_sum_mesh with LPM_PREC_F64) on the same mesh and field, and
    differs from the FP32 far field's."""
    import lpmcxx_b200 as L

    g = golden("direct_icos4_rh.npz")
    out = {}
    for prec in ("f32", "f64"):
        with tempfile.TemporaryDirectory() as d:
            g["face_zeta"].astype("<f8").tofile(f"{d}/zeta.bin")
            env = dict(os.environ, LPM_B200_PRECISION=prec, LPM_MESH_SEED_DIR=str(DRIVER.parent / "meshSeeds"))
            r = subprocess.run([str(DRIVER), "tree", "icos", "4", "8", "32", "0.5", f"{d}/zeta.bin", d],
                               capture_output=True, text=True, env=env, timeout=600)
            assert r.returncode == 0, r.stderr
            out[prec] = np.fromfile(f"{d}/vert_vel.bin").reshape(-1, 3)
    mesh = L.build_mesh("icos", 4)
    vo, _, _ = L.tree_sum_mesh(ctx, L.biot_savart_kernel(), L.tree_solver(L.LPM_PREC_F64, 8, 32, 0.5), mesh,
                               g["face_zeta"])
    assert rel_linf(out["f64"], vo.T) < 1e-13
    assert np.abs(out["f64"] - out["f32"]).max() > 0.0
    assert rel_l2(out["f64"], g["vert_vel"]) < 1e-3
