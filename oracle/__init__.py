"""FP64 CPU oracle for the DirectSum / TreeSum hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this package.  It is
the checker the CUDA library is compared against, never part of the product path.

* liboracle.so: the repo's own C restatement (lpm_oracle.c), pinned against the reference;
* _ref/ref_harness: the unmodified reference built from its sources (Makefile target `ref`),
  present only where the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_HARNESS = HERE / "_ref" / "ref_harness"

_lib = None


def build(ref: bool = False, ref_dir=None) -> None:
    """Compile liboracle.so (and, with ref=True, the reference harness under _ref/ from the reference's
    sources in ref_dir, default the Makefile's REF)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", *([f"REF={ref_dir}"] if ref_dir else [])], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        h = C.CDLL(str(LIB))
        P, I, D = C.c_void_p, C.c_int64, C.c_double
        h.oracle_bs_direct.argtypes = [P, I, P, I, D, D, P]
        h.oracle_poisson_direct.argtypes = [P, I, P, I, P]
        h.oracle_scalar_direct.argtypes = [C.c_int, D, P, I, P, I, P, P]
        h.oracle_rk4_direct.argtypes = [P, I, I, D, D, D, C.c_int]
        h.oracle_tree_build.argtypes = [P, I, P, C.c_int, C.c_int, P, P, P, P, P, P, P, P, I, P]
        _lib = h
    return _lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def pack4(xyz: np.ndarray, w: np.ndarray | None = None) -> np.ndarray:
    out = np.zeros((xyz.shape[0], 4))
    out[:, :3] = xyz
    if w is not None:
        out[:, 3] = w
    return out


def bs_direct(src4: np.ndarray, tgt4: np.ndarray, radius: float = 1.0, delta: float = 0.0) -> np.ndarray:
    """Biot-Savart direct sum (reference formula per pair); returns (3, n_tgt)."""
    src4, tgt4 = _c(src4), _c(tgt4)
    out = np.zeros((3, tgt4.shape[0]))
    lib().oracle_bs_direct(src4.ctypes.data, src4.shape[0], tgt4.ctypes.data, tgt4.shape[0], radius, delta,
                           out.ctypes.data)
    return out


def scalar_direct(kind: int, param: float, src4: np.ndarray, tgt4: np.ndarray, self_idx=None) -> np.ndarray:
    """ScalarKernel-family direct sum (kind 3..6 as LPM_KERNEL_*); self_idx[i] >= 0 is a source index
    target i skips (a singular kernel's own face)."""
    src4, tgt4 = _c(src4), _c(tgt4)
    out = np.zeros(tgt4.shape[0])
    si = None if self_idx is None else np.ascontiguousarray(self_idx, dtype=np.int64)
    lib().oracle_scalar_direct(int(kind), float(param), src4.ctypes.data, src4.shape[0], tgt4.ctypes.data,
                               tgt4.shape[0], None if si is None else si.ctypes.data, out.ctypes.data)
    return out


def poisson_direct(src4: np.ndarray, tgt4: np.ndarray) -> np.ndarray:
    src4, tgt4 = _c(src4), _c(tgt4)
    out = np.zeros(tgt4.shape[0])
    lib().oracle_poisson_direct(src4.ctypes.data, src4.shape[0], tgt4.ctypes.data, tgt4.shape[0], out.ctypes.data)
    return out


def rk4_direct(state: np.ndarray, n_src: int, dt: float, nsteps: int, radius: float = 1.0,
               delta: float = 0.0) -> np.ndarray:
    """nsteps RK4 steps (direct-sum velocity, re-projection); returns the new (n, 4) state."""
    s = _c(state).copy()
    lib().oracle_rk4_direct(s.ctypes.data, n_src, s.shape[0], radius, delta, dt, nsteps)
    return s


def tree_build(pts4: np.ndarray, box, max_per_leaf: int, max_depth: int = 21) -> dict:
    """Recursive octree with the reference's semantics; returns members / leaf_offsets / node arrays
    (nodes in depth-first pre-order) and the overflow mask."""
    pts4 = _c(pts4)
    n = pts4.shape[0]
    cap = max(64, 4 * n + 16)
    box = _c(box)
    members = np.zeros(max(n, 1), np.int64)
    offs = np.zeros(n + 2, np.int64)
    lv, par, cnt = (np.zeros(cap, np.int64) for _ in range(3))
    nbox = np.zeros((cap, 6))
    nl, nm, nn = C.c_int64(), C.c_int64(), C.c_int64()
    flags = lib().oracle_tree_build(pts4.ctypes.data, n, box.ctypes.data, max_per_leaf, max_depth,
                                    members.ctypes.data, offs.ctypes.data, C.byref(nl), C.byref(nm), lv.ctypes.data,
                                    par.ctypes.data, cnt.ctypes.data, nbox.ctypes.data, cap, C.byref(nn))
    k = nn.value
    return {"members": members[:nm.value], "leaf_offsets": offs[:nl.value + 1], "node_level": lv[:k],
            "node_parent": par[:k], "node_count": cnt[:k], "node_box": nbox[:k], "flags": flags}


def leaf_hashes(members: np.ndarray, leaf_offsets: np.ndarray) -> np.ndarray:
    """Per-leaf digest of an ordered member list: sum over the leaf's k-th member m of
    splitmix64(m) * (2k + 1) mod 2^64 (test infrastructure: lets a fixture hold a large tree's leaf
    membership in 8 bytes per leaf)."""
    m = np.asarray(members, dtype=np.uint64)
    off = np.asarray(leaf_offsets, dtype=np.int64)
    with np.errstate(over="ignore"):
        z = m + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        pos = np.arange(m.size, dtype=np.int64) - np.repeat(off[:-1], np.diff(off))
        z = z * (2 * pos.astype(np.uint64) + np.uint64(1))
        return np.add.reduceat(z, off[:-1]) if m.size else np.zeros(0, np.uint64)


def sakajo_tree(xyz: np.ndarray, depth: int, radius: float = 1.0) -> dict:
    """The tree of SakajoTree(order, depth, radius) over points xyz (src/LpmSakajo2009.cpp:25-63) with the
    points dropped into it as computeMoments does (:74-79, 201-213): root Box3d(radius) padded by 1e-5; a node
    of binary level j < 3 depth is bisected along axis (j + 2) mod 3 at its midpoint and keeps a child whose
    box meets the sphere (Box3d::intersectsSphere, src/LpmBox3d.cpp:79-129); a point follows the children whose
    half-open box holds it, down to level 3 depth.  Returns the non-empty nodes in depth-first order (level,
    parent, point count, box) and the leaves' members (increasing index), as the harness dumps them."""
    pts = np.asarray(xyz, dtype=np.float64)

    def mag(x, y, z):
        return float(np.sqrt(x * x + y * y + z * z))

    def meets(b):
        if b[0] <= 0.0 < b[1] and b[2] <= 0.0 < b[3] and b[4] <= 0.0 < b[5]:
            c = (0.0, 0.0, 0.0)
        else:
            c = tuple(lo if lo == hi else (lo if lo >= 0.0 else (hi if hi <= 0.0 else 0.0))
                      for lo, hi in ((b[0], b[1]), (b[2], b[3]), (b[4], b[5])))
        far = max(mag(b[i], b[2 + j], b[4 + k]) for i in (0, 1) for j in (0, 1) for k in (0, 1))
        return mag(*c) <= radius and far >= radius

    r = -radius
    lo, hi = r - 1e-5, radius + 1e-5
    out = {"node_level": [], "node_parent": [], "node_count": [], "node_box": [], "leaf_offsets": [0], "members": []}

    def walk(box, idx, level, parent):
        if idx.size == 0:
            return
        me = len(out["node_level"])
        out["node_level"].append(level)
        out["node_parent"].append(parent)
        out["node_count"].append(idx.size)
        out["node_box"].append(list(box))
        if level == 3 * depth:
            out["members"].extend(idx.tolist())
            out["leaf_offsets"].append(len(out["members"]))
            return
        a = (level + 2) % 3
        mid = 0.5 * (box[2 * a] + box[2 * a + 1])
        below = pts[idx, a] < mid
        for upper in (False, True):
            cb = list(box)
            cb[2 * a + (0 if upper else 1)] = mid
            if meets(cb):
                walk(cb, idx[below != upper], level + 1, me)

    inside = np.all((pts >= [lo, lo, lo]) & (pts < [hi, hi, hi]), axis=1)
    walk([lo, hi, lo, hi, lo, hi], np.nonzero(inside)[0], 0, -1)
    return {"node_level": np.array(out["node_level"]), "node_parent": np.array(out["node_parent"]),
            "node_count": np.array(out["node_count"]), "node_box": np.array(out["node_box"]),
            "leaf_offsets": np.array(out["leaf_offsets"]), "members": np.array(out["members"], dtype=np.int64)}


def mesh_root_box(vert_xyz: np.ndarray) -> np.ndarray:
    """Box3d(maxR) with its 1e-5 padding (src/LpmBox3d.h:21-33), maxR over the vertices
    (Coords::maxR, src/LpmCoords.cpp:136-143) -- the root of TreeSum's mesh constructor."""
    r2 = (vert_xyz[:, 0] * vert_xyz[:, 0] + vert_xyz[:, 1] * vert_xyz[:, 1]) + vert_xyz[:, 2] * vert_xyz[:, 2]
    maxr = float(np.sqrt(r2.max()))
    lo, hi = -maxr - 1e-5, maxr + 1e-5
    return np.array([lo, hi, lo, hi, lo, hi])


def coords_root_box(xyz: np.ndarray) -> np.ndarray:
    """Tree(coords) root box min - 1e-5*min, max + 1e-5*max per axis (src/LpmOctree.cpp:20-25)."""
    mn, mx = xyz.min(axis=0), xyz.max(axis=0)
    lo = mn - 1e-5 * mn
    hi = mx + 1e-5 * mx
    return np.array([lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]])


def run_ref_harness(*args: str, env: dict | None = None) -> str:
    """Run the compiled reference harness (raises FileNotFoundError when it was not built)."""
    if not REF_HARNESS.exists():
        raise FileNotFoundError(str(REF_HARNESS))
    e = dict(os.environ)
    e.setdefault("LPM_MESH_SEED_DIR", str(HERE / "_ref" / "meshSeeds"))
    if env:
        e.update(env)
    p = subprocess.run([str(REF_HARNESS), *map(str, args)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       env=e, check=True)
    return p.stdout
