"""Synthetic inputs of the benchmark workloads (no datasets are involved).

Vorticity fields on the sphere meshes, and the particle layout the RK4 integrator uses: the
undivided faces (centroid particles, strength = vorticity x area) first, then the vertices
(strength 0).
"""
from __future__ import annotations

import numpy as np

from . import SphereMesh, build_mesh


def rossby_haurwitz_4(xyz: np.ndarray, omega: float = 1.0, amp: float = 1.0) -> np.ndarray:
    """zeta = 2 omega sin(phi) - (m+1)(m+2) K cos^m(phi) sin(phi) cos(m lambda), m = 4: the vorticity of
    the Rossby-Haurwitz wave; with omega = K = 1 this is 2 z - sphereHarmonic54
    (src/LpmAnalyticFunctions.h:87-103)."""
    z = xyz[:, 2]
    lam = np.arctan2(xyz[:, 1], xyz[:, 0])
    return 2.0 * omega * z - 30.0 * amp * np.cos(4.0 * lam) * z * (z * z - 1.0) ** 2


def rossby_haurwitz_4_velocity(xyz: np.ndarray) -> np.ndarray:
    """Exact velocity of rossby_haurwitz_4 with omega = K = 1: solid-body (-y, x, 0) minus
    rossbyHaurwitz54Velocity (src/LpmAnalyticFunctions.h:105-120); returns (3, n)."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    lat = np.arctan2(z, np.hypot(x, y))
    lon = np.arctan2(y, x)
    u = 0.5 * np.cos(4 * lon) * np.cos(lat) ** 3 * (5 * np.cos(2 * lat) - 3)
    v = 4 * np.cos(lat) ** 3 * np.sin(lat) * np.sin(4 * lon)
    rh = np.stack([-u * np.sin(lon) - v * np.sin(lat) * np.cos(lon), u * np.cos(lon) - v * np.sin(lat) * np.sin(lon),
                   v * np.cos(lat)])
    return np.stack([-y, x, np.zeros_like(x)]) - rh


def lat_lon_point(lat: float, lon: float) -> np.ndarray:
    return np.array([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])


def gaussian_vortex(xyz: np.ndarray, x0: np.ndarray, amp: float = 4.0 * np.pi, b: float = 16.0) -> np.ndarray:
    """amp * exp(-b |x - x0|^2)."""
    d = xyz - x0[None, :]
    return amp * np.exp(-b * np.einsum("ij,ij->i", d, d))


def particles(mesh: SphereMesh, face_zeta: np.ndarray) -> tuple[np.ndarray, int]:
    """(n, 4) particle array: undivided-face centroids with strength zeta*area, then the vertices."""
    leaf = mesh.leaf
    n_src = int(leaf.sum())
    p = np.zeros((n_src + mesh.n_verts, 4))
    p[:n_src, :3] = mesh.face_xyz[leaf]
    p[:n_src, 3] = face_zeta[leaf] * mesh.face_area[leaf]
    p[n_src:, :3] = mesh.vert_xyz
    return p, n_src


def gaussian_vortex_mesh(kind: str, level: int, lat: float = 0.05, lon: float = 0.75 * np.pi):
    """The Gaussian-vortex workload: zeta = 4 pi exp(-16|x - x0|^2) minus its area-weighted mean over the
    undivided faces, x0 at (lat 0.05, lon 3 pi/4).  Returns (mesh, particles (n,4), n_src)."""
    mesh = build_mesh(kind, level)
    zeta = gaussian_vortex(mesh.face_xyz, lat_lon_point(lat, lon))
    leaf = mesh.leaf
    zeta = zeta - (zeta[leaf] * mesh.face_area[leaf]).sum() / mesh.face_area[leaf].sum()
    p, n_src = particles(mesh, zeta)
    return mesh, p, n_src


def rh_wave_mesh(kind: str, level: int):
    mesh = build_mesh(kind, level)
    p, n_src = particles(mesh, rossby_haurwitz_4(mesh.face_xyz))
    return mesh, p, n_src


def splitmix64_uniform(n: int, seed: int) -> np.ndarray:
    """n doubles in [0, 1) from the splitmix64 generator (Steele, Lea & Flood, OOPSLA 2014): state
    s_i = seed + i * 0x9E3779B97F4A7C15 (i = 1, 2, ...), output mixed by two xor-shift-multiply rounds,
    top 53 bits scaled by 2^-53."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def poisson_cube(n: int = 1_048_576, seed: int = 0x2B) -> np.ndarray:
    """(n, 4) points uniform in [-1, 1]^3 with charges uniform in [-1, 1] (x, y, z, q consecutive draws
    of one splitmix64 stream): the 3D Poisson workload."""
    u = splitmix64_uniform(4 * n, seed).reshape(n, 4)
    return 2.0 * u - 1.0


def ensemble_instances(levels=(5, 6, 7, 8), per_level: int = 16, seed: int = 4000):
    """The ensemble workload: per_level instances on each icosahedral level, each a Rossby-Haurwitz m=4
    wave plus a Gaussian vortex (amplitude U(0.5, 2) 4 pi, width as gaussian_vortex) at a seeded random
    centre, minus its area-weighted mean.  Returns [(level, particles (n, 4), n_src)]."""
    out = []
    k = 0
    for level in levels:
        mesh = build_mesh("icos", level)
        leaf = mesh.leaf
        rh = rossby_haurwitz_4(mesh.face_xyz)
        for _ in range(per_level):
            rng = np.random.default_rng(seed + k)
            x0 = rng.normal(size=3)
            x0 /= np.linalg.norm(x0)
            amp = rng.uniform(0.5, 2.0) * 4.0 * np.pi
            zeta = rh + gaussian_vortex(mesh.face_xyz, x0, amp=amp)
            zeta = zeta - (zeta[leaf] * mesh.face_area[leaf]).sum() / mesh.face_area[leaf].sum()
            p, n_src = particles(mesh, zeta)
            out.append((level, p, n_src))
            k += 1
    return out
