"""FP64 numpy restatement of the treecode's far-field expansion -- TEST INFRASTRUCTURE ONLY.

The kernel of the reference (BiotSavartSphere, src/LpmVectorKernel.h:24-28) on the unit sphere is
(x cross y)/(1 - x.y) = 2 (x cross y) g(y) with g(y) = 1/|x - y|^2.  For a cluster of sources y_j with
strengths w_j, centre c, d = c - x, h = y - c, e = d/|d|^2, s = |e|^2:

    g(c + h) = (1/|d|^2) sum_{q + 2m < P} (-1)^m C(q+m, m) (-2)^q (e.h)^q (s |h|^2)^m

(the Chebyshev-U generating function 1/(1 - 2tu + t^2) = sum U_n(u) t^n with t = |h|/|d|,
u = -(d.h)/(|d||h|)).  These functions restate it literally, per source and per term, so that the
CUDA implementation's moment / coefficient / Horner machinery can be checked against it, and give the
reference per-pair truncation errors used to label training pairs.
"""
from __future__ import annotations

from math import comb

import numpy as np


def g_series(x: np.ndarray, y: np.ndarray, c: np.ndarray, P: int) -> np.ndarray:
    """Truncated series of 1/|x - y|^2 about c (total degree in h below P), for each row of y."""
    d = c - x
    h = y - c
    dd = d @ d
    e = d / dd
    s = 1.0 / dd
    eh = h @ e
    hh = np.einsum("ij,ij->i", h, h)
    out = np.zeros(y.shape[0])
    for m in range(0, (P + 1) // 2):
        for q in range(0, P - 2 * m):
            out += (-1) ** m * comb(q + m, m) * (-2.0) ** q * eh ** q * (s * hh) ** m
    return out / dd


def far_velocity_sum(x: np.ndarray, y: np.ndarray, w: np.ndarray, c: np.ndarray, P: int) -> np.ndarray:
    """sum_j w_j (x cross y_j) 2 g_P(y_j): the far-field contribution of one cluster at target x."""
    g = g_series(x, y, c, P)
    return np.cross(x, (2.0 * w * g)[:, None] * y).sum(axis=0)


def direct_velocity_sum(x: np.ndarray, y: np.ndarray, w: np.ndarray) -> np.ndarray:
    """sum_j w_j (x cross y_j)/(1 - x.y_j) (the reference kernel, without the -1/(4 pi) multiplier)."""
    den = 1.0 - y @ x
    return (np.cross(x, y) * (w / den)[:, None]).sum(axis=0)


# ------------------------------------------------------------------------------------------------------
# 3D Poisson kernel 1/|x - y|.  Two independent restatements of its truncated Taylor series about a
# cluster centre c (total degree in h = y - c at most p, the TaylorSeries3d convention |k| <= p of
# src/LpmTaylorSeries3d.cpp:16-50):
#   (1) the Gegenbauer form: with d = c - x, 1/|d + h| = (1/|d|) sum_n C_n^(1/2)(t) (|h|/|d|)^n,
#       t = -(d.h)/(|d||h|), C_n^(1/2) the Legendre polynomials, expanded per term (what the CUDA
#       coefficient kernel implements after summing over the sources);
#   (2) the Cartesian Taylor coefficients a_k = (1/k!) D_y^k (1/|x - y|) at y = c from the recurrence of
#       Lindsay & Krasny (J. Comput. Phys. 172, 2001) / Duan & Krasny, with R = x - c:
#       |k| |R|^2 a_k - (2|k| - 1) sum_i R_i a_{k - e_i} + (|k| - 1) sum_i a_{k - 2 e_i} = 0, a_0 = 1/|R|,
#       contracted with the ordinary moments M_k = sum_j w_j h_j^k.


def _gegenbauer_half_coef(q: int, m: int) -> float:
    """(-1)^m Gamma(q + m + 1/2) / (Gamma(1/2) m! q!) 2^q: the coefficient of t^q u^(q + 2m) in
    1/sqrt(1 - 2 t u + u^2) = sum_n C_n^(1/2)(t) u^n."""
    g = 1.0
    for k in range(q + m):
        g *= k + 0.5
    from math import factorial

    return (-1) ** m * g / (factorial(m) * factorial(q)) * 2.0 ** q


def potential_series_gegenbauer(x: np.ndarray, y: np.ndarray, w: np.ndarray, c: np.ndarray, p: int) -> float:
    """sum_j w_j [1/|x - y_j|]_p via the Gegenbauer (Legendre) form, term by term per source."""
    d = c - x
    h = y - c
    dd = d @ d
    dh = h @ d
    hh = np.einsum("ij,ij->i", h, h)
    total = np.zeros(y.shape[0])
    for m in range(0, p // 2 + 1):
        for q in range(0, p - 2 * m + 1):
            # t^q u^n = (-(d.h))^q |h|^(2m) / |d|^(2q + 2m) with n = q + 2m
            total += _gegenbauer_half_coef(q, m) * (-dh) ** q * hh ** m / dd ** (q + m)
    return float((w * total).sum() / np.sqrt(dd))


def _multi_indices(p: int):
    return [(a, b, n - a - b) for n in range(p + 1) for a in range(n, -1, -1) for b in range(n - a, -1, -1)]


def potential_series_recurrence(x: np.ndarray, y: np.ndarray, w: np.ndarray, c: np.ndarray, p: int) -> float:
    """sum_{|k| <= p} a_k(x - c) M_k with the Lindsay-Krasny recurrence for a_k."""
    R = x - c
    RR = R @ R
    a = {(0, 0, 0): 1.0 / np.sqrt(RR)}
    for k in _multi_indices(p)[1:]:
        n = sum(k)
        s1 = 0.0
        s2 = 0.0
        for i in range(3):
            km = list(k)
            km[i] -= 1
            if km[i] >= 0:
                s1 += R[i] * a[tuple(km)]
            km[i] -= 1
            if km[i] >= 0:
                s2 += a[tuple(km)]
        a[k] = ((2 * n - 1) * s1 - (n - 1) * s2) / (n * RR)
    h = y - c
    total = 0.0
    for k, ak in a.items():
        total += ak * (w * h[:, 0] ** k[0] * h[:, 1] ** k[1] * h[:, 2] ** k[2]).sum()
    return float(total)


def direct_potential_sum(x: np.ndarray, y: np.ndarray, w: np.ndarray) -> float:
    """sum_j w_j / |x - y_j| (without the 1/(4 pi) multiplier)."""
    return float((w / np.linalg.norm(y - x, axis=1)).sum())
