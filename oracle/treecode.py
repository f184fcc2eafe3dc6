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
