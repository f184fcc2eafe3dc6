"""FP64 numpy restatement of the order-selection MLP -- TEST INFRASTRUCTURE ONLY.

Same parameter layout as the library (W1[64][8] b1[64] W2[64][64] b2[64] W3[12][64] b3[12] mean[8]
inv_std[8]), exact-erf GELU, softmax cross-entropy averaged over the samples.  Used to check the CUDA
forward / backward / inference kernels.  The selector has no counterpart in the reference (whose
TreeSum uses one fixed Taylor order, src/LpmTreeSum.h), so this restatement is pinned by finite
differences of its own loss rather than by reference vectors.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

N_IN, N_H, N_OUT = 8, 64, 12
SIZES = [(N_H, N_IN), (N_H,), (N_H, N_H), (N_H,), (N_OUT, N_H), (N_OUT,)]
N_TRAINABLE = sum(int(np.prod(s)) for s in SIZES)
N_PARAMS = N_TRAINABLE + 2 * N_IN


def unpack(p: np.ndarray):
    out, o = [], 0
    for s in SIZES:
        k = int(np.prod(s))
        out.append(np.asarray(p[o:o + k], dtype=np.float64).reshape(s))
        o += k
    mean = np.asarray(p[o:o + N_IN], dtype=np.float64)
    inv_std = np.asarray(p[o + N_IN:o + 2 * N_IN], dtype=np.float64)
    return out, mean, inv_std


def gelu(a):
    return 0.5 * a * (1.0 + erf(a / np.sqrt(2.0)))


def gelu_grad(a):
    return 0.5 * (1.0 + erf(a / np.sqrt(2.0))) + a * np.exp(-0.5 * a * a) / np.sqrt(2.0 * np.pi)


def forward(p: np.ndarray, feats: np.ndarray):
    (w1, b1, w2, b2, w3, b3), mean, inv_std = unpack(p)
    x = (np.asarray(feats, np.float64) - mean) * inv_std
    a1 = x @ w1.T + b1
    h1 = gelu(a1)
    a2 = h1 @ w2.T + b2
    h2 = gelu(a2)
    z = h2 @ w3.T + b3
    return x, a1, h1, a2, h2, z


def loss_and_grad(p: np.ndarray, feats: np.ndarray, labels: np.ndarray):
    """Mean cross-entropy and its gradient with respect to the trainable parameters (flat)."""
    (w1, b1, w2, b2, w3, b3), _, _ = unpack(p)
    x, a1, h1, a2, h2, z = forward(p, feats)
    n = x.shape[0]
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    prob = e / e.sum(axis=1, keepdims=True)
    loss = -np.log(prob[np.arange(n), labels]).mean()
    dz = prob.copy()
    dz[np.arange(n), labels] -= 1.0
    dz /= n
    gw3 = dz.T @ h2
    gb3 = dz.sum(axis=0)
    da2 = (dz @ w3) * gelu_grad(a2)
    gw2 = da2.T @ h1
    gb2 = da2.sum(axis=0)
    da1 = (da2 @ w2) * gelu_grad(a1)
    gw1 = da1.T @ x
    gb1 = da1.sum(axis=0)
    g = np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3])
    return loss, g


def round_bf16(p: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    u = np.asarray(p, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def logits(p: np.ndarray, feats: np.ndarray) -> np.ndarray:
    return forward(p, feats)[-1]


def predict(p: np.ndarray, feats: np.ndarray) -> np.ndarray:
    return logits(p, feats).argmax(axis=1)


def predict_bf16(p: np.ndarray, feats: np.ndarray):
    """Classes of the BF16 inference path (BF16 weights; standardised inputs and hidden activations
    rounded to BF16 between layers; FP32-or-better accumulation) and the top-2 logit margin."""
    q = np.asarray(p, np.float32).copy()
    q[:N_TRAINABLE] = round_bf16(q[:N_TRAINABLE])
    (w1, b1, w2, b2, w3, b3), mean, inv_std = unpack(q)
    x = round_bf16(((np.asarray(feats, np.float32) - mean.astype(np.float32)) * inv_std.astype(np.float32)))
    h1 = round_bf16(gelu(x.astype(np.float64) @ w1.T + b1))
    h2 = round_bf16(gelu(h1.astype(np.float64) @ w2.T + b2))
    z = h2.astype(np.float64) @ w3.T + b3
    s = np.sort(z, axis=1)
    return z.argmax(axis=1), s[:, -1] - s[:, -2]
