"""Learned Taylor-order selection: training data, training and the shipped selector weights.

The learned treecode accepts (target batch, cluster) pairs by the usual criterion and asks a small MLP
(8 -> 64 -> 64 -> 12, GELU; BF16 weights, FP32 accumulation) for the smallest order 1..11 whose error
stays within a per-pair budget eps * |mult| * sum|w|, or for "none", in which case the cluster is opened
(a leaf or a small cluster is summed directly).  The labels come from the treecode and the FP64 direct
sum themselves (`TreeSum.sample_labels`): for each sampled pair the cluster's exact FP64 contribution at
the batch's targets is compared with its expansion at every order.  Training runs in the library's CUDA
kernels (`mlp_train`); without weights the fixed order is the fallback.

Training set: `n_fields` seeded Gaussian vortex fields (4 pi exp(-16 |x - x0|^2) about a seeded random
centre, minus its mean) on the icosahedral level-8 mesh, `pairs_per_field` labelled pairs each; the
fields cycle through several budgets and acceptance parameters so that both can be chosen at run time.

    python -m lpmcxx_b200.learned --out lpmcxx_b200/data/order_mlp.npz     # needs a GPU
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import (LPM_PREC_F32, Context, TreeSum, biot_savart_kernel, build_mesh, mlp_init, mlp_predict, mlp_train,
               tree_solver)
from .workloads import gaussian_vortex, particles

DATA = Path(__file__).resolve().parent / "data"
DEFAULT_WEIGHTS = DATA / "order_mlp.npz"
DEFAULT_EPS = 2e-8  # per-pair error budget relative to |mult| * sum|w|
TRAIN_EPS = (5e-9, 1e-8, 2e-8, 5e-8, 1e-7)  # field k uses TRAIN_EPS[k % 5]
TRAIN_THETA = (0.5, 0.6, 0.7)               # and TRAIN_THETA[k % 3]
TRAIN_LEAF = 512


def random_unit(rng) -> np.ndarray:
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def seeded_vortex_particles(mesh, seed: int):
    """(particles (n, 4), n_src) of a Gaussian vortex about a seeded random centre, minus its mean."""
    rng = np.random.default_rng(1000 + seed)
    zeta = gaussian_vortex(mesh.face_xyz, random_unit(rng))
    leaf = mesh.leaf
    zeta = zeta - (zeta[leaf] * mesh.face_area[leaf]).sum() / mesh.face_area[leaf].sum()
    return particles(mesh, zeta)


def make_training_set(ctx: Context, n_fields: int = 20, level: int = 8, pairs_per_field: int = 25_000,
                      eps=TRAIN_EPS, theta=TRAIN_THETA, max_per_leaf: int = TRAIN_LEAF, with_errors: bool = False,
                      seeds=None):
    """(features (N, 8), labels (N,), errors (N, 11) or None) from `n_fields` seeded fields."""
    import torch

    eps_list = tuple(np.atleast_1d(eps).tolist())
    theta_list = tuple(np.atleast_1d(theta).tolist())
    ctx.use_torch_stream()
    mesh = build_mesh("icos", level)
    feats, labels, errs = [], [], []
    for k, seed in enumerate(range(n_fields) if seeds is None else seeds):
        p, n_src = seeded_vortex_particles(mesh, seed)
        d = torch.tensor(p, device="cuda")
        solver = tree_solver(LPM_PREC_F32, 8, max_per_leaf, theta_list[k % len(theta_list)], learned=True,
                             tolerance=eps_list[k % len(eps_list)])
        ts = TreeSum(ctx, biot_savart_kernel(), solver, n_src, p.shape[0])
        try:
            f, lab, e = ts.sample_labels(d[:n_src], d, 0, pairs_per_field, with_errors)
        finally:
            ts.close()
        feats.append(f)
        labels.append(lab)
        if e is not None:
            errs.append(e)
    return np.concatenate(feats), np.concatenate(labels), (np.concatenate(errs) if errs else None)


def train(ctx: Context, feats, labels, epochs: int = 40, lr: float = 2e-3, seed: int = 0):
    """(params, per-epoch loss) of a selector trained from a fresh initialisation."""
    params = mlp_init(feats, seed)
    loss = mlp_train(ctx, feats, labels, params, epochs=epochs, minibatch=512, lr=lr, seed=seed)
    return params, loss


def save(path: Path, params, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=np.asarray(params, np.float32), meta=json.dumps(meta))


def load(path: Path = DEFAULT_WEIGHTS):
    """(params, meta) of a saved selector, or (None, None) when the file does not exist."""
    path = Path(path)
    if not path.exists():
        return None, None
    with np.load(path) as z:
        return z["params"].astype(np.float32), json.loads(str(z["meta"]))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=DEFAULT_WEIGHTS)
    ap.add_argument("--fields", type=int, default=20)
    ap.add_argument("--pairs", type=int, default=25_000)
    ap.add_argument("--level", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--save-set", type=Path, default=None, help="also save the labelled pairs (npz)")
    args = ap.parse_args()
    ctx = Context(0)
    t0 = time.time()
    f, lab, err = make_training_set(ctx, args.fields, args.level, args.pairs, with_errors=args.save_set is not None)
    t1 = time.time()
    # the last field's pairs are held out for validation
    n_val = int((lab.shape[0] // max(args.fields, 1))) if args.fields > 1 else 0
    params, loss = train(ctx, f[:-n_val] if n_val else f, lab[:-n_val] if n_val else lab, args.epochs)
    t2 = time.time()
    meta = {"fields": args.fields, "pairs": int(f.shape[0]), "level": args.level, "eps": list(TRAIN_EPS),
            "theta": list(TRAIN_THETA), "max_per_leaf": TRAIN_LEAF, "epochs": args.epochs,
            "loss_first_last": [float(loss[0]), float(loss[-1])] if len(loss) else None,
            "label_histogram": np.bincount(lab, minlength=12).tolist(),
            "seconds_labels": round(t1 - t0, 2), "seconds_train": round(t2 - t1, 2)}
    if n_val:
        pred = mlp_predict(ctx, params, f[-n_val:])
        meta["val_pairs"] = n_val
        meta["val_accuracy"] = float((pred == lab[-n_val:]).mean())
        meta["val_under_predicted"] = float((pred < lab[-n_val:]).mean())
    save(args.out, params, meta)
    if args.save_set is not None:
        np.savez_compressed(args.save_set, feats=f, labels=lab, errs=err)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
