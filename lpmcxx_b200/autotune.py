"""Autotuner for the treecode: picks the fastest (leaf size, acceptance theta, batch cell level, the fixed
order or the learned selector's per-pair budget and order bias, and the near-field tile shape) that meets a
relative L2 tolerance on a workload.

Accuracy is judged on a random sample of targets against the FP64 direct sum (the library's own
`lpm_direct_sum_dev`, which is parity-tested against the reference); time is the median of CUDA-event
timed evaluations on the GPU.  Candidates sharing a leaf size reuse one solver and switch the run-time
parameters (`TreeSum.set_param`), so a sweep costs one octree allocation per leaf size.

    best = autotune(ctx, L.biot_savart_kernel(), src, tgt, tol=1e-6, order_biases=(0, 2))
    solver = tuned_solver(best)            # an lpm_solver_desc for TreeSum / RK4
    # then set_param("batch_level", best.best.batch_level) and set_param("order_bias", best.best.bias),
    # set_param("near_targets", ...), set_param("near_tile", ...) and set_param("near_split", ...) from
    # best.best (apply_tuned does all of these)

The tile shape (targets per thread of the near-field kernel and sources staged per shared-memory tile)
changes no result, only the time, so it is searched last, on the fastest qualifying setting.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import (LPM_KERNEL_POISSON_3D, LPM_PREC_F32, LPM_PREC_F64, Context, KernelDesc, TreeSum, tree_solver)
from . import learned as _learned  # noqa: F401  (shipped selector weights)


@dataclass
class Candidate:
    max_per_leaf: int
    theta: float
    knob: float            # learned: per-pair budget eps; fixed: Taylor order
    batch_level: int | None = None
    bias: int = 0           # learned: orders added to every selector choice
    ms: float | None = None
    rel_err: float | None = None
    near_targets: int = 2   # near-field tile shape (run-time "near_targets", "near_tile", "near_split")
    near_tile: int = 512
    near_split: int = 1


@dataclass
class TuneResult:
    learned: bool
    kernel_kind: int
    best: Candidate | None
    tried: list = field(default_factory=list)

    def as_dict(self) -> dict:
        b = self.best
        return {"learned": self.learned, "max_per_leaf": b.max_per_leaf, "theta": b.theta,
                ("eps" if self.learned else "order"): b.knob, "batch_level": b.batch_level,
                "order_bias": b.bias, "ms": b.ms, "rel_err": b.rel_err, "near_targets": b.near_targets,
                "near_tile": b.near_tile, "near_split": b.near_split}


def default_grid(learned: bool, kernel_kind: int):
    thetas = (0.4, 0.5, 0.6, 0.7)
    leaves = (256, 512, 1024)
    if learned:
        knobs = (1e-8, 2e-8, 4e-8)
    elif kernel_kind == LPM_KERNEL_POISSON_3D:
        knobs = (4, 6, 8, 10)
    else:
        knobs = (8, 10, 11)
    return leaves, thetas, knobs


def _timed_eval(ctx, ts, src, tgt, out, reps):
    import torch

    ts.eval(src, tgt, out)  # sizes the interaction lists
    ms = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ts.eval(src, tgt, out)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.median(ms))


def autotune(ctx: Context, kernel: KernelDesc, src, tgt, tol: float, learned: bool = True, params=None,
             grid=None, batch_levels=(0, -1), sample: int = 4096, reps: int = 3, seed: int = 0,
             safety: float = 0.8, order_biases=(0,),
             tiles=tuple((t, s, g) for g in (1, 2) for t in (2, 4) for s in (256, 512, 1024)),
             also=()) -> TuneResult:
    """Sweep the grid on device-resident src (n_src, 4) / tgt (n_tgt, 4) float64 tensors.

    tol: relative L2 tolerance over the sampled targets (a candidate must reach safety * tol).
    learned: tune the learned selector's budget (Biot-Savart only) instead of the fixed order.
    batch_levels: offsets from each solver's default batch cell level to try (0 = default).
    order_biases: learned only, the selector order biases to try (set_param "order_bias").
    tiles: (near_targets, near_tile, near_split) shapes of the near-field kernel, tried on the best setting.
    also: further (src, tgt) workloads, no larger than the first, that the chosen setting must meet the tolerance
      on too (other states of the same problem: an ensemble's members, later time steps).  Time is judged on the
      first workload only; a candidate faster than the best so far is checked on every workload in `also`, and its
      rel_err is then the largest over all of them.
    """
    import torch

    kind = int(kernel.kind)
    if learned and kind == LPM_KERNEL_POISSON_3D:
        raise ValueError("the learned selector applies to the Biot-Savart kernel only")
    if learned and params is None:
        params, _ = _learned.load()
        if params is None:
            raise FileNotFoundError("no selector weights shipped; pass params")
    leaves, thetas, knobs = grid if grid is not None else default_grid(learned, kind)
    n_src, n_tgt = src.shape[0], tgt.shape[0]
    if any(s2.shape[0] > n_src or t2.shape[0] > n_tgt for s2, t2 in also):
        raise ValueError("autotune: a workload in `also` is larger than the first workload")
    comps = 1 if kind == LPM_KERNEL_POISSON_3D else 3
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(n_tgt, size=min(sample, n_tgt), replace=False))
    idx_t = torch.as_tensor(idx, device=tgt.device)
    ref = torch.empty((comps, idx.size), dtype=torch.float64, device=tgt.device)
    ctx.direct_sum_dev(kernel, LPM_PREC_F64, src, tgt[idx_t].contiguous(), ref)
    ref_norm = float(torch.linalg.norm(ref))
    out = torch.empty((comps, n_tgt), dtype=torch.float64, device=tgt.device)
    checks = []  # (src, tgt, sampled targets, FP64 reference, its norm, output buffer) of each further workload
    for k, (s2, t2) in enumerate(also):
        i2 = torch.as_tensor(np.sort(np.random.default_rng(seed + 1 + k).choice(
            t2.shape[0], size=min(sample, t2.shape[0]), replace=False)), device=t2.device)
        r2 = torch.empty((comps, i2.numel()), dtype=torch.float64, device=t2.device)
        ctx.direct_sum_dev(kernel, LPM_PREC_F64, s2, t2[i2].contiguous(), r2)
        o2 = torch.empty((comps, t2.shape[0]), dtype=torch.float64, device=t2.device)
        checks.append((s2, t2, i2, r2, float(torch.linalg.norm(r2)), o2))

    def worst_error(ts, err):
        """err on the first workload, raised to the largest error over the `also` workloads (stops early once one
        misses the tolerance)."""
        for s2, t2, i2, r2, n2, o2 in checks:
            if err > safety * tol:
                break
            ts.eval(s2, t2, o2)
            err = max(err, float(torch.linalg.norm(o2[:, i2] - r2)) / n2)
        return err

    res = TuneResult(learned=learned, kernel_kind=kind, best=None)
    for leaf in leaves:
        base_knob = 10 if learned else int(knobs[0])
        ts = TreeSum(ctx, kernel, tree_solver(LPM_PREC_F32, base_knob, leaf, thetas[0], learned=learned),
                     n_src, n_tgt)
        try:
            if learned:
                ts.set_mlp(params)
            level0 = None
            for knob in knobs:
                if not learned and int(knob) != base_knob:
                    ts.close()
                    ts = TreeSum(ctx, kernel, tree_solver(LPM_PREC_F32, int(knob), leaf, thetas[0]), n_src, n_tgt)
                    base_knob = int(knob)
                for theta, bias in [(t, b) for t in thetas for b in (order_biases if learned else (0,))]:
                    ts.set_param("theta", theta)
                    if learned:
                        ts.set_param("eps", knob)
                        ts.set_param("order_bias", bias)
                    for off in batch_levels:
                        if level0 is None:
                            level0 = int(ts.get_param("batch_level"))
                        lvl = level0 + off
                        if lvl < 1:
                            continue
                        ts.set_param("batch_level", lvl)
                        ms = _timed_eval(ctx, ts, src, tgt, out, reps)
                        err = float(torch.linalg.norm(out[:, idx_t] - ref)) / ref_norm
                        if checks and err <= safety * tol and (res.best is None or ms < res.best.ms):
                            err = worst_error(ts, err)
                        c = Candidate(leaf, theta, knob, lvl, bias, ms, err, int(ts.get_param("near_targets")),
                                      int(ts.get_param("near_tile")), int(ts.get_param("near_split")))
                        res.tried.append(c)
                        if err <= safety * tol and (res.best is None or ms < res.best.ms):
                            res.best = c
                    ts.set_param("batch_level", level0)
        finally:
            ts.close()
    if res.best is not None and tiles:
        b = res.best
        ts = TreeSum(ctx, kernel, tree_solver(LPM_PREC_F32, 10 if learned else int(b.knob), b.max_per_leaf, b.theta,
                                              learned=learned, tolerance=b.knob if learned else 0.0), n_src, n_tgt)
        try:
            if learned:
                ts.set_mlp(params)
                ts.set_param("order_bias", b.bias)
            ts.set_param("batch_level", b.batch_level)
            for nt, tile, split in tiles:
                ts.set_param("near_targets", nt)
                ts.set_param("near_tile", tile)
                ts.set_param("near_split", split)
                ms = _timed_eval(ctx, ts, src, tgt, out, reps)
                err = float(torch.linalg.norm(out[:, idx_t] - ref)) / ref_norm
                if checks and err <= safety * tol and ms < res.best.ms:
                    err = worst_error(ts, err)
                c = Candidate(b.max_per_leaf, b.theta, b.knob, b.batch_level, b.bias, ms, err, nt, tile, split)
                res.tried.append(c)
                if err <= safety * tol and ms < res.best.ms:
                    res.best = c
        finally:
            ts.close()
    return res


def tuned_solver(result: TuneResult, precision: int = LPM_PREC_F32):
    """lpm_solver_desc of the tuned setting (the batch level, the order bias and the near-field tile shape
    are run-time parameters: apply them with set_param("batch_level", ...), set_param("order_bias", ...),
    set_param("near_targets", ...), set_param("near_tile", ...) and set_param("near_split", ...) on the
    TreeSum / RK4 made from this descriptor; apply_tuned does all of them)."""
    b = result.best
    if b is None:
        raise ValueError("no candidate met the tolerance")
    if result.learned:
        return tree_solver(precision, 10, b.max_per_leaf, b.theta, learned=True, tolerance=b.knob)
    return tree_solver(precision, int(b.knob), b.max_per_leaf, b.theta)


def autotune_direct(ctx: Context, kernel: KernelDesc, src, tgt, shapes=(2, 4, 8), reps: int = 3,
                    n_coincident: int = 0) -> dict:
    """Tile shape of the FP32 direct sum (targets per thread, the context's "direct_targets"): every shape timed
    on device-resident src / tgt (median of `reps` CUDA-event timed sums after one warm-up); the fastest is set on
    the context and returned with the timings and the largest relative deviation between the shapes' sums."""
    import torch

    comps = 1 if int(kernel.kind) == LPM_KERNEL_POISSON_3D else 3
    out = torch.empty((comps, tgt.shape[0]), dtype=torch.float64, device=tgt.device)
    ms, sums = {}, {}
    for t in shapes:
        ctx.set_param("direct_targets", t)
        ctx.direct_sum_dev(kernel, LPM_PREC_F32, src, tgt, out, n_coincident=n_coincident)
        times = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.direct_sum_dev(kernel, LPM_PREC_F32, src, tgt, out, n_coincident=n_coincident)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms[t] = float(np.median(times))
        sums[t] = out.clone()
    best = min(ms, key=ms.get)
    ctx.set_param("direct_targets", best)
    ref = sums[best]
    dev = max(float(torch.linalg.norm(v - ref) / torch.linalg.norm(ref)) for v in sums.values())
    return {"direct_targets": best, "ms": ms, "max_rel_deviation": dev}


def apply_tuned(result: TuneResult, solver) -> None:
    """Set the tuned run-time parameters on a TreeSum or RK4 made from tuned_solver(result)."""
    b = result.best
    solver.set_param("batch_level", b.batch_level)
    if result.learned:
        solver.set_param("order_bias", b.bias)
    solver.set_param("near_targets", b.near_targets)
    solver.set_param("near_tile", b.near_tile)
    solver.set_param("near_split", b.near_split)


__all__ = ["autotune", "autotune_direct", "tuned_solver", "apply_tuned", "TuneResult", "Candidate", "default_grid", "LPM_PREC_F64"]
