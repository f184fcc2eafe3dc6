"""Benchmark: Biot-Savart RK4 steps/s on the icos level-8 Gaussian-vortex workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lpm|reference] [--solver ...]

Workload (synthetic, generated here): icosahedral triangle mesh refined 8 levels -- 1,310,720 face
centroid particles carrying vorticity x area (sources) plus 655,362 vertex particles, 1,966,082
targets -- with zeta = 4 pi exp(-16|x - x0|^2) minus its area-weighted mean, x0 at (lat 0.05,
lon 3 pi/4); RK4 steps of dt = 0.005.  One "step" is one full RK4 step (four velocity evaluations
plus the FP64 updates) of the whole particle set.

Our arm (--impl lpm) runs the headline solver, times K steps with CUDA events on the launching
stream (L2 flushed between steps, outside the timed events), reports the FP64 GPU direct-sum RK4
rate of the same workload beside it, the relative L2 velocity error of the headline solver against
the FP64 direct sum, the dominant kernel's roofline, an end-to-end rate through the host API, the
clocks seen during the timed region and a CPU baseline of the reference's own DirectSum.  Under
torchrun every rank runs an independent replica (the path has no exchange step): value = all
ranks' steps / max-over-ranks time.

The reference arm (--impl reference) times the reference's own CPU DirectSum::meshSolve
(oracle/_ref, built from the reference sources; the oracle's C port where that build is absent) on
the host cores, each step a bounded target slice, extrapolated to full RK4 steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

LEVEL = 8
DT = 0.005
METRIC = "Biot-Savart RK4 steps/s @1.3M pts: FP32 learned tree vs FP64 direct @relL2≤1e-6"
WORKLOAD = ("icos L8 Gaussian vortex: 1,310,720 face-centroid sources + 655,362 vertices "
            "(1,966,082 targets), RK4 dt=0.005")


def workload_name(level: int, n_src: int, n_tgt: int, dt: float) -> str:
    return (f"icos L{level} Gaussian vortex: {n_src:,} face-centroid sources + {n_tgt - n_src:,} vertices "
            f"({n_tgt:,} targets), RK4 dt={dt:g}")
FLOPS_PER_BS_PAIR = 17


def env_int(name: str, default: int) -> int:
    v = os.environ.get(name)
    return int(v) if v not in (None, "") else default


def replica_rate(total_ms: float, steps: int, device: str = "cuda") -> tuple:
    """Replicas (every rank runs its own copy of the workload, no data exchanged): the slowest rank's timed
    milliseconds (max over ranks) and the whole job's steps/s, world x steps over that time."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, world * steps / (total_ms * 1e-3)


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------- CPU baselines
def reference_harness() -> Path | None:
    p = ROOT / "oracle" / "_ref" / "ref_harness"
    return p if p.exists() else None


def time_reference_direct(reps: int, procs: int, targets_per_proc: int = 3, kind: str = "icos",
                          level: int = LEVEL) -> dict:
    """The reference's DirectSum::meshSolve on a `kind` level-`level` mesh (Gaussian vortex), `procs` processes
    each timing a MPIReplicatedData slice of ~targets_per_proc vertex targets, `reps` times.  Returns per-rep
    pair rates."""
    exe = reference_harness()
    n_verts = 2 + (10 if kind == "icos" else 6) * 4 ** level
    size = max(procs, n_verts // targets_per_proc)
    env = dict(os.environ)
    env["LPM_MESH_SEED_DIR"] = str(ROOT / "oracle" / "_ref" / "meshSeeds")
    env["LPM_STUB_SIZE"] = str(size)
    jobs = []
    for r in range(procs):
        e = dict(env)
        e["LPM_STUB_RANK"] = str(r)
        jobs.append(subprocess.Popen([str(exe), "time_direct", kind, str(level), "gauss", str(reps)],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=e))
    results = []
    for j in jobs:
        out, _ = j.communicate()
        line = [ln for ln in out.splitlines() if ln.startswith('{"cmd"')]
        if j.returncode != 0 or not line:
            raise RuntimeError("reference harness failed")
        results.append(json.loads(line[-1]))
    n_src = results[0]["n_leaves"]
    n_tgt = results[0]["n_verts"] + n_src
    pairs = sum((r["vert_targets"] + r["face_targets"]) * n_src for r in results)
    rep_s = [max(r["seconds"][k] for r in results) for k in range(reps)]
    return {"rep_seconds": rep_s, "pairs_per_rep": pairs, "n_src": n_src, "n_tgt": n_tgt,
            "targets_per_rep": sum(r["vert_targets"] + r["face_targets"] for r in results), "procs": procs}


def time_reference_poisson(reps: int, procs: int, n: int, targets_per_proc: int = 4) -> dict:
    """The reference's DirectSum::meshfreeSolve with the 1/(4 pi r) kernel on the n-point cube: `procs`
    processes each timing a MPIReplicatedData slice of ~targets_per_proc targets, `reps` times."""
    exe = reference_harness()
    size = max(procs, n // targets_per_proc)
    jobs = []
    for r in range(procs):
        e = dict(os.environ, LPM_STUB_RANK=str(r), LPM_STUB_SIZE=str(size))
        jobs.append(subprocess.Popen([str(exe), "time_poisson", str(n), "0x2B", str(reps)], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True, env=e))
    results = []
    for j in jobs:
        out, _ = j.communicate()
        line = [ln for ln in out.splitlines() if ln.startswith('{"cmd"')]
        if j.returncode != 0 or not line:
            raise RuntimeError("reference harness failed")
        results.append(json.loads(line[-1]))
    pairs = sum(r["targets"] * r["sources"] for r in results)
    rep_s = [max(r["seconds"][k] for r in results) for k in range(reps)]
    return {"rep_seconds": rep_s, "pairs_per_rep": pairs, "targets_per_rep": sum(r["targets"] for r in results)}


def poisson_cpu_baseline(n: int, reps: int = 2) -> dict | None:
    """evaluations/s of the reference's own FP64 meshfree direct sum on the host cores (bounded target
    slice, extrapolated to all n targets); None without the reference build."""
    if reference_harness() is None:
        return None
    procs = max(1, min(os.cpu_count() or 1, 32))
    r = time_reference_poisson(reps, procs, n)
    pps = float(np.median([r["pairs_per_rep"] / t for t in r["rep_seconds"]]))
    return {"value": pps / (float(n) * float(n)), "unit": "evaluations/s", "cores": procs, "kind": "reference",
            "sample": f"reference DirectSum::meshfreeSolve (FP64, 1/(4 pi r) ScalarKernel), {procs} processes x "
                      f"MPIReplicatedData slice, {r['targets_per_rep']} targets x {n} sources per repetition, "
                      f"extrapolated to {n} targets", "pairs_per_s": pps}


def time_oracle_port(reps: int, threads: int, n_targets: int = 64) -> dict:
    """The oracle's C restatement of the same FP64 direct sum on a slice of n_targets targets."""
    import oracle
    import lpmcxx_b200.workloads as W

    os.environ["ORACLE_THREADS"] = str(threads)
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", LEVEL)
    src = p[:n_src]
    tgt = p[n_src:n_src + n_targets]
    rep_s = []
    for _ in range(reps):
        t0 = time.perf_counter()
        oracle.bs_direct(src, tgt)
        rep_s.append(time.perf_counter() - t0)
    return {"rep_seconds": rep_s, "pairs_per_rep": n_targets * n_src, "n_src": n_src, "n_tgt": p.shape[0],
            "targets_per_rep": n_targets, "procs": threads}


def cpu_baseline(reps: int) -> dict:
    cores = os.cpu_count() or 1
    procs = max(1, min(cores, 32))
    if reference_harness() is not None:
        r = time_reference_direct(reps, procs)
        kind = "reference"
        sample = (f"reference DirectSum::meshSolve (FP64), {procs} processes x MPIReplicatedData slice, "
                  f"{r['targets_per_rep']} vertex targets x {r['n_src']} sources per step, extrapolated")
    else:
        r = time_oracle_port(reps, procs)
        kind = "port"
        sample = (f"oracle C port of the FP64 direct sum, {procs} threads, {r['targets_per_rep']} targets x "
                  f"{r['n_src']} sources per step, extrapolated")
    pairs_full_step = 4.0 * r["n_tgt"] * r["n_src"]
    rates = [r["pairs_per_rep"] / s for s in r["rep_seconds"]]
    steps_per_s = float(np.median(rates)) / pairs_full_step
    return {"value": steps_per_s, "unit": "steps/s", "cores": procs, "kind": kind, "sample": sample,
            "pairs_per_s": float(np.median(rates)), "rep_seconds": r["rep_seconds"]}


# --------------------------------------------------------------------------- GPU arm
def profile_summary_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/), if present."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for ln in f.read_text().splitlines():
            if ln.startswith("traffic_bytes_per_launch") and f"[{kernel}]" in ln:
                try:
                    return float(ln.split(":", 1)[1].split()[0])
                except ValueError:
                    pass
    return None


# (order, theta, max_per_leaf) of the treecodes: "tree_f32" is the fastest fixed setting measured to reach
# relative L2 <= 1e-6 against the FP64 direct sum on this workload; "tree_cfg2a" is the p=8, theta=0.7,
# 512-per-leaf configuration (whose error is ~1e-4); "tree_learned" picks the order per pair with the
# shipped selector (order 10 is its fallback) under the per-pair budget LEARNED_EPS, each chosen order raised
# by LEARNED_ORDER_BIAS, target batches cut at one octree level coarser than the solver's default
# (LEARNED_BATCH_LEVEL_OFFSET): the autotuner at icos L8 (leaf 384/512/768 x theta 0.45..0.55 x budget
# 3e-7..8e-7 x bias 2, 3 x batch level default, default - 1; 8192 sampled targets against the FP64 direct sum)
# gave the fastest 512-per-leaf setting within 0.8 x 1e-6 at theta 0.55, budget 5e-7, bias 2, batch level
# default - 1 (13.5 ms per evaluation, rel L2 5.8e-7, against 14.2 ms for theta 0.5 at the default level).
TREE_SETTINGS = {"tree_f32": (10, 0.5, 256), "tree_cfg2a": (8, 0.7, 512), "tree_learned": (10, 0.55, 512)}
LEARNED_EPS = 5e-7
LEARNED_ORDER_BIAS = 2
LEARNED_BATCH_LEVEL_OFFSET = -1


def solver_desc(name: str):
    import lpmcxx_b200 as L

    if name == "direct_f64":
        return L.direct_solver(L.LPM_PREC_F64)
    if name == "direct_f32":
        return L.direct_solver(L.LPM_PREC_F32)
    if name in TREE_SETTINGS:
        p, theta, leaf = TREE_SETTINGS[name]
        learned = name == "tree_learned"
        return L.tree_solver(L.LPM_PREC_F32, order=p, max_per_leaf=leaf, theta=theta, learned=learned,
                             tolerance=LEARNED_EPS if learned else 0.0)
    raise ValueError(name)


def far_entries(p: int) -> int:
    """Coefficients of the order-p far-field expansion (multi-indices k, m with |k| + 2m < p)."""
    return sum((q * (q + 1) * (q + 2)) // 6 for q in range(p, 0, -2))


def kernel_work(kernel: str, n_src: int, n_tgt: int, stats: dict | None, order: int) -> tuple[float, str] | None:
    """Algorithmic flops of one launch of `kernel`: 17 per Biot-Savart pair (direct and near field), 8 per
    far-field expansion coefficient plus FLOPS_PER_FAR_EVAL per (target, cluster) evaluation."""
    if kernel in ("bs_f32_kernel", "bs_f64_kernel"):
        return FLOPS_PER_BS_PAIR * float(n_src) * float(n_tgt), "TFLOP/s"
    if kernel == "near_kernel" and stats:
        return FLOPS_PER_BS_PAIR * float(stats["near_pairs"]), "TFLOP/s"
    if kernel == "far_kernel" and stats:
        # 4 coefficient FMAs (8 flops) per expansion coefficient + the per-evaluation setup and fold
        return 8.0 * float(stats["far_terms"]) + FLOPS_PER_FAR_EVAL * float(stats["far_evals"]), "TFLOP/s"
    return None


# Per (target, cluster) evaluation outside the Horner scheme: d = c - x (3), |d|^2 (5), 1/|d|^2 (1), the
# scaled offsets e = d/|d|^2 (3) and the folded sum h += (d g0 + g)/|d|^2 (12).
FLOPS_PER_FAR_EVAL = 24.0


POISSON_METRIC = "3D Poisson 1/(4 pi r) treecode evaluations/s @1,048,576 pts (p=6, theta=0.6) vs FP64 direct"
POISSON_SETTINGS = (6, 0.6, 256)  # order (|k| <= p), theta, max per leaf
FLOPS_PER_POISSON_PAIR = 11


def run_gpu_poisson(args) -> None:
    """The 3D Poisson configuration: one treecode evaluation of the potential of n points in [-1, 1]^3
    with charges U(-1, 1) per step (targets = sources, self pairs excluded)."""
    import torch

    import lpmcxx_b200 as L
    import lpmcxx_b200.workloads as W

    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    n = args.points
    pts = W.poisson_cube(n)
    ctx = L.Context(local)
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    kern = L.poisson_kernel()
    order, theta, leaf = POISSON_SETTINGS
    with torch.cuda.stream(stream):
        ctx.use_torch_stream()
        d = torch.tensor(pts, device="cuda")
        out = torch.empty((1, n), dtype=torch.float64, device="cuda")
        ts = L.TreeSum(ctx, kern, L.tree_solver(L.LPM_PREC_F32, order, leaf, theta), n, n)
        for _ in range(args.warmup):
            ts.eval(d, d, out)
        stream.synchronize()
        launches0 = ctx.launch_count
        clocks = ClockSampler(local).start()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ts.eval(d, d, out)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        clk = clocks.stop()
        launches = ctx.launch_count - launches0
        value = world * args.steps / (sum(ms) * 1e-3)
        # end to end: pinned host points in, potentials out
        host_in = torch.tensor(pts).pin_memory()
        host_out = torch.empty((1, n), dtype=torch.float64).pin_memory()
        e2e_s = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            d.copy_(host_in, non_blocking=True)
            ts.eval(d, d, out)
            host_out.copy_(out, non_blocking=True)
            stream.synchronize()
            e2e_s.append(time.perf_counter() - t0)
        ctx.set_profiling(True)
        ts.eval(d, d, out)
        prof = ctx.profile_report()
        ctx.set_profiling(False)
        st = ts.stats()
        ts.close()
        ref = torch.empty((1, n), dtype=torch.float64, device="cuda")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.direct_sum_dev(kern, L.LPM_PREC_F64, d, d, ref)
        e1.record(stream)
        e1.synchronize()
        direct_ms = e0.elapsed_time(e1)
        rel = float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref))
        fp32_peak = ctx.fma_peak_tflops(L.LPM_PREC_F32)
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
    name, pk = dom
    if name == "near_kernel":
        work = FLOPS_PER_POISSON_PAIR * float(st["near_pairs"])
    elif name == "far_kernel":
        work = 2.0 * float(st["far_terms"]) + 12.0 * float(st["far_evals"])
    else:
        work = None
    roof = None
    if work is not None:
        achieved = work / (pk["ms"] * 1e-3) * 1e-12
        roof = {"bound": "fp32", "kernel": name, "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": "measured FMA microbenchmark (lpm_fma_peak) on this GPU",
                "evaluation_ms": pk["ms"], "share": pk["ms"] / sum(v["ms"] for v in prof.values())}
    out_line = {
        "metric": POISSON_METRIC, "value": value, "unit": "evaluations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"{n:,} points uniform in [-1,1]^3, charges U(-1,1), splitmix64 seed 0x2B",
                   "solver": f"Poisson treecode p={order} (|k|<=p), theta={theta}, {leaf} per leaf",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "rel_l2_vs_fp64_direct": rel, "fp64_direct_ms": direct_ms,
        "speedup_vs_fp64_direct": direct_ms / float(np.mean(ms)),
        "roofline": roof, "kernel_profile_ms": dict(sorted(prof.items(), key=lambda kv: -kv[1]["ms"])[:8]),
        "tree_stats": st,
        "e2e": {"value": world * args.steps / sum(e2e_s), "unit": "evaluations/s",
                "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * 8},
        "gpu_launches": launches, "clocks": clk,
    }
    if roof is not None:
        roof["traffic"] = profile_summary_traffic(f"poisson_{name}")
    if env_int("RANK", 0) == 0 and world == 1 and not args.no_cpu_baseline:
        out_line["cpu_baseline"] = poisson_cpu_baseline(n)
    print(json.dumps(out_line))


CUBE_METRIC = "direct-sum RK4 steps/s, cubed sphere L8 (393,216 sources), FP32 (FP64-accumulated) and FP64"


def run_gpu_direct_cube(args) -> None:
    """The at-scale direct-sum configuration: cubed sphere refined 8 levels (393,216 face sources + 393,218
    vertices), Gaussian vortex, RK4 steps of dt = 0.005 by the FP32 direct sum (the line's value) and the FP64
    one; K timed steps each after the warm-up, then the two trajectories compared."""
    import torch

    import lpmcxx_b200 as L
    import lpmcxx_b200.workloads as W

    local = env_int("LOCAL_RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    torch.cuda.set_device(local)
    _, p, n_src = W.gaussian_vortex_mesh("cube", 8)
    n = p.shape[0]
    ctx = L.Context(local)
    stream = torch.cuda.Stream()
    kern = L.biot_savart_kernel()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    res = {}
    with torch.cuda.stream(stream):
        ctx.use_torch_stream()
        state0 = torch.tensor(p, device="cuda")
        from lpmcxx_b200.autotune import autotune_direct

        tile = autotune_direct(ctx, kern, state0[:n_src], state0, n_coincident=n_src)
        for prec in (L.LPM_PREC_F32, L.LPM_PREC_F64):
            rk = L.RK4(ctx, kern, L.direct_solver(prec), n_src, n)
            rk.set_state(state0)
            rk.step(0.005, args.warmup, use_graph=True)
            rk.set_state(state0)
            rk.step(0.005, 1, use_graph=True)
            rk.set_state(state0)
            torch.cuda.synchronize()
            launches0 = ctx.launch_count
            ms = []
            clocks = ClockSampler(local).start() if prec == L.LPM_PREC_F32 else None
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rk.step(0.005, 1, use_graph=True)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            clk = clocks.stop() if clocks else None
            final = rk.get_state()
            ctx.set_profiling(True)
            u = torch.empty((3, n), dtype=torch.float64, device="cuda")
            rk.velocity(u)
            prof = ctx.profile_report()
            ctx.set_profiling(False)
            res[prec] = {"ms": ms, "final": final, "prof": prof, "clk": clk, "launches": ctx.launch_count - launches0}
            if prec == L.LPM_PREC_F32:  # end to end through the host API: pinned state in, one step, state out
                host_in = torch.tensor(p).pin_memory()
                host_out = torch.empty_like(host_in).pin_memory()
                e2e_s = []
                for _ in range(min(args.steps, 3)):
                    t0 = time.perf_counter()
                    rk.set_state(host_in)
                    rk.step(0.005, 1, use_graph=True)
                    rk.get_state(host_out)
                    e2e_s.append(time.perf_counter() - t0)
            rk.close()
        fp32_peak = ctx.fma_peak_tflops(L.LPM_PREC_F32)
        fp64_peak = ctx.fma_peak_tflops(L.LPM_PREC_F64)
    r32, r64 = res[L.LPM_PREC_F32], res[L.LPM_PREC_F64]
    d32 = r32["final"][:, :3] - p[:, :3]
    d64 = r64["final"][:, :3] - p[:, :3]
    pairs = float(n_src) * float(n)
    k32 = r32["prof"]["bs_f32_kernel"]["ms"]
    k64 = r64["prof"]["bs_f64_kernel"]["ms"]
    value = world * args.steps / (sum(r32["ms"]) * 1e-3)
    tf32 = FLOPS_PER_BS_PAIR * pairs / (k32 * 1e-3) * 1e-12
    out = {
        "metric": CUBE_METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(r32["ms"])), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"cube L8 Gaussian vortex: {n_src:,} face-centroid sources + {n - n_src:,} vertices, "
                               "RK4 dt=0.005", "solver": "FP32 direct sum, FP64 accumulation across tiles",
                   "direct_targets": tile["direct_targets"], "tile_ms": tile["ms"],
                   "l2": "flushed (256 MiB write) before every timed step", "graph": "one CUDA graph replay per step"},
        "fp64_direct_steps_per_s": world * args.steps / (sum(r64["ms"]) * 1e-3),
        "rel_displacement_fp32_vs_fp64": float(np.linalg.norm(d32 - d64) / np.linalg.norm(d64)),
        "displacement_steps": args.warmup + 1 + args.steps,
        "roofline": {"bound": "fp32", "kernel": "bs_f32_kernel", "achieved": tf32, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": tf32 / fp32_peak, "traffic": profile_summary_traffic("bs_f32_kernel"),
                     "peak_source": "measured FMA microbenchmark (lpm_fma_peak) on this GPU"},
        "fp64_kernel": {"kernel": "bs_f64_kernel", "tflops": FLOPS_PER_BS_PAIR * pairs / (k64 * 1e-3) * 1e-12,
                        "peak_tflops": fp64_peak},
        "e2e": {"value": world / float(np.mean(e2e_s)), "unit": "steps/s", "h2d_bytes_per_step": n * 32,
                "d2h_bytes_per_step": n * 32},
        "gpu_launches": r32["launches"], "clocks": r32["clk"],
    }
    if env_int("RANK", 0) == 0 and world == 1 and not args.no_cpu_baseline and reference_harness() is not None:
        procs = max(1, min(os.cpu_count() or 1, 32))
        r = time_reference_direct(2, procs, kind="cube", level=8)
        pps = float(np.median([r["pairs_per_rep"] / t for t in r["rep_seconds"]]))
        out["cpu_baseline"] = {"value": pps / (4.0 * pairs), "unit": "steps/s", "cores": procs, "kind": "reference",
                               "sample": f"reference DirectSum::meshSolve (FP64), {procs} processes x "
                                         f"MPIReplicatedData slice, {r['targets_per_rep']} targets x {r['n_src']} "
                                         "sources per repetition, extrapolated to 4 evaluations of all targets",
                               "pairs_per_s": pps}
    print(json.dumps(out))


ENSEMBLE_METRIC = "ensemble RK4 steps/s: 64 instances (icos L5/L6/L7/L8 x 16, 27.85M sources), learned treecode"
ENSEMBLE_TUNE_GRID = ((128, 256, 512), (0.4, 0.5, 0.6), (2e-7, 5e-7))  # leaf sizes, theta, learned budgets
# seeded targets per instance on which the tuner and the reported errors compare with the FP64 direct sum: the
# error concentrates near each vortex core, so the relative L2 over 4096 targets varied up to twofold between
# samples of the same field
ENSEMBLE_SAMPLE = 32768


def ensemble_tune(ctx, kern, inst, tol: float = 1e-6) -> dict:
    """Per size class (icos level): the autotuner (learned selector, order bias 2, leaf x theta x budget x batch
    level, then the near tile shape) timed on the class's first instance; the chosen setting meets the tolerance
    (with the tuner's 0.8 safety factor) on ENSEMBLE_SAMPLE sampled targets of every instance of the class against
    the FP64 direct sum, since the instances carry different vortices."""
    import torch

    from lpmcxx_b200.autotune import autotune

    tuned = {}
    for level in sorted({lvl for lvl, _, _ in inst}):
        members = [torch.tensor(p, device="cuda") for lvl, p, _ in inst if lvl == level]
        n_src = next(n for lvl, _, n in inst if lvl == level)
        d = members[0]
        res = autotune(ctx, kern, d[:n_src], d, tol=tol, learned=True, grid=ENSEMBLE_TUNE_GRID,
                       batch_levels=(0, -1), order_biases=(2,), sample=ENSEMBLE_SAMPLE, reps=2,
                       also=[(m[:n_src], m) for m in members[1:]])
        if res.best is None:
            raise RuntimeError(f"ensemble tuning: no candidate meets {tol} at icos L{level}")
        tuned[level] = res.as_dict()
        tuned[level]["candidates"] = len(res.tried)
    return tuned


ENSEMBLE_EPS_LADDER = (5e-7, 3e-7, 2e-7)  # learned budgets tried per instance, largest first


def ensemble_instance_budgets(ctx, kern, inst, tuned, tol: float = 1e-6, safety: float = 0.8) -> list:
    """Per instance, the largest learned budget of ENSEMBLE_EPS_LADDER, no smaller than its size class's tuned
    budget, with which the class's other tuned settings meet safety * tol on ENSEMBLE_SAMPLE seeded targets of
    that instance against the FP64 direct sum (the class's budget, which every member met in tuning, when none
    of the larger ones does): members whose vortex the class setting over-resolves run with a larger budget."""
    import torch

    import lpmcxx_b200 as L
    from lpmcxx_b200 import learned

    params = learned.load()[0]
    out = []
    for i, (lvl, p, n_src) in enumerate(inst):
        t = tuned[lvl]
        d = torch.tensor(p, device="cuda")
        rng = np.random.default_rng(500 + i)
        idx = torch.as_tensor(np.sort(rng.choice(p.shape[0], size=min(ENSEMBLE_SAMPLE, p.shape[0]), replace=False)),
                              device="cuda")
        ref = torch.empty((3, idx.numel()), dtype=torch.float64, device="cuda")
        ctx.direct_sum_dev(kern, L.LPM_PREC_F64, d[:n_src], d[idx].contiguous(), ref)
        u = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
        ts = L.TreeSum(ctx, kern, L.tree_solver(L.LPM_PREC_F32, 10, t["max_per_leaf"], t["theta"], learned=True,
                                                tolerance=t["eps"]), n_src, p.shape[0])
        try:
            ts.set_mlp(params)
            for name in ("order_bias", "batch_level", "near_targets", "near_tile", "near_split"):
                ts.set_param(name, t[name])
            eps = t["eps"]
            for cand in sorted({e for e in ENSEMBLE_EPS_LADDER if e > t["eps"]}, reverse=True):
                ts.set_param("eps", cand)
                ts.eval(d[:n_src], d, u)
                torch.cuda.synchronize()
                if float(torch.linalg.norm(u[:, idx] - ref) / torch.linalg.norm(ref)) <= safety * tol:
                    eps = cand
                    break
        finally:
            ts.close()
        out.append(eps)
    return out


def ensemble_accuracy(ctx, kern, ens, inst, sample: int = ENSEMBLE_SAMPLE, seed: int = 11) -> list:
    """Relative L2 velocity error of every instance's treecode against the FP64 direct sum, on `sample`
    seeded targets of its current state."""
    import torch

    import lpmcxx_b200 as L

    errs = []
    rng = np.random.default_rng(seed)
    for i, (_, p, n_src) in enumerate(inst):
        rk = ens.instance(i)
        state = torch.empty((p.shape[0], 4), dtype=torch.float64, device="cuda")
        rk.get_state(state)
        u = torch.empty((3, p.shape[0]), dtype=torch.float64, device="cuda")
        rk.velocity(u)
        torch.cuda.synchronize()
        idx = torch.as_tensor(np.sort(rng.choice(p.shape[0], size=min(sample, p.shape[0]), replace=False)),
                              device="cuda")
        ref = torch.empty((3, idx.numel()), dtype=torch.float64, device="cuda")
        ctx.direct_sum_dev(kern, L.LPM_PREC_F64, state[:n_src], state[idx].contiguous(), ref)
        torch.cuda.synchronize()
        errs.append(float(torch.linalg.norm(u[:, idx] - ref) / torch.linalg.norm(ref)))
    return errs


def run_gpu_ensemble(args) -> None:
    """The ensemble configuration: 64 Biot-Savart RK4 instances of uneven sizes (icos L5..L8), each with the
    solver settings the autotuner picked for its size class; a step advances every instance by one RK4 step
    (one replay of the ensemble's graph)."""
    import torch

    import lpmcxx_b200 as L
    import lpmcxx_b200.workloads as W
    from lpmcxx_b200 import learned

    local = env_int("LOCAL_RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    torch.cuda.set_device(local)
    levels = tuple(int(v) for v in args.ens_levels.split(","))
    inst = W.ensemble_instances(levels=levels, per_level=args.ens_per_level)
    ctx = L.Context(local)
    kern = L.biot_savart_kernel()
    ctx.use_torch_stream()
    tuned = ensemble_tune(ctx, kern, inst)
    eps_inst = ensemble_instance_budgets(ctx, kern, inst, tuned)
    solvers = [L.tree_solver(L.LPM_PREC_F32, 10, tuned[lvl]["max_per_leaf"], tuned[lvl]["theta"], learned=True,
                             tolerance=eps_inst[i]) for i, (lvl, _, _) in enumerate(inst)]
    ens = L.Ensemble(ctx, kern, solvers, [n for _, _, n in inst], [p.shape[0] for _, p, _ in inst], lanes=args.lanes)
    ens.set_mlp(learned.load()[0])
    for i, (lvl, p, _) in enumerate(inst):
        rk = ens.instance(i)
        rk.set_param("order_bias", tuned[lvl]["order_bias"])
        rk.set_param("batch_level", tuned[lvl]["batch_level"])
        rk.set_param("near_targets", tuned[lvl]["near_targets"])
        rk.set_param("near_tile", tuned[lvl]["near_tile"])
        rk.set_param("near_split", tuned[lvl]["near_split"])
        rk.set_state(p)
    err_t0 = ensemble_accuracy(ctx, kern, ens, inst)
    dt = 0.01
    ens.step(dt, args.warmup, use_graph=True)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    clocks = ClockSampler(local).start()
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ens.step(dt, 1, use_graph=True)  # synchronous: replays on the ensemble's stream, waits for it
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    launches = ctx.launch_count - launches0
    value = world * args.steps / (sum(ms) * 1e-3)
    err_final = ensemble_accuracy(ctx, kern, ens, inst)
    # the same ensemble with the fused launches in one group, and in lane mode (each instance's far and near
    # launches on its lane), for comparison: a few steps after their own warm-up step and capture
    states = [ens.instance(i).get_state() for i in range(len(inst))]
    groups = int(ens.get_param("fused_groups"))

    def compare_ms(name, value):
        ens.set_param(name, value)
        ens.step(dt, 1, use_graph=True)
        torch.cuda.synchronize()
        out_ms = []
        for _ in range(min(args.steps, 3)):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            ens.step(dt, 1, use_graph=True)
            e1.record()
            e1.synchronize()
            out_ms.append(e0.elapsed_time(e1))
        return float(np.mean(out_ms))

    groups_ms = {g: compare_ms("fused_groups", g) for g in (1, 4) if g != groups}
    ens.set_param("fused_groups", groups)
    lane_ms = compare_ms("fused", 0)
    ens.set_param("fused", 1)
    for i, st in enumerate(states):
        ens.instance(i).set_state(st)
    ens.step(dt, 2, use_graph=True)  # fused graph captured again (outside every timed region)
    # work of one step: four evaluations per instance, each as its last one (tree statistics)
    work = 0.0
    for i in range(len(inst)):
        st = ens.instance(i).tree_stats()
        work += 4.0 * (FLOPS_PER_BS_PAIR * st["near_pairs"] + 8.0 * st["far_terms"] + FLOPS_PER_FAR_EVAL * st["far_evals"])
    fp32_peak = ctx.fma_peak_tflops(L.LPM_PREC_F32)
    achieved = work / (float(np.mean(ms)) * 1e-3) * 1e-12
    # end to end: every instance's state from pinned host memory, one step, every state back
    host = [torch.tensor(p).pin_memory() for _, p, _ in inst]
    back = [torch.empty_like(h).pin_memory() for h in host]
    e2e_s = []
    for _ in range(max(1, min(args.steps, 5))):
        t0 = time.perf_counter()
        for i, h in enumerate(host):
            ens.instance(i).set_state(h)
        ens.step(dt, 1, use_graph=True)
        for i, b in enumerate(back):
            ens.instance(i).get_state(b)
        e2e_s.append(time.perf_counter() - t0)
    state_bytes = int(sum(p.shape[0] for _, p, _ in inst)) * 32
    n_total = int(sum(p.shape[0] for _, p, _ in inst))
    pairs_step = float(sum(4.0 * p.shape[0] * n for _, p, n in inst))
    out = {
        "metric": ENSEMBLE_METRIC if (levels, args.ens_per_level) == ((5, 6, 7, 8), 16) else
        f"ensemble RK4 steps/s: {len(inst)} instances, learned treecode", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"{len(inst)} instances: icos L{'/L'.join(map(str, levels))} x {args.ens_per_level}, "
                               f"RH m=4 + seeded Gaussian, {n_total:,} particles",
                   "solver": "learned treecode, per size class the autotuned leaf / theta / budget / batch level / "
                             "near tile (order bias 2); per instance the largest budget of "
                             f"{list(ENSEMBLE_EPS_LADDER)} (no smaller than its class's) that still meets 0.8e-6",
                   "tuned": {f"L{k}": v for k, v in tuned.items()},
                   "instance_eps": {f"L{k}": [e for (lvl, _, _), e in zip(inst, eps_inst) if lvl == k]
                                    for k in tuned},
                   "lanes": args.lanes, "dt": dt,
                   "graph": "one CUDA graph replay per ensemble step; per RK4 stage, the far field of each group "
                            "of instances (the lanes in fused_groups groups stepping independently) is one "
                            "persistent launch per Taylor order and their near field one per near tile shape",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "rel_l2_vs_fp64_direct": {"sample": f"{ENSEMBLE_SAMPLE} seeded targets per instance, FP64 GPU direct sum",
                                  "t0_max": max(err_t0), "t0_median": float(np.median(err_t0)),
                                  "final_max": max(err_final), "final_median": float(np.median(err_final)),
                                  "final_step": args.warmup + args.steps},
        "particle_steps_per_s": value * n_total,
        "fused_groups": groups, "other_fused_groups_ms_per_step": {str(g): v for g, v in groups_ms.items()},
        "lane_mode_ms_per_step": lane_ms,
        "roofline": {"bound": "fp32", "kernel": "whole step (near + far field, all instances)",
                     "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": None, "peak_source": "measured FMA microbenchmark (lpm_fma_peak) on this GPU",
                     "work": "17 flops per near pair + 8 per far coefficient + 24 per far evaluation, 4 "
                             "evaluations per step, from each instance's tree statistics"},
        "e2e": {"value": world / float(np.mean(e2e_s)), "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes},
        "gpu_launches": launches, "clocks": clk,
    }
    ens.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(reps=2)
        out["cpu_baseline"] = {"value": base["pairs_per_s"] / pairs_step, "unit": "steps/s", "cores": base["cores"],
                               "kind": base["kind"],
                               "sample": base["sample"] + f"; the ensemble step's {pairs_step:.3e} pairs at that rate"}
    print(json.dumps(out))


def pairwise_direct_f32(ctx, kern, state0, n_src: int, fp32_peak: float, u64, stream) -> dict:
    """The FP32 direct-sum kernel (bs_f32_kernel) on the headline workload: one warm-up evaluation, then
    one evaluation timed by the library's per-launch CUDA events; its TFLOP/s at 17 flops per pair
    against the measured FP32 FMA peak, and its error against the FP64 direct sum."""
    import torch

    import lpmcxx_b200 as L

    n = state0.shape[0]
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    ctx.direct_sum_dev(kern, L.LPM_PREC_F32, state0[:n_src], state0, out, n_coincident=n_src)
    ctx.set_profiling(True)
    ctx.direct_sum_dev(kern, L.LPM_PREC_F32, state0[:n_src], state0, out, n_coincident=n_src)
    prof = ctx.profile_report()
    ctx.set_profiling(False)
    ms = prof["bs_f32_kernel"]["ms"]
    tflops = FLOPS_PER_BS_PAIR * float(n_src) * float(n) / (ms * 1e-3) * 1e-12
    return {"kernel": "bs_f32_kernel", "ms": ms, "pairs": n_src * n, "achieved_tflops": tflops,
            "peak_tflops": fp32_peak, "frac": tflops / fp32_peak,
            "rel_l2_vs_fp64_direct": float(torch.linalg.norm(out - u64) / torch.linalg.norm(u64)),
            "timing": "one evaluation after one warm-up, CUDA events around the launch"}


def poisson_summary(ctx, device: int, n: int = 1_048_576, reps: int = 5, cpu: bool = True) -> dict:
    """The 3D Poisson treecode configuration inside the headline run: evaluations/s at n points (median
    of `reps` evaluations after 3 warm-up ones), its error against the FP64 direct sum, the dominant
    kernel's roofline and the near / far split."""
    import torch

    import lpmcxx_b200 as L
    import lpmcxx_b200.workloads as W

    ctx.use_torch_stream()  # the library enqueues on the stream the CUDA events below are recorded on
    pts = torch.tensor(W.poisson_cube(n), device="cuda")
    kern = L.poisson_kernel()
    order, theta, leaf = POISSON_SETTINGS
    ts = L.TreeSum(ctx, kern, L.tree_solver(L.LPM_PREC_F32, order, leaf, theta), n, n)
    out = torch.empty((1, n), dtype=torch.float64, device="cuda")
    for _ in range(3):
        ts.eval(pts, pts, out)
    stream = torch.cuda.current_stream()
    ms = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ts.eval(pts, pts, out)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    ctx.set_profiling(True)
    ts.eval(pts, pts, out)
    prof = ctx.profile_report()
    ctx.set_profiling(False)
    st = ts.stats()
    ts.close()
    ref = torch.empty_like(out)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.direct_sum_dev(kern, L.LPM_PREC_F64, pts, pts, ref)
    e1.record(stream)
    e1.synchronize()
    fp32_peak = ctx.fma_peak_tflops(L.LPM_PREC_F32)
    near_ms = prof.get("near_kernel", {}).get("ms", float("nan"))
    far_ms = prof.get("far_kernel", {}).get("ms", float("nan"))
    near_tf = FLOPS_PER_POISSON_PAIR * float(st["near_pairs"]) / (near_ms * 1e-3) * 1e-12
    far_tf = (2.0 * float(st["far_terms"]) + 12.0 * float(st["far_evals"])) / (far_ms * 1e-3) * 1e-12
    med = float(np.median(ms))
    return {"workload": f"{n:,} points uniform in [-1,1]^3, charges U(-1,1), splitmix64 seed 0x2B",
            "solver": f"Poisson treecode p={order} (|k|<=p), theta={theta}, {leaf} per leaf",
            "evaluations_per_s": 1e3 / med, "ms_per_evaluation": med,
            "rel_l2_vs_fp64_direct": float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref)),
            "fp64_direct_ms": e0.elapsed_time(e1), "speedup_vs_fp64_direct": e0.elapsed_time(e1) / med,
            "near_kernel": {"ms": near_ms, "tflops": near_tf, "frac": near_tf / fp32_peak},
            "far_kernel": {"ms": far_ms, "tflops": far_tf, "frac": far_tf / fp32_peak,
                           "launches": prof.get("far_kernel", {}).get("launches")},
            "peak_tflops_fp32": fp32_peak, "tree_stats": st,
            "cpu_baseline": poisson_cpu_baseline(n) if cpu else None}


def run_gpu(args) -> None:
    import torch
    import torch.distributed as dist

    import lpmcxx_b200 as L
    import lpmcxx_b200.workloads as W

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    mesh, p, n_src = W.gaussian_vortex_mesh("icos", args.level)
    n = p.shape[0]
    stream = torch.cuda.Stream()
    ctx = L.Context(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    state0 = torch.tensor(p, device="cuda")
    kern = L.biot_savart_kernel()
    head = args.solver
    with torch.cuda.stream(stream):
        ctx.use_torch_stream()
        # ---- headline solver: warm-up then K timed steps
        rk = L.RK4(ctx, kern, solver_desc(head), n_src, n)
        if head == "tree_learned":
            from lpmcxx_b200 import learned

            params, _ = learned.load()
            if params is None:
                raise SystemExit("tree_learned: the shipped selector weights are missing")
            rk.set_mlp(params)
            rk.set_param("order_bias", LEARNED_ORDER_BIAS)
            rk.set_param("batch_level", rk.get_param("batch_level") + LEARNED_BATCH_LEVEL_OFFSET)
        rk.set_state(state0)
        rk.step(args.dt, args.warmup, use_graph=True)
        stream.synchronize()
        launches0 = ctx.launch_count
        step_ms = []
        clocks = ClockSampler(local).start()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rk.step(args.dt, 1, use_graph=True)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        clk = clocks.stop()
        launches = ctx.launch_count - launches0
        total_ms = float(sum(step_ms))
        # the state after the warm-up and timed steps, for the accuracy check at the final state
        state_final = torch.empty_like(state0)
        rk.get_state(state_final)
        total_ms, value = replica_rate(total_ms, args.steps)
        if world > 1:
            dist.barrier()

        # ---- end to end through the host API: pinned host state in, step, state out
        host_in = torch.tensor(p).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        rk.set_state(host_in)
        rk.step(args.dt, 1, use_graph=True)
        torch.cuda.synchronize()
        e2e_s = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            rk.set_state(host_in)
            rk.step(args.dt, 1, use_graph=True)
            rk.get_state(host_out)
            e2e_s.append(time.perf_counter() - t0)
        e2e_value = world * args.steps / sum(e2e_s)
        state_bytes = n * 4 * 8

        # ---- accuracy of the headline velocity against the FP64 direct sum at the initial state
        # (one uncaptured evaluation, with per-kernel CUDA-event timing for the roofline) and at the state
        # the timed steps reached
        rk.set_state(state0)
        u_head = torch.empty((3, n), dtype=torch.float64, device="cuda")
        ctx.set_profiling(True)
        rk.velocity(u_head)
        prof = ctx.profile_report()
        ctx.set_profiling(False)
        tstats = rk.tree_stats() if head.startswith("tree") else None
        rk.set_state(state_final)
        u_head_final = torch.empty((3, n), dtype=torch.float64, device="cuda")
        rk.velocity(u_head_final)
        rk.close()

        # ---- FP64 GPU direct sum on the same workload (one RK4 step), its velocity at the initial and the
        # final state, and the FP64-pipe share of its kernel
        u64 = torch.empty((3, n), dtype=torch.float64, device="cuda")
        u64_final = torch.empty((3, n), dtype=torch.float64, device="cuda")
        fp64_sps = None
        if head != "direct_f64":
            rk64 = L.RK4(ctx, kern, solver_desc("direct_f64"), n_src, n)
            rk64.set_state(state_final)
            rk64.velocity(u64_final)
            rk64.set_state(state0)
            rk64.velocity(u64)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rk64.step(args.dt, 1, use_graph=False)
            e1.record(stream)
            e1.synchronize()
            fp64_sps = 1e3 / e0.elapsed_time(e1)
            rk64.close()
        else:
            u64.copy_(u_head)
            u64_final.copy_(u_head_final)
            fp64_sps = value / world
        rel_l2 = float(torch.linalg.norm(u_head - u64) / torch.linalg.norm(u64))
        rel_l2_final = float(torch.linalg.norm(u_head_final - u64_final) / torch.linalg.norm(u64_final))
        rel_linf = float((u_head - u64).abs().max() / u64.abs().max())
        fp32_peak = ctx.fma_peak_tflops(L.LPM_PREC_F32)
        fp64_peak = ctx.fma_peak_tflops(L.LPM_PREC_F64)
        pairwise = None if args.no_extras else pairwise_direct_f32(ctx, kern, state0, n_src, fp32_peak, u64, stream)
    torch.cuda.synchronize()
    poisson = None if (args.no_extras or world > 1) else poisson_summary(ctx, local, cpu=not args.no_cpu_baseline)

    # dominant kernel of the headline step
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"]) if prof else (None, None)
    roof = None
    if dom[0] is not None:
        name, st = dom
        # the profile covers one velocity evaluation: its work over the kernel's summed time there (the far
        # field runs as one launch per Taylor order present)
        avg_ms = st["ms"] / st["launches"]
        eval_ms = st["ms"]
        order = TREE_SETTINGS.get(head, (0,))[0]
        work = kernel_work(name, n_src, n, tstats, order)
        fp64_bound = "f64" in name
        peak = fp64_peak if fp64_bound else fp32_peak
        if work is not None:
            achieved = work[0] / (eval_ms * 1e-3) * 1e-12
            roof = {"bound": "fp64" if fp64_bound else "fp32", "kernel": name, "achieved": achieved,
                    "peak": peak, "unit": work[1], "frac": achieved / peak, "traffic": profile_summary_traffic(name),
                    "peak_source": "measured FMA microbenchmark (lpm_fma_peak) on this GPU",
                    "avg_launch_ms": avg_ms, "launches_per_evaluation": st["launches"], "evaluation_ms": eval_ms,
                    "share": st["ms"] / sum(v["ms"] for v in prof.values())}
    out = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32" if head != "direct_f64" else "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.level, n_src, n, args.dt), "solver": head,
                   **({"selector": f"budget {LEARNED_EPS}, order bias {LEARNED_ORDER_BIAS}, "
                                   f"theta {TREE_SETTINGS['tree_learned'][1]}, 512 per leaf, batch level "
                                   f"default {LEARNED_BATCH_LEVEL_OFFSET:+d}"}
                      if head == "tree_learned" else {}),
                   "n_sources": n_src,
                   "n_targets": n, "dt": args.dt,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed (256 MiB write) before every timed step, outside the timed events",
                   "graph": "one CUDA graph replay per RK4 step"},
        "rel_l2_vs_fp64_direct": rel_l2,
        "rel_l2_t0": rel_l2,
        "rel_l2_final": rel_l2_final,
        "rel_linf_t0": rel_linf,
        "accuracy_states": f"t0 = the initial state; final = after the {args.warmup} warm-up and {args.steps} timed "
                           f"steps (dt {args.dt:g}); FP64 GPU direct sum at each",
        "fp64_direct_steps_per_s": fp64_sps,
        "speedup_vs_fp64_direct": (value / world) / fp64_sps if fp64_sps else None,
        # absolute rates: the direct sum's (target, source) interactions the step replaces, and the work the
        # treecode computed (near pairs, far target-cluster evaluations) per second
        "interactions_per_s": {
            "direct_equivalent_pairs": value * 4.0 * n_src * n,
            **({"near_pairs": value * 4.0 * tstats["near_pairs"], "far_evals": value * 4.0 * tstats["far_evals"]}
               if tstats and "near_pairs" in tstats else {})},
        "roofline": roof,
        "kernel_profile_ms": {k: v for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])[:12]},
        "tree_stats": tstats,
        "fma_peaks_tflops": {"fp32": fp32_peak, "fp64": fp64_peak},
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes},
        "gpu_launches": launches,
        "clocks": clk,
        "pairwise_direct_f32": pairwise,
        "poisson_treecode": poisson,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(reps=2)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def run_reference(args) -> None:
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    base = cpu_baseline(reps=args.warmup + args.steps)
    reps = base["rep_seconds"][args.warmup:]
    n_src = 20 * 4 ** LEVEL
    n_tgt = n_src + 2 + 10 * 4 ** LEVEL
    rates = [base["pairs_per_s"]] if not reps else None
    value = base["value"]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": env_int("WORLD_SIZE", 1),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "solver": "reference DirectSum::meshSolve (FP64, CPU)",
                   "n_sources": n_src, "n_targets": n_tgt, "dt": DT, "host_cores": cores},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": base["cores"], "kind": base["kind"],
                         "sample": base["sample"]},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del rates
    print(json.dumps(out))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lpm", choices=["lpm", "reference"])
    ap.add_argument("--solver", default="tree_learned",
                    choices=["direct_f32", "direct_f64", "tree_f32", "tree_cfg2a", "tree_learned"])
    ap.add_argument("--level", type=int, default=LEVEL)
    ap.add_argument("--dt", type=float, default=DT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra keys of the headline line (FP32 direct-sum kernel, Poisson treecode)")
    ap.add_argument("--workload", default="sphere_rk4",
                    choices=["sphere_rk4", "poisson_cube", "ensemble", "direct_cube"],
                    help="sphere_rk4: the Biot-Savart RK4 headline; poisson_cube: the 3D Poisson treecode; "
                         "ensemble: 64 uneven RK4 instances; direct_cube: FP32 / FP64 direct-sum RK4 at cube L8")
    ap.add_argument("--lanes", type=int, default=8, help="ensemble: streams the instances are spread over")
    ap.add_argument("--ens-levels", default="5,6,7,8",
                    help="ensemble: icosahedral levels of the instances (a smaller ensemble for profiling)")
    ap.add_argument("--ens-per-level", type=int, default=16, help="ensemble: instances per level")
    ap.add_argument("--points", type=int, default=1_048_576, help="poisson_cube: number of points")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "poisson_cube":
        run_gpu_poisson(args)
    elif args.workload == "ensemble":
        run_gpu_ensemble(args)
    elif args.workload == "direct_cube":
        run_gpu_direct_cube(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
