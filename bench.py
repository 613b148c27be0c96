#!/usr/bin/env python3
"""Benchmark of the compact sparse-grid hot path on B200.

Workload (the reference's at-scale GPU case): a regular sparse grid with
d=10 and n=10 levels (N = 32,978,945 points, S = 92,378 subspaces, FP32),
values f(x) = exp(-sum x_k^2) at the grid points; one step hierarchizes the
grid from its nodal values and evaluates the interpolant at 2^24 query
points uniform on [0,1)^10 (seed 1; rank r uses seed 1 + r).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  `value` is whole-job evals/s with inputs resident
in HBM; `e2e` is the same metric through the C ABI's host-buffer calls
(sg_set_values / sg_hierarchize / sg_evaluate) with the host<->device copies
inside the timed region.  Inputs (132 MB grid + 671 MB points per rank) are
larger than the 126 MB L2, so no flush is needed between steps.
With --gpus N > 1 and no torchrun environment, the bench starts N local
ranks itself (torch.distributed.run, NCCL); each rank holds a replica of the
grid and evaluates its own 2^24 points (weak scaling), and the step time is
the slowest rank's.
`--impl reference` times the reference's own C/OpenMP code
(omp_hierarchize3 + omp_evaluate5, compiled in place into oracle/_ref) on the
host cores, on a bounded sample of the same workload, with inputs built by
the checker side (oracle/) only.  Before timing, the library's autotuner
picks the evaluation and sweep settings on the bench's own buffers (no
setting changes a result).  At N=1 the default line also carries compact
results of the other workloads (`batched`, `served`, `adaptive`), each with
its error against the FP64 oracle.

Other workloads (`--workload`): `adaptive` (the limits-adaptive d=6 grid
refined by sg_refine, 2^22 points), `batched` (4096 grids of mixed d and n
in one batch), `served` (the serving loop under a Poisson request sweep,
with p50/p99 latency and the plain one-call-per-request comparison).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

D, NLEV, M_EVAL, SEED = 10, 10, 1 << 24, 1
N_POINTS, N_SUBSPACES = 32_978_945, 92_378
WORKLOAD = "regular sparse grid d=10 n=10 (N=32,978,945), f=exp(-|x|^2), hierarchize + evaluate 2^24 uniform points"
EVAL_SRC = os.path.join(ROOT, "adaptive_sparse_grid_bench_b200", "csrc", "eval_impl.cuh")
# Figures of one k_evaluate launch of the default workload, measured with ncu
# on the evaluation source whose sha256 starts with `source_sha16`; they are
# reported only while that source is unchanged (null otherwise).
#   dram_bytes: dram__bytes_read.sum + dram__bytes_write.sum of one full
#     2^24-point launch (one-pass metrics, so the full launch was captured);
#   inst_per_pair: smsp__inst_executed.sum x 32 / (points x subspaces) of a
#     1,048,576-point launch of the same grid (two points per thread, wide preset).
#   (either may be None: not captured on this source)
EVAL_CAPTURE = {"source_sha16": "ab15c4c8da0625a8", "captured": "2026-12-04", "dram_bytes": 2.953e9 + 0.588e9,
                "inst_per_pair": 7.14}
SM_COUNT, SCHEDULERS_PER_SM = 148, 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--points", type=int, default=None,
                    help="query points per rank and step (default: the workload's, 2^24 for single)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="single: leave out the compact batched/served/adaptive results of the N=1 line")
    ap.add_argument("--cpu-seconds", type=float, default=None,
                    help="CPU work per reference step (default: about 150 s over all steps, 1.5..12 s each)")
    ap.add_argument("--workload", default="single", choices=["single", "adaptive", "batched", "served"],
                    help="single: the d=10 n=10 grid (default); adaptive: the refined d=6 grid; batched: many "
                         "grids of mixed d and n; served: Poisson request stream against resident grids")
    ap.add_argument("--grids", type=int, default=4096, help="batched: number of grids")
    ap.add_argument("--eval-config", default=None,
                    help="single/adaptive: PPT,BLOCKING (e.g. 2,1) set after the autotuner, so that a profiler "
                         "captures a named kernel (the autotuner's own timings are distorted under a profiler)")
    ap.add_argument("--no-graph", action="store_true",
                    help="batched: launch kernels directly instead of replaying CUDA graphs (for profilers that "
                         "cannot follow stream capture)")
    ap.add_argument("--rates", default="4000,8000,16000,20000,24000,28000",
                    help="served: arrival rates (requests/s)")
    ap.add_argument("--requests", type=int, default=3000, help="served: requests per rate")
    ap.add_argument("--cap-gb", type=float, default=60.0, help="served: resident-grid byte cap")
    ap.add_argument("--create-frac", type=float, default=0.05, help="served: share of create+hierarchize requests")
    ap.add_argument("--batch-points", type=int, default=1 << 18, help="served: points per batch")
    ap.add_argument("--pool", type=int, default=512, help="served: resident grids at the start")
    ap.add_argument("--zero-copy", type=int, default=None, choices=[0, 1],
                    help="served: SG_SRV_OPT_ZERO_COPY (batches read and write pinned host memory in place)")
    ap.add_argument("--heavy-pairs", type=int, default=None,
                    help="served: SG_SRV_OPT_HEAVY_PAIRS (requests with this much work take the heavy lane)")
    ap.add_argument("--light-slots", type=int, default=None,
                    help="served: SG_SRV_OPT_LIGHT_SLOTS (light-lane batches in flight at once)")
    ap.add_argument("--sort-heavy", type=int, default=None, choices=[0, 1],
                    help="served: SG_SRV_OPT_SORT_HEAVY (spatial ordering of heavy requests' points)")
    ap.add_argument("--served-dump", default=None,
                    help="served: save each rate's per-request timeline (ms to batch, launch, completion, delivery; "
                         "points; pairs) to PREFIX_<rate>.npy")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def single_workload():
    """The d=10 n=10 regular grid of exp(-|x|^2) at 2^24 uniform points."""
    from adaptive_sparse_grid_bench_b200 import Grid, inputs
    from adaptive_sparse_grid_bench_b200._lib import SG_FN_GAUSS
    return {"name": WORKLOAD, "d": D, "n": NLEV, "limits": None, "fn": SG_FN_GAUSS, "params": (),
            "m_eval": M_EVAL, "make_grid": lambda: Grid(D, NLEV),
            "points": lambda rank, m: inputs.uniform_points(rank_seed(SEED, rank), m, D),
            "l2": "inputs larger than L2 (132 MB grid + 671 MB points)", "info": {}}


def adaptive_workload(args):
    """Limits-adaptive grid, d=6: from the regular level-4 grid, refine the
    children of subspaces holding a surplus above 1e-4 up to level 13
    (0-based) per dimension on exp(-50 |x - 0.3|^2), stopping before a grid
    above the regular level-14 bound (109,051,905 points); evaluate 2^22
    points, half uniform on [0,1)^6 and half N(0.3, 0.1^2) clipped to [0,1)
    (seed 2)."""
    from adaptive_sparse_grid_bench_b200 import inputs, refine
    from adaptive_sparse_grid_bench_b200._lib import SG_FN_BUMP
    d, m_eval, info = 6, 1 << 22, {}

    def make_grid():
        t0 = time.perf_counter()
        g, it = refine(d, 4, SG_FN_BUMP, (0.3, 50.0), tol=1e-4, max_level=13, max_points=109_051_905, max_iters=32)
        info.update({"refine_s": time.perf_counter() - t0, "grids_built": it, "n": g.n,
                     "limits": [int(x) for x in g.limits]})
        wl["n"], wl["limits"] = g.n, [int(x) for x in g.limits]
        return g

    def points(rank, m):
        h = m // 2
        seed = rank_seed(2, rank, 100)
        return np.concatenate([inputs.uniform_points(seed, h, d),
                               inputs.gaussian_points(seed, m - h, d, 0.3, 0.1, start=1 << 40)])

    wl = {"name": "limits-adaptive grid d=6 from n=4, tol 1e-4, level <= 13, f=exp(-50|x-0.3|^2), "
                  "evaluate 2^22 points (half uniform, half N(0.3,0.1) clipped)",
          "d": d, "n": None, "limits": None, "fn": SG_FN_BUMP, "params": (0.3, 50.0), "m_eval": m_eval,
          "make_grid": make_grid, "points": points, "l2": "points larger than L2", "info": info}
    return wl


def cpu_step_seconds(args) -> float:
    """CPU time per reference step: about 150 s over warm-up + timed steps,
    between 1.5 and 12 s per step."""
    if args.cpu_seconds is not None:
        return args.cpu_seconds
    return min(12.0, max(1.5, 150.0 / max(1, args.steps + args.warmup)))


class ReferenceCPU:
    """The reference's own CPU path (oracle/_ref, compiled in place) on one
    grid: a step is omp_hierarchize3 over the whole grid (c:1180) plus
    omp_evaluate5 (c:1708) over a fixed sample of the query points, sized
    once to `seconds` of CPU work; the step's evals/s is extrapolated
    linearly from the sample to the workload's point count."""

    def __init__(self, d, n, limits, values, X, m_step, seconds):
        from oracle.oracle import Reference
        self.r = Reference(d, n, limits)
        self.values, self.X, self.m_step = values, X, m_step
        self.r.set_values(values)
        t0 = time.perf_counter()
        self.r.hierarchize(9)
        t_h = time.perf_counter() - t0
        probe = min(2048, X.shape[0])
        t0 = time.perf_counter()
        self.r.evaluate(X[:probe], 7)
        t_probe = time.perf_counter() - t0
        m = int(probe * max(seconds - t_h, 0.5) / max(t_probe, 1e-6))
        self.m = int(min(X.shape[0], max(probe, (m // 2048) * 2048)))
        self.cores = int(self.r.lib().ref_max_threads())

    def step(self):
        """One step; returns (seconds measured, extrapolated evals/s, parts)."""
        self.r.set_values(self.values)
        t0 = time.perf_counter()
        self.r.hierarchize(9)
        t_h = time.perf_counter() - t0
        t0 = time.perf_counter()
        out = self.r.evaluate(self.X[:self.m], 7)
        t_e = time.perf_counter() - t0
        full = t_h + t_e * (self.m_step / self.m)
        return t_h + t_e, self.m_step / full, {"t_hierarchize_s": t_h, "t_eval_sample_s": t_e, "out": out}

    def one_thread(self, npts: int):
        """The serial variants: hierarchize7 (c:1009) over the whole grid and
        evaluate5 (c:1558) over `npts` points."""
        self.r.set_values(self.values)
        t0 = time.perf_counter()
        self.r.hierarchize(7)
        t_h = time.perf_counter() - t0
        npts = min(npts, self.X.shape[0])
        t0 = time.perf_counter()
        self.r.evaluate(self.X[:npts], 5)
        t_e = time.perf_counter() - t0
        return t_h, t_e, npts


def reference_cpu(values: np.ndarray, X: np.ndarray, seconds: float, wl=None, one_thread_points: int = 0):
    """cpu_baseline of the b200 line: one ReferenceCPU step (after one
    warm-up step) and, optionally, the 1-thread variants."""
    wl = wl or single_workload()
    rc = ReferenceCPU(wl["d"], wl["n"], wl["limits"], values, X, wl["m_eval"], seconds)
    rc.step()
    _, rate, parts = rc.step()
    hier_bytes = 8.0 * wl["d"] * values.size
    info = {"cores": rc.cores, "sample_points": rc.m, "ref_out": parts["out"], "surplus": rc.r.values(),
            "hierarchize_gbs": {"omp_hierarchize3": hier_bytes / parts["t_hierarchize_s"] / 1e9,
                                "threads": rc.cores, "bytes": "8*d*N"}}
    if one_thread_points:
        t_h, t_e, npts = rc.one_thread(one_thread_points)
        info["one_thread"] = {"evals_per_s": wl["m_eval"] / (t_h + t_e * wl["m_eval"] / npts),
                              "hierarchize7_gbs": hier_bytes / t_h / 1e9, "evaluate5_evals_per_s": npts / t_e,
                              "sample_points": npts}
    return rate, info


def error_vs_fp64(values: np.ndarray, gpu_out: np.ndarray, X: np.ndarray, nsample: int = 1024, ref_out=None,
                  wl=None):
    """Error of the GPU results against the FP64 oracle (FP64 hierarchize +
    evaluate of the same nodal values) on `nsample` query points spread over
    the launch (checker only).  max_rel_floor1e-2 is the per-point relative
    error |u - u64| / max(|u64|, 1e-2 max|u64|), the tests' bound."""
    from oracle.oracle import Oracle
    wl = wl or single_workload()
    o = Oracle(wl["d"], wl["n"], wl["limits"])
    s64 = o.hierarchize_f64(values.astype(np.float64))
    idx = np.linspace(0, X.shape[0] - 1, nsample).astype(np.int64)
    u64 = o.evaluate_f64(s64, X[idx])
    err = np.abs(gpu_out[idx].astype(np.float64) - u64)
    scale = float(np.max(np.abs(u64)))
    floor = 1e-2 * scale
    res = {"points": int(nsample), "max_abs": float(err.max()), "norm_rel": float(err.max() / scale),
           "max_rel_floor1e-2": float(np.max(err / np.maximum(np.abs(u64), floor)))}
    if ref_out is not None:
        e2 = np.abs(ref_out[idx[idx < ref_out.shape[0]]].astype(np.float64) - u64[idx < ref_out.shape[0]])
        if e2.size:
            res["reference_fp32_max_abs"] = float(e2.max())
            res["reference_fp32_norm_rel"] = float(e2.max() / scale)
    return res


def single_config(world: int, m: int, precision: str = "fp32") -> dict:
    """`config` of the default workload's line (both arms)."""
    return {"workload": WORKLOAD, "points_per_step_per_rank": m, "d": D, "n": NLEV, "limits": [NLEV - 1] * D,
            "num_points": N_POINTS, "num_subspaces": N_SUBSPACES, "hier_precision": precision,
            "l2": "inputs larger than L2 (132 MB grid + 671 MB points)",
            "parallelism": f"grid replicated, points sharded over {world} rank(s)"}


def repo_libraries() -> list:
    """The in-repo shared libraries mapped into this process."""
    libs = set()
    try:
        for ln in open("/proc/self/maps"):
            path = ln.split()[-1] if ln.strip() else ""
            if path.endswith(".so") and path.startswith(ROOT):
                libs.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(libs)


def run_reference_arm(args, rank: int, world: int):
    """The reference's CPU implementation (oracle/_ref) on the default
    workload; inputs come from the checker side (oracle/) only, so the
    product library is never loaded.  Rank 0 alone runs."""
    if rank != 0:
        return None
    if args.workload != "single":
        # the other workloads carry the reference's CPU time in their own
        # line (cpu_baseline / plain per-grid arms)
        return {"impl": "reference", "workload": args.workload,
                "unavailable": "the reference arm times the default single-grid workload only"}
    from oracle import workload as owl
    from oracle.oracle import Oracle
    vals = owl.grid_values(Oracle(D, NLEV), owl.f_gauss)
    m_step = args.points or M_EVAL
    X = owl.uniform_points(SEED, min(m_step, 1 << 20), D)
    rc = ReferenceCPU(D, NLEV, None, vals, X, m_step, cpu_step_seconds(args))
    secs, rates = [], []
    for it in range(args.warmup + args.steps):
        t, v, _ = rc.step()
        if it >= args.warmup:
            secs.append(t)
            rates.append(v)
    value = float(statistics.mean(rates))
    sample = (f"per step: omp_hierarchize3 on the full grid + omp_evaluate5 on {rc.m} of {m_step} points; "
              f"evals/s extrapolated linearly to {m_step} points")
    return {
        "impl": "reference", "metric": "evals/s", "value": value, "unit": "evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(statistics.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded SplitMix64)", "config": single_config(world, m_step),
        "extrapolated_from_points": rc.m,
        "ms_per_step_note": "measured time of one sampled step; value is extrapolated to the full step",
        "libraries": repo_libraries(),
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": rc.cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def device_inputs(g, wl, rank, npts, torch, dev):
    g.sample_function(wl["fn"], wl["params"])
    vals = torch.empty(g.num_points, dtype=torch.float32, device=dev)
    g.get_values_device(vals)
    torch.cuda.synchronize()
    return vals, wl["points"](rank, npts)


class EventTimer:
    """CUDA events on the launching stream around the timed steps."""

    def __init__(self, stream):
        import torch
        self.stream = stream
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def start(self):
        self.e0.record(self.stream)

    def stop(self):
        self.e1.record(self.stream)

    def ms(self) -> float:
        self.e1.synchronize()
        return self.e0.elapsed_time(self.e1)


def timed_steps(step, steps: int, world: int, barrier, timer, device=None):
    """The timed region every rank runs: barrier, `steps` calls of step()
    between the timer's marks, barrier; returns (this rank's ms, the max over
    ranks).  Every rank takes the same collective steps."""
    from adaptive_sparse_grid_bench_b200.sharding import max_over_ranks
    barrier()
    timer.start()
    for _ in range(steps):
        step()
    timer.stop()
    barrier()
    ms = timer.ms()
    return ms, (max_over_ranks(ms, device) if world > 1 else ms)


def job_rate(points_per_rank: int, world: int, steps: int, ms_max: float) -> float:
    """Whole-job evals/s: every rank evaluates its own points each step
    (weak scaling), the job's time is the slowest rank's."""
    return world * points_per_rank * steps / (ms_max / 1e3)


def ev_gflops(d: int, pairs_per_s: float) -> float:
    """The reference's own evaluation FLOP count (EV_FLOPS, c:51-52:
    11 d + 2 per point-subspace pair) per second, in GFLOP/s: a nominal
    figure for comparing with its printed numbers, not counted operations."""
    return pairs_per_s * (11 * d + 2) / 1e9


def hi_gflops(d: int, num_points: int, ms: float) -> float:
    """The reference's hierarchization FLOP count (HI_FLOPS, c:48-49: 3 d
    per grid point) per second, in GFLOP/s (nominal, as ev_gflops)."""
    return 3.0 * d * num_points / (ms / 1e3) / 1e9


def rank_seed(base: int, rank: int, stride: int = 1) -> int:
    """Rank r draws its query points from stream base + stride * r."""
    return base + stride * rank


def capture_figures():
    """EVAL_CAPTURE while the evaluation source is the one it was measured on."""
    import hashlib
    try:
        sha = hashlib.sha256(open(EVAL_SRC, "rb").read()).hexdigest()[:16]
    except OSError:
        sha = None
    return (EVAL_CAPTURE if sha == EVAL_CAPTURE["source_sha16"] else None), sha


def run_b200(args, rank: int, world: int, local_rank: int, wl=None, extras: bool = False, err: bool = False):
    import torch
    import torch.distributed as dist
    from adaptive_sparse_grid_bench_b200._lib import (SG_OPT_EVAL_BLOCKING, SG_OPT_EVAL_PPT, SG_OPT_EVAL_SORT,
                                                      SG_OPT_HIER_KERNEL, SG_OPT_PROFILE, kernel_launches)

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    wl = wl or single_workload()
    D = wl["d"]
    g = wl["make_grid"]()
    g.precision = args.precision
    g.set_option(SG_OPT_PROFILE, 1)
    vals_d, X = device_inputs(g, wl, rank, args.points if args.points else wl["m_eval"], torch, dev)
    m = X.shape[0]
    X_d = torch.from_numpy(X).to(dev)
    out_d = torch.empty(m, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    # the library's autotuner picks the evaluation and sweep settings on
    # this workload's own buffers (no setting changes a result)
    tuned = g.autotune(X_d, out_d, m, stream)
    if args.eval_config:
        ppt, blocking = (int(v) for v in args.eval_config.split(","))
        g.set_option(SG_OPT_EVAL_PPT, ppt)
        g.set_option(SG_OPT_EVAL_BLOCKING, blocking)
    tuned["chosen"] = {"ppt": g.get_option(SG_OPT_EVAL_PPT), "sort": g.get_option(SG_OPT_EVAL_SORT),
                       "blocking": g.get_option(SG_OPT_EVAL_BLOCKING),
                       "hier_kernel": g.get_option(SG_OPT_HIER_KERNEL)}
    t_hier, t_eval, t_sort = [], [], []

    def step():
        g.set_values_device(vals_d, stream)
        g.hierarchize_async(stream)
        g.evaluate_device(X_d, out_d, m, stream)

    def step_timed():
        step()
        t = g.timings()  # waits for this step's phase events
        t_hier.append(t["hierarchize"])
        t_sort.append(t["sort"])
        t_eval.append(t["evaluate"])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    g.sync(stream)
    barrier()
    with Clocks(local_rank) as clk:
        launches0 = kernel_launches()
        ms, ms_max = timed_steps(step_timed, args.steps, world, barrier, EventTimer(stream), dev)
        launches = kernel_launches() - launches0
    g.sync(stream)
    value = job_rate(m, world, args.steps, ms_max)

    # end-to-end through the host-buffer C ABI, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        vals_h = torch.empty(g.num_points, dtype=torch.float32, pin_memory=True)
        vals_h.copy_(vals_d)
        X_h = torch.empty((m, D), dtype=torch.float32, pin_memory=True)
        X_h.copy_(torch.from_numpy(X))
        out_h = torch.empty(m, dtype=torch.float32, pin_memory=True)
        vh, xh, oh = vals_h.numpy(), X_h.numpy(), out_h.numpy()
        import ctypes
        from adaptive_sparse_grid_bench_b200._lib import check, lib

        def step_e2e():
            check(lib().sg_set_values(g.handle, vh.ctypes.data))
            check(lib().sg_hierarchize(g.handle))
            check(lib().sg_evaluate(g.handle, xh.ctypes.data, oh.ctypes.data, ctypes.c_int64(m)))

        step_e2e()
        barrier()
        _, e_ms = timed_steps(step_e2e, args.steps, world, barrier, EventTimer(torch.cuda.current_stream()), dev)
        e2e = {"value": job_rate(m, world, args.steps, e_ms), "unit": "evals/s",
               "h2d_bytes_per_step": int(g.num_points * 4 + m * D * 4), "d2h_bytes_per_step": int(m * 4)}
        if not np.array_equal(oh, out_d.cpu().numpy()):
            raise RuntimeError("host-buffer and device-pointer evaluations differ")

    if rank != 0:
        return None
    S = g.num_subspaces
    hier_ms = statistics.mean(t_hier)
    eval_ms = statistics.mean(t_eval)
    hier_gbs = 8.0 * D * g.num_points / (hier_ms / 1e3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        peaks = json.load(open(peaks_path))
        peak = float(peaks["hbm_gbs"])
        peak_src = "measured"
    except (OSError, KeyError, ValueError):
        peaks, peak, peak_src = {}, 6650.0, "fallback"
    eval_bytes = 4.0 * (S + D + 1) * m
    achieved = eval_bytes / (eval_ms / 1e3) / 1e9
    clocks = clk.summary()
    pairs_per_s = m * S / (eval_ms / 1e3)
    cap, src_sha = capture_figures()
    default_case = wl["name"] == WORKLOAD and m == M_EVAL
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": cap["dram_bytes"] if (cap and default_case) else None,
            "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one full launch, captured "
                               f"{cap['captured']} on evaluation source {cap['source_sha16']}") if cap else
                              f"no capture for evaluation source {src_sha}",
            "kernel": "k_evaluate", "peak_source": peak_src,
            "bytes": "4*(S+d+1) per query point (cache-served surplus reads counted)"}
    if cap and cap["inst_per_pair"]:
        # SM issue roofline: thread instructions per pair (ncu) x pairs/s
        # against 148 SMs x 4 schedulers x one warp instruction per clock
        mhz = clocks.get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
        issue = cap["inst_per_pair"] * pairs_per_s / 32.0
        roof["issue"] = {"warp_inst_per_s": issue, "peak_warp_inst_per_s": SM_COUNT * SCHEDULERS_PER_SM * mhz * 1e6,
                         "frac": issue / (SM_COUNT * SCHEDULERS_PER_SM * mhz * 1e6),
                         "inst_per_pair": cap["inst_per_pair"]}
    line = {
        "metric": "evals/s", "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64; values sampled on device)",
        "config": (single_config(world, m, args.precision) if wl["name"] == WORKLOAD else
                   {"workload": wl["name"], "points_per_step_per_rank": m, "d": D, "n": g.n,
                    "limits": [int(x) for x in g.limits], "num_points": g.num_points, "num_subspaces": S,
                    "hier_precision": args.precision, "l2": wl["l2"],
                    "parallelism": f"grid replicated, points sharded over {world} rank(s)", **wl["info"]}),
        "hierarchize": {"value": hier_gbs, "unit": "GB/s", "ms": hier_ms, "bytes": "8*d*N",
                        "frac_of_peak": hier_gbs / peak,
                        "ref_gflops": hi_gflops(D, g.num_points, hier_ms)},
        "evaluate": {"ms": eval_ms, "sort_ms": statistics.mean(t_sort), "evals_per_s": m / (eval_ms / 1e3),
                     "pairs_per_s": pairs_per_s, "ref_gflops": ev_gflops(D, pairs_per_s)},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "autotune_ms": tuned,
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        vals = vals_d.cpu().numpy()
        cpu_v, info = reference_cpu(vals, X[:1 << 20], cpu_step_seconds(args), wl,
                                    one_thread_points=4096 if extras else 0)
        line["cpu_baseline"] = {
            "value": cpu_v, "unit": "evals/s", "cores": info["cores"], "kind": "reference",
            "sample": (f"reference omp_hierarchize3 on the full grid + omp_evaluate5 on {info['sample_points']} "
                       f"of {wl['m_eval']} points, extrapolated linearly"),
            "hierarchize_gbs": info["hierarchize_gbs"]}
        if "one_thread" in info:
            line["cpu_baseline"]["one_thread"] = info["one_thread"]
        line["err_vs_fp64"] = error_vs_fp64(vals, out_d.cpu().numpy(), X, ref_out=info["ref_out"], wl=wl)
    elif world == 1 and err:
        line["err_vs_fp64"] = error_vs_fp64(vals_d.cpu().numpy(), out_d.cpu().numpy(), X, nsample=256, wl=wl)
    if world == 1 and extras:
        line["reference_gpu"] = reference_gpu(g, X, out_d.cpu().numpy(), nodal=vals_d.cpu().numpy())
    del X_d, out_d, vals_d
    g.close()
    return line


def run_batched(args, rank: int, world: int, local_rank: int):
    """Batched workload: `--grids` grids with d uniform in 2..12 and n in
    3..9 (at most 2e6 points each), f = prod_k (a_k + b_k x + c_k x^2) with
    coefficients ~U(-1,1) (seed 3), each evaluated at a log-uniform
    256..65536 uniform points.  One step = restore nodal values, hierarchize
    every grid (one graph launch), evaluate every grid (one graph launch).
    Also timed: the same grids one plain launch sequence per grid (a sample
    of grids), the reference's arrangement of one grid per run."""
    import torch
    from adaptive_sparse_grid_bench_b200 import Batch, Grid, inputs
    from adaptive_sparse_grid_bench_b200._lib import (SG_FN_QUAD, SG_HIER_FP32, SG_HIER_FP64, SG_OPT_HIER_PRECISION,
                                                      SG_OPT_USE_GRAPH, kernel_launches)
    from adaptive_sparse_grid_bench_b200.sharding import max_over_ranks
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dims, levels, coef, counts = inputs.batch_workload(rank_seed(3, rank), args.grids)
    b = Batch(dims, levels)
    b.set_option(SG_OPT_HIER_PRECISION, SG_HIER_FP64 if args.precision == "fp64" else SG_HIER_FP32)
    b.set_option(SG_OPT_USE_GRAPH, 0 if args.no_graph else 1)
    b.sample_function(SG_FN_QUAD, coef)
    vals = torch.empty(b.num_values, dtype=torch.float32, device=dev)
    b.get_values_device(vals)
    po = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    nflt = int(np.sum(counts * dims))
    X = torch.from_numpy(inputs.uniform01(rank_seed(SEED + 100, rank), nflt)).to(dev)
    out = torch.empty(int(po[-1]), dtype=torch.float32, device=dev)
    # a stream of its own: the legacy default stream cannot be captured, and
    # on this one the batch captures its launches once and replays the graphs
    stream = torch.cuda.Stream(device=dev)
    stream.wait_stream(torch.cuda.current_stream())
    b.set_values_device(vals, stream)
    b.hierarchize_async(stream)
    tuned = b.autotune(po, X, out, stream)  # points per thread and blocking per dimension
    tuned_ppt = {}
    for d in range(tuned.shape[2]):
        if tuned[0, 0, d] >= 0:
            bl, pp = np.unravel_index(int(np.argmin(tuned[:, :, d])), tuned.shape[:2])
            tuned_ppt[d] = {"ppt": int(pp) + 1, "blocking": int(bl) + 1}
    npts = [inputs.regular_grid_size(int(d), int(n))[0] for d, n in zip(dims, levels)]

    def step():
        b.set_values_device(vals, stream)
        b.hierarchize_async(stream)
        b.evaluate_device(po, X, out, stream)

    for _ in range(args.warmup):
        step()
    b.sync(stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    th, te = [], []
    with Clocks(local_rank) as clk:
        torch.cuda.synchronize()
        l0 = kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            b.set_values_device(vals, stream)
            ev[0].record(stream)
            b.hierarchize_async(stream)
            ev[1].record(stream)
            b.evaluate_device(po, X, out, stream)
            ev[2].record(stream)
            ev[2].synchronize()
            th.append(ev[0].elapsed_time(ev[1]))
            te.append(ev[1].elapsed_time(ev[2]))
        e1.record(stream)
        torch.cuda.synchronize()
        launches = kernel_launches() - l0
    b.sync(stream)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, dev) if world > 1 else ms
    total_pts = int(po[-1])
    value = world * total_pts * args.steps / (ms_max / 1e3)

    # one plain launch sequence per grid (sample of grids, extrapolated)
    sample = list(range(0, len(dims), max(1, len(dims) // 128)))
    plain_pts, plain_ms = 0, 0.0
    xs = X.cpu().numpy()
    coff = np.concatenate([[0], np.cumsum(counts * dims)])
    for g in sample:
        one = Grid(int(dims[g]), int(levels[g]))
        one.sample_function(SG_FN_QUAD, coef[g, :3 * dims[g]])
        nod = torch.empty(one.num_points, device=dev)
        one.get_values_device(nod)
        xg = torch.from_numpy(xs[coff[g]:coff[g + 1]].copy()).to(dev)
        og = torch.empty(int(counts[g]), device=dev)
        for rep in range(2):
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            one.set_values_device(nod, stream)
            one.hierarchize_async(stream)
            one.evaluate_device(xg, og, int(counts[g]), stream)
            s1.record(stream)
            s1.synchronize()
        plain_ms += s0.elapsed_time(s1)
        plain_pts += int(counts[g])
        one.close()
    plain_value = plain_pts / (plain_ms / 1e3)
    if rank != 0:
        return None
    err = None
    if world == 1 and not args.no_cpu_baseline:
        err = batch_error_vs_fp64(b, vals.cpu().numpy(), dims, levels, out.cpu().numpy(), xs, po, coff)
    hier_bytes = 8.0 * float(np.sum(np.array(npts) * dims))
    line = {
        "metric": "evals/s (batched grids)", "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64)",
        "config": {"workload": f"{len(dims)} grids, d in 2..12, n in 3..9, <= 2e6 points each, f = prod(a+bx+cx^2),"
                               f" 256..65536 log-uniform points per grid", "grids": len(dims),
                   "grid_points": int(sum(npts)), "query_points": total_pts, "hier_precision": args.precision,
                   "cuda_graphs": not args.no_graph},
        "hierarchize": {"ms": statistics.mean(th), "GB/s_8dN": hier_bytes / (statistics.mean(th) / 1e3) / 1e9,
                        "grids_per_s": len(dims) / (statistics.mean(th) / 1e3)},
        "evaluate": {"ms": statistics.mean(te), "evals_per_s": total_pts / (statistics.mean(te) / 1e3)},
        "plain_per_grid": {"evals_per_s": plain_value, "grids_sampled": len(sample),
                           "note": "one set_values/hierarchize/evaluate launch sequence per grid, summed"},
        "speedup_vs_plain": value / plain_value, "autotuned_by_d": tuned_ppt,
        "gpu_launches": int(launches), "clocks": clk.summary(),
    }
    if err is not None:
        line["err_vs_fp64"] = err
    b.close()
    return line


def batch_error_vs_fp64(b, nodal: np.ndarray, dims, levels, out: np.ndarray, xs: np.ndarray, po, coff,
                        per_d: int = 2, npts: int = 64):
    """Error of the batched results against the FP64 oracle (checker only):
    for `per_d` grids of every dimension, FP64 hierarchization of the grid's
    nodal values and FP64 evaluation at `npts` of its query points."""
    from oracle.oracle import Oracle
    worst_abs, worst_rel, worst_pt, checked = 0.0, 0.0, 0.0, 0
    for d in sorted(set(int(x) for x in dims)):
        for g in [int(i) for i in np.flatnonzero(dims == d)[:per_d]]:
            o = Oracle(d, int(levels[g]), None)
            s64 = o.hierarchize_f64(b.grid_values(nodal, g).astype(np.float64))
            m = int(po[g + 1] - po[g])
            idx = np.linspace(0, m - 1, min(npts, m)).astype(np.int64)
            Xg = xs[coff[g]:coff[g + 1]].reshape(m, d)
            u64 = o.evaluate_f64(s64, Xg[idx])
            e = np.abs(out[po[g]:po[g + 1]][idx].astype(np.float64) - u64)
            scale = max(float(np.max(np.abs(u64))), 1e-30)
            worst_abs = max(worst_abs, float(e.max()))
            worst_rel = max(worst_rel, float(e.max()) / scale)
            worst_pt = max(worst_pt, float(np.max(e / np.maximum(np.abs(u64), 1e-2 * scale))))
            checked += 1
    return {"grids": checked, "points_per_grid": npts, "max_abs": worst_abs, "max_norm_rel": worst_rel,
            "max_rel_floor1e-2": worst_pt,
            "note": "FP32 batched results vs FP64 hierarchize + evaluate of the same nodal values"}


def served_error_vs_fp64(served, gsrc, dims, levels, coef, npts: int = 256):
    """Served results against the FP64 oracle (checker only): each request's
    grid is sampled again on the device (the same kernel the server used),
    hierarchized and evaluated in FP64 at the request's first `npts` points."""
    from adaptive_sparse_grid_bench_b200 import Grid
    from adaptive_sparse_grid_bench_b200._lib import SG_FN_QUAD
    from oracle.oracle import Oracle
    worst_abs = worst_norm = worst_pt = 0.0
    for gid, X, out in served:
        k = gsrc[gid]
        d, n = int(dims[k]), int(levels[k])
        one = Grid(d, n)
        one.sample_function(SG_FN_QUAD, coef[k, :3 * d])
        nodal = one.get_values()
        one.close()
        o = Oracle(d, n)
        u64 = o.evaluate_f64(o.hierarchize_f64(nodal.astype(np.float64)), X[:npts])
        e = np.abs(out[:npts].astype(np.float64) - u64)
        scale = max(float(np.max(np.abs(u64))), 1e-30)
        worst_abs = max(worst_abs, float(e.max()))
        worst_norm = max(worst_norm, float(e.max()) / scale)
        worst_pt = max(worst_pt, float(np.max(e / np.maximum(np.abs(u64), 1e-2 * scale))))
    return {"requests": len(served), "points_per_request": npts, "max_abs": worst_abs, "max_norm_rel": worst_norm,
            "max_rel_floor1e-2": worst_pt}


def run_served(args, rank: int, world: int, local_rank: int):
    """Served workload: a pool of `--pool` resident grids drawn like the
    batched ones (seed 4) under a byte cap; at each swept rate a Poisson
    stream of `--requests` requests, 95% evaluate (random resident grid,
    log-uniform 1..65536 uniform points) and 5% create+hierarchize of a new
    grid (admitted by a separate thread, evicting LRU grids when the cap
    binds).  Latency = submit -> results in the caller's host buffer.  Then
    the same kind of requests as one burst (the server's capacity) and one
    plain sg_evaluate call per request (the arrangement without the server).
    One GPU: rank 0 serves, other ranks exit."""
    import queue
    import threading
    import torch
    from adaptive_sparse_grid_bench_b200 import Server, inputs
    from adaptive_sparse_grid_bench_b200._lib import SG_FN_QUAD, kernel_launches
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return None
    ngrid = args.pool
    dims, levels, coef, _ = inputs.batch_workload(4, ngrid)
    srv = Server(int(args.cap_gb * (1 << 30)), max_batch_points=max(args.batch_points, 65536))
    if args.zero_copy is not None:
        from adaptive_sparse_grid_bench_b200._lib import SG_SRV_OPT_ZERO_COPY
        srv.set_option(SG_SRV_OPT_ZERO_COPY, args.zero_copy)
    if args.heavy_pairs is not None:
        from adaptive_sparse_grid_bench_b200._lib import SG_SRV_OPT_HEAVY_PAIRS
        srv.set_option(SG_SRV_OPT_HEAVY_PAIRS, args.heavy_pairs)
    if args.sort_heavy is not None:
        from adaptive_sparse_grid_bench_b200._lib import SG_SRV_OPT_SORT_HEAVY
        srv.set_option(SG_SRV_OPT_SORT_HEAVY, args.sort_heavy)
    if args.light_slots is not None:
        from adaptive_sparse_grid_bench_b200._lib import SG_SRV_OPT_LIGHT_SLOTS
        srv.set_option(SG_SRV_OPT_LIGHT_SLOTS, args.light_slots)
    t0 = time.perf_counter()
    ids = [srv.add_grid(int(d), int(n), SG_FN_QUAD, coef[g, :3 * d]) for g, (d, n) in enumerate(zip(dims, levels))]
    admit_s = time.perf_counter() - t0
    gdim = {i: int(d) for i, d in zip(ids, dims)}
    gsrc = {gid: k for k, gid in enumerate(ids)}  # grid id -> its workload entry
    resident = list(ids)
    pool = inputs.uniform01(40, 65536 * 12 * 4)  # query coordinates: slices of one uniform stream
    u = inputs.uniform01(4, 64 * args.requests + 4096)
    draw = [0]

    def nxt():
        v = float(u[draw[0] % u.size])
        draw[0] += 1
        return v

    def coords(m, d):
        off = int(nxt() * (pool.size - m * d))
        return pool[off:off + m * d].reshape(m, d)

    def make_requests(nreq, create_frac):
        reqs = []
        for _ in range(nreq):
            if nxt() < create_frac:
                reqs.append(("create", int(nxt() * ngrid), None))
            else:
                gid = resident[int(nxt() * len(resident))]
                m = max(1, min(65536, int(round(np.exp(nxt() * np.log(65536.0))))))
                reqs.append(("eval", gid, coords(m, gdim[gid])))
        return reqs

    # warm-up: every grid once (loads every kernel the stream will use)
    for t in [srv.submit(g, coords(600, gdim[g])) for g in ids]:
        srv.wait(t)

    def serve(reqs, rate):
        creates = queue.Queue()
        new_ids, admit_ms, tickets = [], [], []

        def admitter():
            while True:
                g = creates.get()
                if g is None:
                    return
                a0 = time.perf_counter()
                try:
                    nid = srv.add_grid(int(dims[g]), int(levels[g]), SG_FN_QUAD, coef[g, :3 * dims[g]])
                except Exception:
                    continue
                admit_ms.append(1e3 * (time.perf_counter() - a0))
                gdim[nid] = int(dims[g])
                gsrc[nid] = g
                new_ids.append(nid)

        th = threading.Thread(target=admitter)
        th.start()
        if rate > 0:
            ut = inputs.uniform01(5, len(reqs), start=int(rate)).astype(np.float64)
            gaps = -np.log(np.maximum(1.0 - ut, 1e-12)) / rate
        else:
            gaps = np.zeros(len(reqs))
        rejected = 0
        start = time.perf_counter()
        t_next = start
        for (kind, g, X), gap in zip(reqs, gaps):
            t_next += gap
            while time.perf_counter() < t_next:
                pass
            if kind == "create":
                creates.put(g)
                continue
            try:
                tickets.append((srv.submit(g, X), g, X))
            except Exception:
                rejected += 1  # the grid was evicted after the request was drawn
        rows, pts = [], 0
        for t, g, X in tickets:
            _, tl = srv.wait_detail(t)
            rows.append((tl["take_ms"], tl["launch_ms"], tl["gpu_ms"], tl["latency_ms"], X.shape[0], tl["pairs"]))
            pts += X.shape[0]
        wall = time.perf_counter() - start
        creates.put(None)
        th.join()
        resident.extend(new_ids)
        tl = np.array(rows, np.float64).reshape(-1, 6)
        lat = tl[:, 3]
        small = lat[tl[:, 4] <= 4096]
        heavy = tl[:, 5] >= np.percentile(tl[:, 5], 90)  # the 10 % of requests with the most work
        if args.served_dump:
            np.save(f"{args.served_dump}_{rate if rate > 0 else 'burst'}.npy", tl)
        pct = lambda a, q: float(np.percentile(a, q)) if a.size else None  # noqa: E731
        return {"rate_req_s": rate if rate > 0 else "burst", "requests": len(tickets), "rejected": rejected,
                "evals_per_s": pts / wall, "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "max_ms": float(lat.max()),
                "p99_ms_le4096pts": pct(small, 99), "p99_ms_heaviest10pct": pct(lat[heavy], 99),
                "p99_ms_other90pct": pct(lat[~heavy], 99),
                "stages_p50_ms": {"queued": pct(tl[:, 0], 50), "staged": pct(tl[:, 1] - tl[:, 0], 50),
                                  "device": pct(tl[:, 2] - tl[:, 1], 50), "delivered": pct(tl[:, 3] - tl[:, 2], 50)},
                "stages_p99_ms": {"queued": pct(tl[:, 0], 99), "staged": pct(tl[:, 1] - tl[:, 0], 99),
                                  "device": pct(tl[:, 2] - tl[:, 1], 99), "delivered": pct(tl[:, 3] - tl[:, 2], 99)},
                "creates": len(new_ids), "admit_ms_mean": float(np.mean(admit_ms)) if admit_ms else None}

    sweep = []
    with Clocks(local_rank) as clk:
        l0 = kernel_launches()
        for rate in [float(r) for r in args.rates.split(",") if r]:
            sweep.append(serve(make_requests(args.requests, args.create_frac), rate))
        burst = serve(make_requests(args.requests, 0.0), 0.0)
        launches = kernel_launches() - l0

    # served results equal the plain single-grid call (a sample): bit for bit,
    # or within 1e-5 * max|u| + 2e-7 where the server split the sums
    from adaptive_sparse_grid_bench_b200 import SgError
    checked = bitwise = 0
    served = []
    for kind, g, X in make_requests(64, 0.0):
        try:
            out, _ = srv.wait(srv.submit(g, X))
            want = srv.evaluate_now(g, X)
        except SgError:
            continue  # evicted under a small cap
        bitwise += int(np.array_equal(out.view(np.uint32), want.view(np.uint32)))
        err = np.abs(out.astype(np.float64) - want)
        if not np.all(err <= 1e-5 * max(float(np.max(np.abs(want))), 1e-30) + 2e-7):
            raise RuntimeError("served and plain results differ")
        checked += 1
        served.append((g, X, out))
    err64 = served_error_vs_fp64(served[:8], gsrc, dims, levels, coef)

    # the same kind of requests, one plain sg_evaluate call each (buffers warmed first)
    plain = []
    for r in make_requests(min(args.requests, 1000), 0.0):
        try:
            srv.evaluate_now(r[1], r[2][:1])
            plain.append(r)
        except SgError:
            pass
    for g in {g for _, g, _ in plain}:
        srv.evaluate_now(g, coords(65536, gdim[g]))
    pp, pt, plat = 0, 0.0, []
    for _, g, X in plain:
        t1 = time.perf_counter()
        srv.evaluate_now(g, X)
        dt = time.perf_counter() - t1
        pp += X.shape[0]
        pt += dt
        plat.append(dt * 1e3)
    plain_rate = pp / pt
    st = srv.stats()
    srv.close()
    ok = [r for r in sweep if r["p99_ms"] <= 2.0]
    best = max(ok, key=lambda r: r["evals_per_s"]) if ok else None
    line = {
        "metric": "served evals/s (burst capacity)", "value": burst["evals_per_s"], "unit": "evals/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded SplitMix64)",
        "config": {"workload": f"{ngrid} resident grids (d 2..12, n 3..9, <= 2e6 points), Poisson arrivals, "
                               f"{100 - 100 * args.create_frac:g}% evaluate (1..65536 log-uniform points), "
                               f"{100 * args.create_frac:g}% create+hierarchize", "cap_gb": args.cap_gb,
                   "requests_per_rate": args.requests, "batch_points": max(args.batch_points, 65536),
                   "zero_copy": args.zero_copy, "heavy_pairs": args.heavy_pairs, "light_slots": args.light_slots,
                   "sort_heavy": args.sort_heavy},
        "sweep": sweep, "burst": burst,
        "best_rate_with_p99_le_2ms": best,
        "plain_per_request": {"evals_per_s": plain_rate, "requests": len(plain),
                              "p50_ms": float(np.percentile(plat, 50)), "p99_ms": float(np.percentile(plat, 99))},
        "speedup_vs_plain": burst["evals_per_s"] / plain_rate, "checked_vs_plain": checked, "bitwise_vs_plain": bitwise,
        "err_vs_fp64": err64, "admit_ms_per_grid_initial": 1e3 * admit_s / ngrid, "server_stats": st,
        "gpu_launches": int(launches), "clocks": clk.summary(),
    }
    return line


def free_port() -> int:
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_ranks(n: int, argv) -> int:
    """Starts this script as n local ranks (one process per GPU) through
    torch.distributed.run and returns its exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__), *argv]
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")  # the NCCL log names every rank of the communicator
    return subprocess.call(cmd, env=env)


def compact(line: dict | None, keys) -> dict | None:
    return None if line is None else {k: line[k] for k in keys if k in line}


def reference_gpu(g, X: np.ndarray, ours: np.ndarray, m: int = 1 << 18, nodal: np.ndarray | None = None) -> dict:
    """The reference's own CUDA evaluation kernel (evaluate5, cu:1522-1598,
    compiled in place by oracle/ref_cuda_harness.cu) on the same hierarchized
    grid and the first m query points, points per warp swept over the values
    its run script uses (run.sh:14-18).  kernel: its kernel alone; copies: its
    own timed region (coordinates in, kernel, results out, cu:1829-1897).
    With the nodal values, also its hierarchization (hierarchize7,
    cu:1053-1160, with the warp barriers it lacks added) of the whole grid:
    the median of 5 runs after one warm-up, and whether its surpluses are
    bit-identical to this library's."""
    from oracle.oracle import ReferenceCUDA
    if not ReferenceCUDA.available():
        return {"unavailable": "oracle/_ref/libasgb_refcuda.so not built"}
    surplus = g.get_values()
    Xm = np.ascontiguousarray(X[:m])
    sweep, best = {}, None
    for P in (32, 64, 128, 256):
        out, tk, tt = ReferenceCUDA.evaluate5(g.d, g.n, surplus, Xm, P, reps=2)
        sweep[P] = tk
        if best is None or tk < best[1]:
            best = (P, tk, tt, out)
    P, out = best[0], best[3]
    # the best P timed again: median of 5 single runs after warm-up
    runs = [ReferenceCUDA.evaluate5(g.d, g.n, surplus, Xm, P, reps=1)[1:] for _ in range(5)]
    tk = statistics.median(r[0] for r in runs)
    tt = statistics.median(r[1] for r in runs)
    scale = float(np.max(np.abs(ours[:m])))
    pairs = m * g.num_subspaces / (tk / 1e3)
    hier = None
    if nodal is not None and 6 <= g.n <= 10:
        hout = ReferenceCUDA.hierarchize7(g.d, g.n, nodal, reps=1)[0]
        hruns = [ReferenceCUDA.hierarchize7(g.d, g.n, nodal, reps=1)[1:] for _ in range(5)]
        hk = statistics.median(r[0] for r in hruns)
        ht = statistics.median(r[1] for r in hruns)
        hier = {"kernel": "reference hierarchize7 (cu:1053-1160), one launch per dimension",
                "kernel_ms": hk, "copies_ms": ht, "timing": "median of 5 runs",
                "gbs_kernel": 8.0 * g.d * g.num_points / (hk / 1e3) / 1e9, "bytes": "8*d*N",
                "ref_gflops_kernel": hi_gflops(g.d, g.num_points, hk),
                "bitexact_vs_b200": bool(np.array_equal(hout.view(np.uint32), surplus.view(np.uint32)))}
    return {"kernel": "reference evaluate5 (cu:1522-1598)", "hierarchize": hier, "points": m, "points_per_warp": P,
            "kernel_ms": tk, "copies_ms": tt, "timing": "median of 5 runs at the best points per warp",
            "evals_per_s_kernel": m / (tk / 1e3),
            "evals_per_s_copies": m / (tt / 1e3), "pairs_per_s_kernel": pairs,
            "ref_gflops_kernel": ev_gflops(g.d, pairs),
            "kernel_ms_by_points_per_warp": sweep,
            "max_abs_diff_vs_b200": float(np.max(np.abs(out.astype(np.float64) - ours[:m]))),
            "max_abs_b200": scale}


def run_extras(args, rank: int, world: int, local_rank: int) -> dict:
    """Short runs of the other workloads for the N=1 default line: the
    batched step on 1024 grids, the served sweep at four rates with 3000
    requests each, and the limits-adaptive grid; each with its error against
    the FP64 oracle."""
    import copy
    out = {}
    a = copy.copy(args)
    a.steps, a.warmup = min(args.steps, 10), 3
    a.grids = 1024
    out["batched"] = compact(run_batched(a, rank, world, local_rank),
                             ["value", "unit", "ms_per_step", "config", "hierarchize", "evaluate", "plain_per_grid",
                              "speedup_vs_plain", "autotuned_by_d", "err_vs_fp64", "gpu_launches"])
    a = copy.copy(args)
    a.rates, a.requests = "16000,20000,24000,28000", 3000
    srv = run_served(a, rank, world, local_rank)
    if srv is not None:
        srv = compact(srv, ["value", "unit", "sweep", "burst", "best_rate_with_p99_le_2ms", "plain_per_request",
                            "speedup_vs_plain", "checked_vs_plain", "bitwise_vs_plain", "err_vs_fp64"])
        for r in srv.get("sweep", []) + [srv.get("burst") or {}]:
            for k in ("creates", "admit_ms_mean", "rejected", "max_ms"):
                r.pop(k, None)
    out["served"] = srv
    a = copy.copy(args)
    a.steps, a.warmup, a.no_e2e, a.no_cpu_baseline, a.points = min(args.steps, 10), 3, True, True, None
    out["adaptive"] = compact(run_b200(a, rank, world, local_rank, adaptive_workload(a), err=True),
                              ["value", "unit", "ms_per_step", "config", "hierarchize", "evaluate", "err_vs_fp64",
                               "autotune_ms", "gpu_launches"])
    return out


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args.gpus, sys.argv[1:]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but {world} rank(s) were started")
    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "batched":
            line = run_batched(args, rank, world, local_rank)
        elif args.workload == "served":
            line = run_served(args, rank, world, local_rank)
        elif args.workload == "adaptive":
            line = run_b200(args, rank, world, local_rank, adaptive_workload(args))
        else:
            extras = world == 1 and not args.no_extras
            line = run_b200(args, rank, world, local_rank, extras=extras)
            if line is not None and extras:
                line.update(run_extras(args, rank, world, local_rank))
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
