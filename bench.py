"""Benchmark of the PageRank hot path (one JSON line on rank 0).

Default workload (the headline): plain PageRank on a directed R-MAT scale-25
graph (33,554,432 vertices, edgefactor 16, a/b/c/d 0.57/0.19/0.19/0.05,
seed 2, self-loops and duplicates removed), edge weights i.i.d. U(0,1] FP32
with weighted out-degree normalisation, alpha 0.85.  A step is one full solve
of SWEEPS sweeps with tol = 0 (the reference's stop rule, tol 1e-7 here, ends
a scale-25 solve after one sweep, so throughput is measured at a fixed sweep
count): set-up, SWEEPS fused sweeps, the FP64 correction sweep and the
normalisation.  value = GTEPS per sweep = nnz * SWEEPS / step time, summed
over ranks (replicas: every rank solves its own copy; scaling "weak").

The line also carries: the roofline of the sweep kernel, the end-to-end rate
through the drop-in C ABI entry (host CSR in page-locked and in pageable
memory), parity against the FP64 oracle (stop rule at the config's tolerance
and fixed 10-sweep solves), the reference's own cuSPARSE GPU solve timed on
the same graph, the oracle's OpenMP restatement of the reference's CPU path
timed on the host, the scale-22 config (R-MAT scale 22, seed 1, unweighted)
measured the same way as a secondary object, and (one GPU) the batched-PPR
config (R-MAT scale 20, k=256 seed sets) and the serving config (Poisson
arrivals over 64 graphs, and long solves on one large graph, each with and
without session-level continuous batching), each measured after the timed
region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat25w|rmat22|rmat<scale>[w]|ppr|batch|serving|precision25]

--impl reference times the reference's own CPU algorithm for the path (the
oracle's port of cpp_easygraph's OpenMP _pagerank, all host threads) on the
same workload and prints the same metric.
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PageRank GTEPS/iter + HBM GB/s; PPR solves/s and p99 at L1 err ≤1e-6"
L2_BYTES = 126 * 2**20
SWEEPS = 20


def _rank_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(dist, vals, device):
    """Each value's maximum over the ranks of the process group (the values
    themselves on a single process): a multi-GPU time is the slowest rank's."""
    if not dist:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(world, units_per_rank, seconds):
    """Units all ranks processed (each rank does the same work) per second of the slowest rank."""
    return world * units_per_rank / seconds


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel_file):
    """dram bytes per launch recorded by an ncu capture summary under profiles/."""
    p = ROOT / "profiles" / kernel_file
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_launch_full:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = [x.strip() for x in vis.split(",")] if vis else None
        self.index = ids[local_rank] if ids and local_rank < len(ids) else str(local_rank)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.index], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline_port(csr, alpha, budget_s=10.0):
    """The oracle's port of the reference's OpenMP CPU PageRank, timed on this host."""
    from oracle import oracle

    threads = oracle.max_threads()
    sweeps_done, t_total = 0, 0.0
    while t_total < budget_s or sweeps_done < 2:
        t0 = time.perf_counter()
        _, sw = oracle.cpu_pagerank_omp(csr.V, csr.E, csr.W, alpha=alpha, max_iter=2, threshold=0.0, threads=threads)
        t_total += time.perf_counter() - t0
        sweeps_done += sw
    return {"value": csr.m * sweeps_done / t_total / 1e9, "unit": "GTEPS/iter", "cores": threads, "kind": "port",
            "label": "restatement",
            "sample": f"{sweeps_done} sweeps of the same graph in solves of 2 sweeps (tol 0), "
                      f"{t_total:.1f} s: the oracle's FP64 OpenMP restatement of the reference's CPU PageRank "
                      "(push with atomic adds, cpp_easygraph/functions/pagerank/pagerank.cpp:21-122) over the "
                      "same CSR"}


def make_workload(name):
    """rmat<scale>[w]: the R-MAT graphs of the configs (scale 22: seed 1, unweighted;
    scale 25: seed 2, weighted); other scales (smaller profiling cases) use seed 2."""
    from eggpu_b200 import synth

    m = re.fullmatch(r"rmat(\d+)(w?)", name)
    if not m:
        raise SystemExit(f"unknown workload {name}")
    scale, weighted = int(m.group(1)), m.group(2) == "w"
    if not 10 <= scale <= 26:
        raise SystemExit(f"R-MAT scale {scale} out of range [10, 26]")
    seed = 1 if scale == 22 else 2
    csr = synth.rmat(scale=scale, edgefactor=16, seed=seed, weighted=weighted)
    desc = (f"R-MAT scale {scale} ({1 << scale:,} vertices, edgefactor 16, a/b/c/d 0.57/0.19/0.19/0.05, "
            f"seed {seed}, self-loops and duplicates removed, "
            + ("weights i.i.d. U(0,1] FP32, weighted out-degree normalisation" if weighted else "unweighted")
            + "), alpha 0.85")
    return csr, desc


def run_reference(args):
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    from oracle import oracle

    csr, desc = make_workload(args.workload)
    threads = oracle.max_threads()
    sweeps = 2
    for _ in range(args.warmup):
        oracle.cpu_pagerank_omp(csr.V, csr.E, csr.W, alpha=0.85, max_iter=1, threshold=0.0, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, sw = oracle.cpu_pagerank_omp(csr.V, csr.E, csr.W, alpha=0.85, max_iter=sweeps, threshold=0.0,
                                        threads=threads)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    value = csr.m * sweeps / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS/iter", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}", "n": csr.n, "nnz": csr.m, "sweeps_per_step": sweeps,
                   "tol": 0.0},
        "cpu_baseline": {"value": value, "unit": "GTEPS/iter", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} solves of {sweeps} sweeps on the full graph; OpenMP port of "
                                   "cpp_easygraph/functions/pagerank/pagerank.cpp:21-122 (the reference's C++ "
                                   "CPU PageRank needs pybind11/CPython to build, so the port is timed)"},
        "e2e": {"value": value, "unit": "GTEPS/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_tol(name):
    """The stop-rule tolerance of the workload's config: 1e-7 for the scale-25
    precision config, 1e-6 otherwise."""
    return 1e-7 if name.startswith("rmat25") else 1e-6


def time_solves(pg, stream, steps, warmup, sweeps, dist):
    """Device time of `steps` whole solves of `sweeps` sweeps (tol 0) and of
    steps//2 solves of 2*sweeps, CUDA events on the solve's stream, max over
    ranks.  Returns (t_step, t_sweep, stats, stats2)."""
    import torch

    def timed(k, n_sweeps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k):
            pg.enqueue(alpha=0.85, max_iter=n_sweeps, tol=0.0)
        e1.record(stream)
        torch.cuda.synchronize()
        _, st = pg.collect(copy=False)
        return e0.elapsed_time(e1) / k / 1e3, st

    for _ in range(max(warmup, 3)):
        pg.enqueue(alpha=0.85, max_iter=sweeps, tol=0.0)
    pg.collect(copy=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_step, st = timed(steps, sweeps)
    t_step2, st2 = timed(max(1, steps // 2), 2 * sweeps)
    torch.cuda.synchronize()
    t_step, t_step2 = max_over_ranks(dist, [t_step, t_step2], "cuda")
    if dist:
        dist.barrier()
    return t_step, max((t_step2 - t_step) / sweeps, 1e-9), st, st2


def measure_e2e(csr, sweeps, steps, rank, world, dist, pinned=True):
    """Whole solves through the drop-in C ABI entry egpr_pagerank_csr, every
    step: H2D of the host CSR, GPU preparation, `sweeps` sweeps, D2H of the
    FP64 ranks.  pinned: the CSR sits in page-locked memory; otherwise in
    ordinary (pageable) numpy arrays, which the library stages itself."""
    import torch

    from eggpu_b200 import _native

    if pinned:
        V = torch.from_numpy(csr.V).pin_memory().numpy()
        E = torch.from_numpy(csr.E).pin_memory().numpy()
        W = None if csr.W is None else torch.from_numpy(csr.W).pin_memory().numpy()
    else:
        V, E, W = csr.V, csr.E, csr.W
    PR = _native.pinned_empty(csr.n)  # the caller's result vector, reused across calls
    _native.cache_reset()
    _native.pagerank_csr(V, E, W, 10**9 + rank, 0.85, sweeps, 0.0, out=PR)  # warm the code path
    _native.cache_reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        _native.pagerank_csr(V, E, W, 2 * 10**9 + i, 0.85, sweeps, 0.0, out=PR)
        _native.cache_reset()  # the next step prepares the graph again
    t = (time.perf_counter() - t0) / steps
    (t,) = max_over_ranks(dist, [t], "cuda")
    nnz = int(np.count_nonzero((csr.E >= 0) & (csr.E < csr.n)))
    h2d = csr.V.nbytes + csr.E.nbytes + (0 if csr.W is None else csr.W.nbytes)
    return {"value": whole_job_rate(world, nnz * sweeps, t) / 1e9, "unit": "GTEPS/iter",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(8 * csr.n), "ms_per_step": t * 1e3,
            "steps": steps,
            "path": "egpr_pagerank_csr (drop-in for gpu_easygraph::pagerank): H2D of the out-edge CSR from "
                    + ("page-locked" if pinned else "pageable") + " host memory, GPU preparation, "
                    f"{sweeps} sweeps, FP64 correction, D2H of FP64 ranks into the caller's page-locked result "
                    "vector, every step"}


def parity_vs_oracle(pg, csr, tol):
    """The reference's stop rule at the config's tolerance, and fixed 10-sweep
    solves with and without the FP64 correction sweep, against the FP64
    oracle (iterations, L1 and max-abs error)."""
    from oracle import oracle

    inbound = oracle.build_inbound(csr.V, csr.E, csr.W)
    out = {}
    for label, max_iter, t, corr in ((f"rule_tol{tol:g}", 100, tol, True), ("fixed10", 10, 0.0, True),
                                     ("fixed10_no_correction", 10, 0.0, False)):
        ranks, st = pg.pagerank(alpha=0.85, max_iter=max_iter, tol=t, correction=corr)
        ref, it, _ = oracle.pagerank_pull(csr.V, csr.E, csr.W, alpha=0.85, max_iter=max_iter, tol=t,
                                          inbound=inbound)
        out[label] = {"iterations": st["iterations"], "oracle_iterations": it,
                      "l1_vs_fp64_oracle": float(np.abs(ranks - ref).sum()),
                      "max_abs_vs_fp64_oracle": float(np.abs(ranks - ref).max()),
                      "solve_ms": st["kernel_seconds"] * 1e3}
    return out


def reference_gpu_baseline(csr, sweeps, ours_sweep_ms, ours_e2e_ms):
    """The reference's own GPU solve on the same graph and box: cuda_pagerank
    (cuSPARSE CSR SpMV + cuBLAS dot + two kernels and two host round trips per
    sweep, gpu_easygraph/functions/centrality/pagerank.cu:352-713), compiled
    for sm_100a from the reference sources into oracle/_ref.  Its per-sweep
    time is read from its own CUDA events around the sweep loop
    (pagerank.cu:578,666-676): (T(2S) - T(S)) / S on the warm workspace."""
    from oracle import oracle

    if not oracle.ref_available():
        return {"unavailable": "oracle/_ref/libref_pagerank.so not built (needs the reference tree at build time)"}
    t0 = time.perf_counter()
    oracle.ref_cuda_pagerank(csr.V, csr.E, csr.W, 0.85, sweeps, 0.0)  # cold: host transpose, H2D, set-up
    cold = time.perf_counter() - t0
    _, ks1 = oracle.ref_cuda_pagerank(csr.V, csr.E, csr.W, 0.85, sweeps, 0.0)  # warm: cached device graph
    _, ks2 = oracle.ref_cuda_pagerank(csr.V, csr.E, csr.W, 0.85, 2 * sweeps, 0.0)
    per_sweep = max((ks2 - ks1) / sweeps, 1e-9)
    nnz = int(np.count_nonzero((csr.E >= 0) & (csr.E < csr.n)))
    return {"impl": "reference cuda_pagerank (cuSPARSE CSR_ALG2 SpMV + cublasSdot), sm_100a build",
            "sweep_ms": per_sweep * 1e3, "gteps_per_iter": nnz / per_sweep / 1e9,
            "loop_ms_for_sweeps": ks1 * 1e3, "sweeps": sweeps,
            "cold_call_ms": cold * 1e3,
            "cold_call_note": "one call on a new graph: host-side inbound CSR build, H2D, cuSPARSE set-up, "
                              f"{sweeps} sweeps, D2H and host normalisation (wall clock)",
            "ours_over_reference_sweep_speedup": per_sweep * 1e3 / ours_sweep_ms,
            "ours_e2e_over_reference_cold_call_speedup": (cold * 1e3 / ours_e2e_ms) if ours_e2e_ms else None}


def measure_workload(name, args, rank, world, local, dist, sweeps, with_e2e=True, e2e_pageable=False):
    """One workload on this rank: prepared graph, autotuned layout, timed solves,
    roofline and end-to-end legs.  Returns (csr, desc, pg, result dict)."""
    import torch

    from eggpu_b200 import _native

    csr, desc = make_workload(name)
    pg = _native.PreparedGraph(csr.V, csr.E, csr.W)
    nnz = pg.nnz
    # the sweep layout chosen by the per-graph tuner, before any timing (a
    # long-lived prepared graph is tuned once)
    tuning = pg.tuning() if args.no_autotune else pg.autotune(sweep=True, spmm=False)
    stream = torch.cuda.Stream()
    pg.set_stream(stream.cuda_stream)
    with ClockSampler(local) as clk:
        t_step, t_sweep, st, st2 = time_solves(pg, stream, args.steps, args.warmup, sweeps, dist)
    pg.set_stream(None)
    bytes_per_iter = st["bytes_per_iter"]
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_iter / t_sweep / 1e9
    res = {
        "value": whole_job_rate(world, nnz * sweeps, t_step) / 1e9,
        "ms_per_step": t_step * 1e3,
        "config": {"workload": f"{name}: {desc}", "n": csr.n, "nnz": int(nnz), "sweeps_per_step": sweeps,
                   "tol": 0.0, "parallelism": f"replicas{world}",
                   "l2": f"inputs larger than L2 (inbound CSR {(4 * (csr.n + 1) + 4 * nnz) / 1e6:.0f} MB > "
                         f"{L2_BYTES / 1e6:.0f} MB), no flush between steps",
                   "precision": "FP32 ranks and products; FP64 residual, dangling mass and rank sums; final FP64 "
                                "correction sweep",
                   "layout": {"chunks_per_warp": tuning["chunks_per_warp"], "row_cost": tuning["row_cost"],
                              "chosen_by": "defaults (--no-autotune)" if args.no_autotune
                              else "egpr_graph_autotune before timing"}},
        "hbm_gbs": bytes_per_iter * sweeps / t_step / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profile_traffic(f"k_sweep_{name}.md"),
                     "kernel": "k_sweep<float> (fused sweep)", "peak_source": peak_kind,
                     "bytes_per_launch": bytes_per_iter, "launch_ms": t_sweep * 1e3,
                     "timing": "CUDA events on the launch stream; per-sweep time = (T(2S) - T(S)) / S"},
        "gpu_launches": int(st["launches"] * args.steps + st2["launches"] * max(1, args.steps // 2)),
        "gpu_launches_per_step": st["launches"],
        "clocks": clk.summary(),
    }
    if with_e2e and not args.no_e2e:
        e2e_steps = max(2, min(args.steps, 5))
        res["e2e"] = measure_e2e(csr, sweeps, e2e_steps, rank, world, dist, pinned=True)
        if e2e_pageable:
            res["e2e_pageable"] = measure_e2e(csr, sweeps, e2e_steps, rank, world, dist, pinned=False)
    return csr, desc, pg, res


def run_ours(args):
    import torch

    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", device_id=torch.device("cuda", local),
                                    timeout=datetime.timedelta(seconds=600))
        dist = dist_mod
    sweeps = args.sweeps
    csr, desc, pg, res = measure_workload(args.workload, args, rank, world, local, dist, sweeps,
                                          e2e_pageable=not args.no_pageable)
    secondary = None
    if args.secondary and args.secondary != args.workload:
        _, _, pg2, sec = measure_workload(args.secondary, args, rank, world, local, dist, sweeps)
        pg2.close()
        secondary = {k: sec[k] for k in ("value", "ms_per_step", "config", "hbm_gbs", "roofline", "e2e",
                                         "gpu_launches_per_step") if k in sec}
    parity = ref_gpu = cpu = None
    if rank == 0 and not args.no_parity:
        parity = parity_vs_oracle(pg, csr, workload_tol(args.workload))
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_baseline(csr, sweeps, res["roofline"]["launch_ms"],
                                         res.get("e2e", {}).get("ms_per_step"))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(csr, 0.85, budget_s=args.cpu_seconds)
    # the batched-PPR and serving configs, measured after the timed region
    ppr = served = None
    if rank == 0 and world == 1 and args.with_ppr:
        got = measure_ppr(args)
        if got is not None:
            ppr = {"config": got[1], **got[0]}
    if rank == 0 and world == 1 and args.with_serving:
        out, cfg = measure_serving(args)
        served = {"config": cfg, **out}
    if rank == 0:
        line = {"metric": METRIC, "value": res["value"], "unit": "GTEPS/iter", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": res["config"], "hbm_gbs": res["hbm_gbs"],
                "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res.get("e2e"),
                "e2e_pageable": res.get("e2e_pageable"), "gpu_launches": res["gpu_launches"],
                "gpu_launches_per_step": res["gpu_launches_per_step"], "clocks": res["clocks"],
                "parity": parity, "reference_gpu": ref_gpu, "secondary": secondary, "ppr": ppr,
                "serving": served}
        print(json.dumps(line), flush=True)
    pg.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _ppr_teleport(n, s):
    p = np.zeros(n)
    p[np.unique(s)] = 1.0
    return p / p.sum()


def run_ppr(args):
    """Batched PPR (R-MAT scale 20, seed 3, k=256 seed sets of 1-64 vertices) against
    k plain single-vector solves on the same GPU; accuracy against the FP64 oracle."""
    import torch

    torch.cuda.set_device(0)
    res = measure_ppr(args)
    if res is None:
        return
    out, cfg = res
    line = {"metric": METRIC, "value": out["rule"]["batched_solves_per_s_e2e"], "unit": "PPR solves/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic", "dtype": "f32", "config": cfg, "ppr": out}
    print(json.dumps(line), flush=True)


def measure_ppr(args):
    from eggpu_b200 import _native, synth
    from oracle import oracle

    g = synth.rmat(scale=20, edgefactor=16, seed=3)
    sets = synth.seed_sets(g.n, 256, 1, 64, seed=3)
    pg = _native.PreparedGraph(g.V, g.E)
    if args.ppr_profile:  # a short case for a profiler: warm-up solve, then the profiled one
        k = int(args.ppr_profile)
        for _ in range(2):
            _, sts = pg.pagerank_seeds(sets[:k], alpha=0.85, max_iter=4, tol=0.0)
        print(json.dumps({"ppr_profile": {"k": k, "sweeps": 4, "device_ms": sts[0]["kernel_seconds"] * 1e3}}))
        return None
    out = {}
    res = _native.pinned_empty((len(sets), g.n))  # the result array a serving caller keeps and reuses
    for label, max_iter, tol in (("rule", 100, 1e-6), ("fixed20", 20, 0.0)):
        pg.pagerank_seeds(sets, alpha=0.85, max_iter=max_iter, tol=tol, out=res)  # warm-up
        t0 = time.perf_counter()
        reps = max(1, args.steps // 50)
        for _ in range(reps):
            ranks, sts = pg.pagerank_seeds(sets, alpha=0.85, max_iter=max_iter, tol=tol, out=res)
        wall = (time.perf_counter() - t0) / reps
        dev = sts[0]["kernel_seconds"]
        sample = list(range(0, 256, 32))
        t0 = time.perf_counter()
        dev_single = 0.0
        for j in sample:
            _, st = pg.pagerank(alpha=0.85, max_iter=max_iter, tol=tol, personalization=_ppr_teleport(g.n, sets[j]))
            dev_single += st["kernel_seconds"]
        wall_single = (time.perf_counter() - t0) / len(sample)
        dev_single /= len(sample)
        errs = []
        for j in sample[:4]:
            ref, it, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=max_iter, tol=tol,
                                              teleport=_ppr_teleport(g.n, sets[j]))
            errs.append((float(np.abs(ranks[j] - ref).sum()), float(np.abs(ranks[j] - ref).max()),
                         sts[j]["iterations"], it))
        out[label] = {
            "batched_solves_per_s_device": 256 / dev, "batched_solves_per_s_e2e": 256 / wall,
            "plain_solves_per_s_device": 1 / dev_single, "plain_solves_per_s_e2e": 1 / wall_single,
            "speedup_device": (256 / dev) / (1 / dev_single), "speedup_e2e": (256 / wall) / (1 / wall_single),
            "iterations": sts[0]["iterations"], "batch_device_ms": dev * 1e3, "batch_wall_ms": wall * 1e3,
            "max_l1_vs_fp64_oracle": max(e[0] for e in errs), "max_abs_vs_fp64_oracle": max(e[1] for e in errs),
            "iterations_vs_oracle": [(e[2], e[3]) for e in errs],
            "bytes_per_sweep_ppr": sts[0]["bytes_per_iter"],
        }
    cfg = {"workload": "ppr: R-MAT scale 20 (seed 3, edgefactor 16), k=256 teleport vectors uniform over seed sets "
                       "of 1-64 vertices (numpy PCG64 seed 3), alpha 0.85; 'rule' = tol 1e-6 max_iter 100, 'fixed20' = "
                       "20 sweeps", "n": g.n, "nnz": pg.nnz}
    for label in out:  # per-sweep device time of the batched solve (k = 256: eight 32-column panels)
        out[label]["batch_sweep_ms"] = out[label]["batch_device_ms"] / max(1, out[label]["iterations"])
    pg.close()
    return out, cfg


def run_batch(args):
    """512 independent Erdos-Renyi graphs in one persistent launch per sweep vs one solve per graph."""
    import torch

    from eggpu_b200 import _native, synth

    torch.cuda.set_device(0)
    rng = np.random.Generator(np.random.PCG64(1000))
    count = 512
    ns = np.exp(rng.uniform(np.log(1e3), np.log(2e5), size=count)).astype(np.int64)
    ds = rng.uniform(8.0, 32.0, size=count)
    graphs, nnz = [], 0
    for i in range(count):
        c = synth.erdos_renyi(int(ns[i]), float(ds[i]), seed=1000 + i)
        pg = _native.PreparedGraph(c.V, c.E)
        nnz += pg.nnz
        graphs.append(pg)
    _native.pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6)
    # median over repetitions: an occasional call costs several times the
    # others (host page faults of the fresh result block)
    walls = []
    for _ in range(max(5, args.steps // 20)):
        t0 = time.perf_counter()
        outs, sts = _native.pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6)
        walls.append(time.perf_counter() - t0)
    wall = statistics.median(walls)
    dev = sts[0]["kernel_seconds"]
    its = [s["iterations"] for s in sts]
    t0 = time.perf_counter()
    dev_single = 0.0
    for pg in graphs:
        _, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
        dev_single += st["kernel_seconds"]
    wall_single = time.perf_counter() - t0
    sweeps_edges = sum(pg.nnz * it for pg, it in zip(graphs, its))
    line = {"metric": METRIC, "value": count / wall, "unit": "graph solves/s", "higher_is_better": True,
            "n_gpus": 1, "data": "synthetic", "dtype": "f32",
            "config": {"workload": "batch: 512 directed Erdos-Renyi graphs, n log-uniform in [1e3, 2e5], mean "
                                   "out-degree uniform in [8, 32] (numpy PCG64 seed 1000), graph seeds 1000-1511, "
                                   "alpha 0.85, tol 1e-6", "total_nnz": int(nnz)},
            "batch": {"multi_solves_per_s_e2e": count / wall, "multi_solves_per_s_device": count / dev,
                      "plain_solves_per_s_e2e": count / wall_single, "plain_solves_per_s_device": count / dev_single,
                      "speedup_e2e": wall_single / wall, "speedup_device": dev_single / dev,
                      "multi_device_ms": dev * 1e3, "multi_wall_ms": wall * 1e3,
                      "iterations_min_max": [min(its), max(its)], "gteps_device": sweeps_edges / dev / 1e9}}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Poisson arrivals (1000 req/s, 50/50 PageRank/PPR with 1-16 seeds) over 64 R-MAT graphs
    (n log-uniform in [1e3, 1e7], edgefactor uniform in [8, 32], seeds 2000-2063)."""
    import torch

    torch.cuda.set_device(0)
    out, cfg = measure_serving(args)
    line = {"metric": METRIC, "value": out["solves_per_s"], "unit": "solves/s", "higher_is_better": True,
            "n_gpus": 1, "data": "synthetic", "dtype": "f32", "config": cfg, "serving": out}
    print(json.dumps(line), flush=True)


def quiet_gc():
    """Before a measured replay: collect, then move every live object (the
    load generator's request lists, futures and locks among them) out of the
    collector's reach, so that a full collection over them does not land
    inside the replay as a pause of the serving threads."""
    gc.collect()
    gc.freeze()


def measure_serving(args):
    from eggpu_b200 import _native, serving, synth

    rng = np.random.Generator(np.random.PCG64(2000))
    count = 64
    max_n = int(args.serving_max_n)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(max_n), size=count)).astype(np.int64)
    efs = rng.integers(8, 33, size=count)
    src = {}
    for i in range(count):
        scale = int(np.ceil(np.log2(ns[i])))
        c = synth.rmat(scale=scale, edgefactor=int(efs[i]), seed=2000 + i, keep_n=int(ns[i]))
        src[i] = (c.V, c.E, None)
    n_req = int(args.serving_requests)
    kinds = rng.random(n_req) < 0.5
    gids = rng.integers(0, count, size=n_req)
    reqs = []
    for k, gid in zip(kinds, gids):
        n = src[int(gid)][0].shape[0] - 1
        # a served result is handed over and dropped (not kept by the load generator)
        if k:
            reqs.append(serving.Request(int(gid), "pr", keep_result=False))
        else:
            size = int(rng.integers(1, 17))
            reqs.append(serving.Request(int(gid), "ppr", seeds=rng.choice(n, min(size, n), replace=False),
                                        keep_result=False))
    budget = int(args.serving_hbm_gb * 2**30)
    reg = serving.GraphRegistry(src, budget_bytes=budget)
    warm_s = reg.warm(range(count))  # graphs are loaded before traffic starts
    workers = int(os.environ.get("EGPR_SERVING_WORKERS", "4"))
    times = serving.poisson_arrivals(1000.0, n_req, seed=2001)
    # steady state: a warm-up burst of every request (host and device memory
    # pools grown, every graph's batched layout built) before any measured
    # replay, so neither mode pays first-use costs the other does not
    n_warm = n_req
    warm = [serving.Request(r.graph, r.kind, seeds=r.seeds, keep_result=False) for r in reqs]
    srv_w = serving.Server(reg, workers=workers)
    serving.replay(srv_w, warm, np.zeros(n_req))
    srv_w.close()
    # ... then the first 2,000 arrivals at their own times (the result sizes
    # of single requests, whose page-locked buffers the burst did not ask for)
    warm = [serving.Request(r.graph, r.kind, seeds=r.seeds, keep_result=False) for r in reqs[:2000]]
    srv_w = serving.Server(reg, workers=workers)
    serving.replay(srv_w, warm, times[:2000])
    srv_w.close()
    srv = serving.Server(reg, workers=workers)
    quiet_gc()
    wall = serving.replay(srv, reqs, times)
    srv.close()
    lat = serving.latency_summary(reqs)
    # the same arrivals with one-shot batching only (no egpr_session; the
    # default server opens sessions only for long solves on large graphs,
    # which this traffic has not)
    again = [serving.Request(r.graph, r.kind, seeds=r.seeds, keep_result=False) for r in reqs]
    srv1 = serving.Server(reg, workers=workers, sessions=False)
    quiet_gc()
    wall1 = serving.replay(srv1, again, times)
    srv1.close()
    lat_one_shot = serving.latency_summary(again)
    # capacity: the same requests all at once (queued requests fold into batched solves)
    burst = [serving.Request(r.graph, r.kind, seeds=r.seeds, keep_result=False) for r in reqs]
    srv2 = serving.Server(reg, workers=workers)
    quiet_gc()
    burst_wall = serving.replay(srv2, burst, np.zeros(n_req))
    srv2.close()
    burst1 = [serving.Request(r.graph, r.kind, seeds=r.seeds, keep_result=False) for r in reqs]
    srv3 = serving.Server(reg, workers=workers, sessions=False)
    quiet_gc()
    burst1_wall = serving.replay(srv3, burst1, np.zeros(n_req))
    srv3.close()
    long_solves = measure_long_solves(workers)
    # plain unbatched per-request solves of a sample, on the same GPU
    sample = reqs[:: max(1, n_req // 200)]
    plain_lat = []
    for r in sample:
        pg = reg.acquire(r.graph)
        try:
            t0 = time.perf_counter()
            if r.kind == "pr":
                pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
            else:
                pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=_ppr_teleport(pg.n, r.seeds))
            plain_lat.append(time.perf_counter() - t0)
        finally:
            reg.release(r.graph)
    plain = np.array(plain_lat)
    cfg = {"workload": "serving: Poisson arrivals at 1000 req/s, 50/50 PageRank/PPR (1-16 seeds), 64 "
                       f"R-MAT graphs n log-uniform in [1e3, {max_n:.0e}] (ids >= n dropped), edgefactor "
                       "uniform in [8, 32], seeds 2000-2063, alpha 0.85, tol 1e-6",
           "requests": n_req, "hbm_budget_gb": args.serving_hbm_gb,
           "warmup": f"a burst of all {n_warm} requests, then the first 2,000 at their arrival times, before the "
                     "measured replays",
           "gc": "Python's collector run and live objects frozen before each measured replay",
           "graphs_loaded_before_traffic_s": warm_s,
           "total_nnz": int(sum(len(v[1]) for v in src.values()))}
    out = {"latency": lat, "solves_per_s": n_req / wall, "offered_req_per_s": 1000.0,
           "server_stats": dict(srv.stats), "admissions": reg.admissions, "evictions": reg.evictions,
           "one_shot": {"latency": lat_one_shot, "solves_per_s": n_req / wall1, "server_stats": dict(srv1.stats)},
           "capacity_burst": {"solves_per_s": n_req / burst_wall, "wall_s": burst_wall,
                              "server_stats": dict(srv2.stats),
                              "one_shot": {"solves_per_s": n_req / burst1_wall, "wall_s": burst1_wall,
                                           "server_stats": dict(srv3.stats)}},
           "plain_unbatched_service_ms": {"p50": float(np.percentile(plain, 50) * 1e3),
                                          "p99": float(np.percentile(plain, 99) * 1e3),
                                          "mean": float(plain.mean() * 1e3)},
           "plain_unbatched_capacity_solves_per_s": float(1.0 / plain.mean()),
           "long_solves": long_solves}
    reg.close()
    return out, cfg


def measure_long_solves(workers):
    """Long solves on a large graph, where slot-level continuous batching
    pays: fixed-sweep PPR requests (100 sweeps, tol 0, 1-16 seeds) at 200 req/s
    on one R-MAT scale-20 graph (seed 3, edgefactor 16), served by the default
    server (which runs them in an egpr_session) and with one-shot batched
    solves only."""
    from eggpu_b200 import serving, synth

    c = synth.rmat(scale=20, edgefactor=16, seed=3)
    reg = serving.GraphRegistry({0: (c.V, c.E, None)}, budget_bytes=16 << 30)
    reg.warm([0])
    n = c.V.shape[0] - 1
    rng = np.random.Generator(np.random.PCG64(6))
    seeds = [rng.choice(n, int(rng.integers(1, 17)), replace=False) for _ in range(2000)]
    times = serving.poisson_arrivals(200.0, len(seeds), seed=7)
    out = {"config": "R-MAT scale 20 (seed 3, edgefactor 16), 2000 PPR requests of 100 sweeps (tol 0) with 1-16 "
                     "seeds (numpy PCG64 seed 6), Poisson arrivals at 200 req/s (seed 7), after a warm-up replay "
                     "of 300 requests; Python's collector run and live objects frozen before each measured replay"}
    for label, sessions in (("default", True), ("one_shot", False)):
        warm = [serving.Request(0, "ppr", seeds=s, tol=0.0, max_iter=100, keep_result=False) for s in seeds[:300]]
        srv = serving.Server(reg, workers=workers, sessions=sessions)
        serving.replay(srv, warm, times[:300])
        srv.close()
        reqs = [serving.Request(0, "ppr", seeds=s, tol=0.0, max_iter=100, keep_result=False) for s in seeds]
        srv = serving.Server(reg, workers=workers, sessions=sessions)
        quiet_gc()
        wall = serving.replay(srv, reqs, times)
        srv.close()
        out[label] = {"latency": serving.latency_summary(reqs), "solves_per_s": len(reqs) / wall,
                      "server_stats": dict(srv.stats)}
    reg.close()
    return out


def run_precision25(args):
    """R-MAT scale 25 weighted (seed 2), tol 1e-7: error of the engine against the FP64 oracle."""
    import torch

    from eggpu_b200 import _native, synth
    from oracle import oracle

    torch.cuda.set_device(0)
    g = synth.rmat(scale=25, edgefactor=16, seed=2, weighted=True)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    res = {}
    for label, max_iter, tol, corr in (("rule_tol1e-7", 100, 1e-7, True), ("fixed10", 10, 0.0, True),
                                       ("fixed10_no_correction", 10, 0.0, False)):
        ranks, st = pg.pagerank(alpha=0.85, max_iter=max_iter, tol=tol, correction=corr)
        ref, it, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=max_iter, tol=tol)
        res[label] = {"iterations": st["iterations"], "oracle_iterations": it,
                      "l1_vs_fp64_oracle": float(np.abs(ranks - ref).sum()),
                      "max_abs_vs_fp64_oracle": float(np.abs(ranks - ref).max()),
                      "solve_ms": st["kernel_seconds"] * 1e3}
    ranks, st = pg.pagerank(alpha=0.85, max_iter=20, tol=0.0)
    gteps = pg.nnz * 20 / st["kernel_seconds"] / 1e9
    line = {"metric": METRIC, "value": gteps, "unit": "GTEPS/iter", "higher_is_better": True, "n_gpus": 1,
            "data": "synthetic", "dtype": "f32",
            "config": {"workload": "rmat25w: R-MAT scale 25 (seed 2, edgefactor 16), weights U(0,1] FP32, alpha 0.85",
                       "n": g.n, "nnz": pg.nnz},
            "precision": res, "hbm_gbs_20_sweeps": st["bytes_per_iter"] * 20 / st["kernel_seconds"] / 1e9}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="rmat25w",
                    help="rmat<scale>[w] (rmat25w: the scale-25 weighted config, rmat22: the scale-22 config), "
                         "ppr, batch, serving, precision25")
    ap.add_argument("--secondary", default="rmat22",
                    help="a second plain-PageRank workload measured the same way and reported inside the line "
                         "('' for none)")
    ap.add_argument("--sweeps", type=int, default=SWEEPS)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-pageable", action="store_true", help="skip the end-to-end leg from pageable memory")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own cuSPARSE solve on the same graph")
    ap.add_argument("--with-ppr", action=argparse.BooleanOptionalAction, default=True,
                    help="plain-PageRank workloads: also measure the batched-PPR config (R-MAT 20, k=256) and "
                         "report it inside the line")
    ap.add_argument("--with-serving", action=argparse.BooleanOptionalAction, default=True,
                    help="plain-PageRank workloads: also run the serving config and report it inside the line")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default sweep layout (a profiler then sees only the timed launches)")
    ap.add_argument("--serving-max-n", type=float, default=1e7)
    ap.add_argument("--serving-requests", type=int, default=10000)
    ap.add_argument("--serving-hbm-gb", type=float, default=64.0)
    ap.add_argument("--ppr-profile", type=int, default=0, metavar="K",
                    help="ppr workload: only two batched solves of K columns and 4 sweeps (a case for ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ppr":
        run_ppr(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "precision25":
        run_precision25(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
