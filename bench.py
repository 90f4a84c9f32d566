"""Benchmark: PageRank GTEPS per iteration on R-MAT scale 24 (directed,
weighted), mixed FP32 + FP64-refined path versus the all-FP64 GPU path, both
to the reference's stopping rule at L1 change <= 1e-9.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: R-MAT scale 24, edge factor 16 (2^28 draws), a/b/c/d =
0.57/0.19/0.19/0.05, self-loops and duplicate arcs removed, lognormal(0, 1)
arc strengths rounded to FP32; PageRank with damping 0.85, uniform teleport,
dangling nodes jumping by the teleport vector, weights as strengths, tol 1e-9.
The graph is generated on the device from seeded Philox streams (synthetic;
no dataset). A step is one PageRank solve.

Metric: GTEPS per iteration = arcs / (solve time / sweeps) / 1e9.
- `value`: the mixed path with the graph resident in HBM (device time of the
  solve, CUDA events on the library's stream).
- `e2e`: the same call through the C ABI with host buffers: the teleport
  vector is copied from pinned host memory and the scores back to pinned
  host memory inside the timed region.
- `roofline`: the dominant kernel (the sweep kernel the per-operator tuner
  picked, normally the sliced sweep; FP32, anchor, refinement and FP64
  sweeps reported separately), its algorithmic bytes per launch over its
  average CUDA-event duration, against the measured HBM copy bandwidth.
- `cpu_baseline`: the oracle's restatement of the reference's multithreaded
  CPU PageRank iteration (oracle/), timed on this host's cores on a bounded
  sample of the same workload.
With --impl reference the reference arm runs instead: the CPU restatement
(the Rust reference cannot be built here) times whole calls of the
reference's net_pagerank (per-call set-up and every iteration) on the same
graph, generated by the oracle's own generators.

Multi-GPU (torchrun, one process per GPU): this line runs independent
replicas of the same solve; value is the arcs all ranks processed per
iteration-second, timed as the maximum over ranks. `--workload rows` splits
one solve of the same graph by rows instead (net_shard_*: each rank sweeps
its rows, one NCCL all-gather of the payloads per sweep, every rank finishes
the sweep over all nodes). The batched (c4a) and packed-graph (c4b)
workloads shard with no exchange: under torchrun each rank solves its
contiguous share of teleport vectors or graphs, the slowest rank's device
time is reported, and the scores are gathered on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PageRank GTEPS/iter & % HBM peak, R-MAT 24: mixed vs FP64 at L1≤1e-9"
UNIT = "GTEPS/iter"
SCALE, EDGE_FACTOR, A, B, C = 24, 16, 0.57, 0.19, 0.19
SEED, WSEED = 20240601, 20240602
DAMPING, TOL = 0.85, 1e-9


# sweep kernels by their tuning code (net_set_tuning key 4)
KERNEL_NAMES = {
    8: "warp_spmv (merge-path warp tiles on the layout renumbered by column count, 16 warps "
       "per CTA)",
    9: "slice_spmv (sliced layout: long rows by whole warps, the others one lane per row in "
       "32-row slices; 48 resident warps per SM, 4 arcs per lane in flight)",
    10: "slice_spmv (sliced layout, 64 resident warps per SM, 4 arcs per lane in flight)",
    11: "slice_spmv (sliced layout, one 32-warp CTA per SM, most gathered values in shared "
        "memory)",
    12: "slice_bulk_spmv (sliced layout, arc streams staged in shared memory by bulk copies, "
        "32 resident warps per SM)",
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    from knappnet_b200 import ranks
    if n_gpus <= 1 and "WORLD_SIZE" not in os.environ:
        return 0, 1, 0, None
    return ranks.init("nccl", timeout_s=300.0)


def barrier(dist):
    from knappnet_b200 import ranks
    ranks.barrier(dist)


def max_over_ranks(dist, x: float) -> float:
    from knappnet_b200 import ranks
    return ranks.max_over_ranks(dist, x)


def sum_over_ranks(dist, x: float) -> float:
    from knappnet_b200 import ranks
    return ranks.sum_over_ranks(dist, x)


def make_graph(scale: int = SCALE):
    import knappnet_b200 as K
    g = K.generate_rmat(scale, EDGE_FACTOR, A, B, C, seed=SEED, clean=True, symmetrize=False,
                        lognormal=True, wseed=WSEED)
    K.device_sync()
    return g


def pinned(n: int):
    """A pinned host float64 array of n values (torch pinned memory)."""
    import torch
    t = torch.empty(n, dtype=torch.float64, pin_memory=True)
    return t, t.numpy()


def cpu_sample(g, budget_s: float, full_iters: int):
    """The oracle's PageRank iteration on this host (all cores), on the same
    pull operator, for about `budget_s` seconds: returns (GTEPS/iter, cores,
    iterations, seconds)."""
    from oracle import oracle as O
    off, cols, w = g.csr(1)
    # out-strength = column sums of the pull operator (the graph has no loops)
    outs = g.degree(mode=1, loops=True, weighted=True)
    cores = O.threads_for(0, g.n, len(cols) // 2)
    secs1, _ = O.pagerank_time_op(off, cols, w, outs, DAMPING, 1, 0)
    iters = int(max(1, min(full_iters, budget_s / max(secs1, 1e-3))))
    secs, _ = O.pagerank_time_op(off, cols, w, outs, DAMPING, iters, 0)
    return len(cols) * iters / secs / 1e9, cores, iters, secs


def run_ours(args):
    import knappnet_b200 as K
    rank, world, local, dist = dist_setup(args.gpus)
    hbm, peak_kind = peaks()
    g = make_graph(args.scale)
    n, m = g.n, g.m

    import torch
    # scores stay in device memory for the device-resident measurements
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")

    def solve(precision):
        return g.pagerank_device(d_out.data_ptr(), DAMPING, True, True, None, 0, 0, TOL, 0,
                                 precision)

    # FP64 solve on the GPU (the all-FP64 path) and its timing
    K.set_sweep_timing(True)
    for _ in range(max(1, args.warmup // 2)):
        info64 = solve(K.PREC_FP64)
    t64 = []
    for _ in range(max(2, args.steps // 2)):
        info64 = solve(K.PREC_FP64)
        t64.append(info64.seconds)
    x64 = d_out.cpu().numpy()
    sw64 = K.sweep_timing(1)

    # warm-up of the measured (mixed) path
    for _ in range(args.warmup):
        infom = solve(K.PREC_MIXED)

    # timed region: K mixed solves, device-resident graph and scores
    with ClockSampler(local) as clocks:
        barrier(dist)
        torch.cuda.synchronize()
        wall0 = time.perf_counter()
        dev_s, sweeps, launches = 0.0, 0, 0
        sw32_ms = sw32_n = sw64m_ms = sw64m_n = swr_ms = swr_n = 0.0
        for _ in range(args.steps):
            infom = solve(K.PREC_MIXED)
            dev_s += infom.seconds
            sweeps += infom.iterations
            launches += infom.kernel_launches
            a = K.sweep_timing(0)
            b = K.sweep_timing(1)
            c = K.sweep_timing(2)
            sw32_n += a[0]
            sw32_ms += a[1]
            sw64m_n += b[0]
            sw64m_ms += b[1]
            swr_n += c[0]
            swr_ms += c[1]
            bytes32, bytes64, bytesr = a[2], b[2], c[2]
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        barrier(dist)
    xm = d_out.cpu().numpy()
    dev_s = max_over_ranks(dist, dev_s)
    total_arcs_iters = sum_over_ranks(dist, float(m) * sweeps)
    value = total_arcs_iters / dev_s / 1e9

    # end to end through the C ABI with host buffers (pinned)
    tp, p_host = pinned(n)
    p_host[:] = 1.0 / n
    to, out_host = pinned(n)
    for _ in range(max(1, args.warmup // 2)):
        g.pagerank_ex(DAMPING, True, True, p_host, 0, 0, TOL, 0, K.PREC_MIXED, out=out_host)
    barrier(dist)
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    e_sweeps = 0
    for _ in range(args.steps):
        xe, infoe = g.pagerank_ex(DAMPING, True, True, p_host, 0, 0, TOL, 0, K.PREC_MIXED,
                                  out=out_host)
        e_sweeps += infoe.iterations
    torch.cuda.synchronize()
    e_wall = max_over_ranks(dist, time.perf_counter() - e0)
    e2e_value = sum_over_ranks(dist, float(m) * e_sweeps) / e_wall / 1e9

    # accuracy of the mixed path against the all-FP64 path (which matches
    # the CPU oracle to 1e-12 L1 in the tests)
    l1 = float(np.abs(xm - x64).sum())
    linf = float(np.abs(xm - x64).max())
    top64 = np.argsort(-x64, kind="stable")[:100]
    topm = np.argsort(-xm, kind="stable")[:100]
    fp64_time = statistics.median(t64)
    mixed_time = dev_s / args.steps

    def roof(ms, cnt, nbytes):
        if cnt <= 0:
            return None
        dur = ms / cnt * 1e-3
        ach = nbytes / dur / 1e9
        return {"achieved": round(ach, 1), "duration_ms": round(dur * 1e3, 4),
                "launches": int(cnt), "bytes_per_launch": nbytes, "frac": round(ach / hbm, 4)}

    r32 = roof(sw32_ms, sw32_n, bytes32)
    r64m = roof(sw64m_ms, sw64m_n, bytes64)
    rr = roof(swr_ms, swr_n, bytesr)
    r64 = roof(sw64[1], sw64[0], sw64[2])
    # dominant kernel of the measured path: the sweep kind with most time
    kname = KERNEL_NAMES.get(infom.sweep_kernel, f"sweep kernel {infom.sweep_kernel}")
    kdesc = (f"{kname}; long rows from {infom.long_row} arcs" if infom.long_row else kname) + \
        f"; gathers of the {infom.hot_columns:,} most gathered columns allocate in L1"
    kinds = [(sw32_ms, r32, "fp32", "FP32 sweep: " + kdesc),
             (swr_ms, rr, "refine", "refinement sweep (FP32 gathers of the correction, FP64 "
                                  "update): " + kdesc),
             (sw64m_ms, r64m, "fp64", "FP64 sweep: " + kdesc)]
    _, dom, dom_kind, dom_name = max(kinds, key=lambda k: k[0])
    traffic = None
    tfile = ROOT / "profiles" / "sweep_traffic.json"
    if tfile.exists():
        tdoc = json.loads(tfile.read_text())
        if dom_kind in tdoc:
            traffic = tdoc[dom_kind].get("bytes_per_launch_full_scale")

    # The gather bound: random 4-byte loads per second from an array the size
    # of the FP32 iterate (L2-resident), measured on this GPU after the timed
    # region. Gathers that miss L1 (the ncu capture's hit rate) go to L2.
    gather_rate = K.measure_gather(0, n)
    hit = None
    if tfile.exists():
        hit = json.loads(tfile.read_text()).get("fp32", {}).get("l1_sector_hit_rate_scale22")
    gather = {"l2_gathers_per_s": round(gather_rate, 0), "gathers_per_sweep": m,
              "array": f"{n:,} FP32 values, the size of the FP32 iterate",
              "all_from_l2_ms": round(m / gather_rate * 1e3, 4)}
    if hit is not None and r32:
        l2_ms = m * (1.0 - hit) / gather_rate * 1e3
        gather.update({"l1_hit_rate_ncu": hit, "l1_misses_from_l2_ms": round(l2_ms, 4),
                       "fp32_sweep_frac_of_gather_bound": round(l2_ms / r32["duration_ms"], 4)})

    clock = clocks.summary()
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dev_s / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
        "data": "synthetic (R-MAT generated on the device from seeded Philox streams)",
        "config": {"workload": f"R-MAT scale {args.scale}, edge factor 16, a/b/c/d=.57/.19/.19/.05, "
                               "directed, loops and duplicates removed, lognormal(0,1) FP32 "
                               "strengths; PageRank d=0.85, uniform teleport, tol 1e-9 (L1)",
                   "nodes": n, "arcs": m,
                   "precision": "mixed (FP32 sweeps; one FP64 anchor sweep; refinement sweeps "
                                "gathering the FP32 correction, FP64 update)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (arc arrays 2.1 GB per sweep)"},
        "gpu_launches": launches,
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "ms_per_step": round(e_wall / args.steps * 1e3, 3)},
        "roofline": {"bound": "hbm", "kernel": dom_name,
                     "achieved": dom["achieved"] if dom else None, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": dom["frac"] if dom else None, "traffic": traffic,
                     "fp32_sweep": r32, "fp64_sweep_in_mixed": r64m, "refine_sweep": rr,
                     "fp64_path_sweep": r64, "gather_bound": gather},
        "clocks": clock,
        "fp64_path": {"value": round(float(m) * info64.iterations / fp64_time / 1e9, 3),
                      "time_to_solution_ms": round(fp64_time * 1e3, 3),
                      "sweeps": info64.iterations},
        "sweep_kernel": {"mixed": {"kernel": int(infom.sweep_kernel),
                                   "long_row": int(infom.long_row),
                                   "hot_columns": int(infom.hot_columns)},
                         "fp64": {"kernel": int(info64.sweep_kernel),
                                  "long_row": int(info64.long_row),
                                  "hot_columns": int(info64.hot_columns)},
                         "picked_by": "per-operator timing of the candidates on the first "
                                      "solve (warm-up)"},
        "mixed_path": {"time_to_solution_ms": round(mixed_time * 1e3, 3),
                       "sweeps": infom.iterations, "fp32_sweeps": infom.iterations_fp32,
                       "speedup_vs_fp64": round(fp64_time / mixed_time, 3),
                       "l1_vs_fp64": l1, "linf_vs_fp64": linf,
                       "top100_identical": bool(np.array_equal(top64, topm))},
        "wall_s_timed": round(wall, 3),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        gteps, cores, iters, secs = cpu_sample(g, args.cpu_budget, info64.iterations)
        line["cpu_baseline"] = {"value": round(gteps, 4), "unit": UNIT, "cores": cores,
                                "kind": "port",
                                "sample": f"{iters} reference PageRank iterations (FP64, "
                                          f"serial scalar passes, threaded row-block SpMV) on "
                                          f"the same operator, {secs:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def oracle_graph(scale: int = SCALE):
    """The benchmark graph made by the oracle's restatement of the generators
    (same Philox streams, same cleaning, lognormal strengths within one FP32
    ulp of the device's), so the reference arm runs without the library."""
    from oracle import oracle as O
    src, tgt = O.rmat(scale, EDGE_FACTOR, A, B, C, SEED, clean=True)
    w = O.lognormal(len(src), WSEED).astype(np.float64)
    return 1 << scale, src, tgt, w


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's net_pagerank
    (oracle/: per-call operator set-up, threaded row-block products, serial
    scalar passes, the reference's stopping rule) on this host's cores. Each
    step is one whole call: set-up plus every iteration to tol 1e-9. Only
    rank 0 runs; the library is never loaded."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    from oracle import oracle as O
    t0 = time.perf_counter()
    n, s, t, w = oracle_graph(args.scale)
    og = O.Graph(n, s, t, w, True)
    build_s = time.perf_counter() - t0
    m = len(s)
    del s, t, w
    cores = O.threads_for(0, n, m // 2)
    # A CPU solve has no warm-up effects beyond first touch; one warm-up
    # solve (at most args.warmup) keeps the arm within a few minutes.
    warm = min(args.warmup, 1)
    for _ in range(warm):
        og.pagerank(DAMPING, True, True, None, 0, 0, TOL, 0, 0)
    times, iters = [], 0
    for _ in range(args.steps):
        t1 = time.perf_counter()
        og.pagerank(DAMPING, True, True, None, 0, 0, TOL, 0, 0)
        times.append(time.perf_counter() - t1)
        iters = og.last_iters
    total = sum(times)
    value = m * iters * args.steps / total / 1e9
    sample = (f"one whole net_pagerank call per step (operator set-up and all {iters} "
              f"iterations to tol {TOL:g}); graph generation and build {build_s:.1f} s excluded")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": warm,
            "ms_per_step": round(total / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (the same R-MAT graph, made by the oracle's generators)",
            "config": {"workload": f"R-MAT scale {args.scale}, edge factor 16, a/b/c/d=.57/.19/.19/.05, "
                                   "directed, loops and duplicates removed, lognormal(0,1) FP32 "
                                   "strengths; PageRank d=0.85, uniform teleport, tol 1e-9 (L1)",
                       "nodes": n, "arcs": m, "iterations": iters,
                       "parallelism": f"{cores} CPU threads"},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- other configurations
# One JSON line per configuration, for the workloads the benchmark line does
# not cover: device time (median of `--steps` runs after `--warmup`),
# accuracy against the CPU restatement of the reference (oracle/), and the
# restatement's time on this host where it finishes in a bounded sample.

def _median_device(fn, steps, warmup):
    for _ in range(warmup):
        fn()
    return statistics.median(fn() for _ in range(max(steps, 1)))


def run_c1(args):
    """ER G(10,000, 50,000) undirected, FP64 PageRank at tol 1e-12."""
    import knappnet_b200 as K
    from oracle import oracle as O
    s, t = K.generate_gnm(10_000, 50_000, False, False, seed=20240701)
    g = K.Graph(10_000, s, t, None, False)
    og = O.Graph(10_000, s, t, None, False)
    last = {}

    def gpu():
        x, info = g.pagerank_ex(tol=1e-12, precision=K.PREC_FP64)
        last["x"], last["it"] = x, info.iterations
        return info.seconds
    sec = _median_device(gpu, args.steps, args.warmup)
    t0 = time.perf_counter()
    ref = og.pagerank(tol=1e-12)
    cpu = time.perf_counter() - t0
    return {"workload": "c1: ER G(n=10000, m=50000) undirected, PageRank FP64, tol 1e-12",
            "metric": "solve ms", "value": round(sec * 1e3, 4), "unit": "ms",
            "higher_is_better": False, "iterations": last["it"],
            "oracle_iterations": og.last_iters,
            "l1_vs_oracle": float(np.abs(last["x"] - ref).sum()),
            "cpu_restatement_ms": round(cpu * 1e3, 3),
            "cores": O.threads_for(0, 10_000, 50_000)}


def run_c2(args):
    """Symmetrised R-MAT 20, eigenvector centrality by Lanczos, tol 1e-10:
    FP64 products against FP32 products with FP64 reorthogonalisation."""
    import knappnet_b200 as K
    from oracle import oracle as O
    g = K.generate_rmat(20, 16, seed=20240702, clean=True, symmetrize=True)
    out = {"workload": "c2: R-MAT 20 symmetrised (a/b/c/d .57/.19/.19/.05, cleaned), "
                       "eigenvector centrality mode all, Lanczos, tol 1e-10",
           "nodes": g.n, "edges": g.m}
    res = {}
    for prec in (0, 1):
        keep = {}

        def gpu():
            x, info = g.eigenvector_ex(mode=3, tol=1e-10, precision=prec)
            keep["x"], keep["info"] = x, info
            return info.seconds
        sec = _median_device(gpu, args.steps, args.warmup)
        res[prec] = (sec, keep["x"], keep["info"])
    s, t, _ = g.edges()
    og = O.Graph(g.n, s, t, None, False)
    t0 = time.perf_counter()
    ox, olam, _ = og.eigenvector(mode=3, tol=1e-10)
    cpu = time.perf_counter() - t0
    for prec, name in ((0, "fp64"), (1, "fp32_products")):
        sec, x, info = res[prec]
        out[name] = {"ms": round(sec * 1e3, 3), "matvecs": int(info.iterations),
                     "matvecs_fp32": int(info.iterations_fp32),
                     "eigenvalue": info.eigenvalue,
                     "eigenvalue_rel_vs_oracle": abs(info.eigenvalue - olam) / olam,
                     "linf_vs_oracle": float(np.abs(x - ox).max()),
                     "l1_vs_oracle": float(np.abs(x - ox).sum())}
    out.update({"metric": "Lanczos solve ms (FP32 products)", "value": out["fp32_products"]["ms"],
                "unit": "ms", "higher_is_better": False,
                "cpu_restatement_ms": round(cpu * 1e3, 1),
                "cores": O.threads_for(0, g.n, g.m)})
    return out


def run_c4a(args):
    """R-MAT 22 directed, 256 personalisation vectors (1-64 seeds each), one
    batched solve, mixed precision (another scale with --scale, for
    profiling captures)."""
    import knappnet_b200 as K
    from oracle import oracle as O
    scale = args.scale if args.scale != SCALE else 22
    g = K.generate_rmat(scale, 16, seed=20240703, clean=True)
    n, B = g.n, 256
    rng = np.random.default_rng(20240704)
    P = np.zeros((B, n))
    for b in range(B):
        k = int(rng.integers(1, 65))
        P[b, rng.choice(n, size=k, replace=False)] = 1.0 / k
    keep = {}

    def gpu():
        x, info = g.pagerank_batch(P, precision=K.PREC_MIXED, tol=1e-10)
        keep["x"], keep["info"] = x, info
        return info.seconds
    sec = _median_device(gpu, args.steps, args.warmup)
    info = keep["info"]
    # the same solve with teleport vectors and scores in device memory: the
    # device time of the solve and of its sweeps alone
    import torch
    dP = torch.from_numpy(P).cuda()
    dX = torch.empty_like(dP)
    dev = {}

    def gpu_dev():
        i = g.pagerank_batch_device(dP.data_ptr(), B, dX.data_ptr(), precision=K.PREC_MIXED,
                                    tol=1e-10)
        dev["info"] = i
        return i.seconds
    dsec = _median_device(gpu_dev, args.steps, args.warmup)
    dinfo = dev["info"]
    same = bool(np.array_equal(dX.cpu().numpy(), keep["x"]))
    del dP, dX
    s, t, _ = g.edges()
    og = O.Graph(n, s, t, None, True)
    errs, cpu = [], 0.0
    for b in (0, 1):
        t0 = time.perf_counter()
        ref = og.pagerank(personalization=P[b], tol=1e-10)
        cpu += time.perf_counter() - t0
        errs.append(float(np.abs(keep["x"][b] - ref).sum()))
    arcs = int(g.csr(1)[0][-1])
    hbm, peak_kind = peaks()
    # Algorithmic bytes of the sweeps, each array counted once: every sweep
    # reads the row offsets, the column indices and the gathered n x B block
    # (4 or 8 bytes a value, all columns: a node's B values are one run);
    # each column still active in a sweep also reads its previous iterate
    # and writes its new iterate and scaled iterate (3 n values). Converged
    # columns are left alone, so active column-sweeps come from the solve's
    # own counts per phase.
    s32, s64 = int(dinfo.sweeps_fp32), int(dinfo.sweeps - dinfo.sweeps_fp32)
    c32 = int(dinfo.column_iterations_fp32)
    c64 = int(dinfo.column_iterations) - c32
    refined = bool(dinfo.refined)
    base = 4.0 * (n + 1) + 4.0 * arcs  # row offsets and column indices, every sweep
    if refined:
        # the FP64 phase: one anchor sweep (FP64 gathers; y_ref read, s_ref,
        # e and z_e written: 24 bytes a node and column) and refinement sweeps
        # (FP32 gathers; y_ref, s_ref and e read, e and z_e written: 28 bytes)
        alg64 = (base + 8.0 * n * B + B * 24.0 * n +
                 (s64 - 1) * (base + 4.0 * n * B) + (c64 - B) * 28.0 * n)
        rows64 = (base + 8.0 * arcs * B + B * 24.0 * n +
                  (s64 - 1) * (base + 4.0 * arcs * B) + (c64 - B) * 28.0 * n)
    else:
        alg64 = s64 * (base + 8.0 * n * B) + c64 * 24.0 * n
        rows64 = s64 * (base + 8.0 * arcs * B) + c64 * 24.0 * n
    alg = s32 * (base + 4.0 * n * B) + c32 * 12.0 * n + alg64
    ach = alg / dinfo.sweep_seconds / 1e9
    # The same sweeps if every arc's gathered row (B values) came from DRAM,
    # as it must when the n x B iterate (4.3 GB in FP32) cannot stay in L2:
    # what the kernel moves, against the bandwidth.
    rows = s32 * (base + 4.0 * arcs * B) + c32 * 12.0 * n + rows64
    ach_rows = rows / dinfo.sweep_seconds / 1e9
    return {"workload": f"c4a: R-MAT {scale} directed, 256 personalisation vectors (uniform over "
                        "1-64 seed nodes), batched SpMM PageRank, mixed precision, tol 1e-10",
            "device_pointers": {"solve_ms": round(dsec * 1e3, 2),
                                "sweeps_ms": round(dinfo.sweep_seconds * 1e3, 2),
                                "gteps_b_per_sweep": round(arcs * B * dinfo.sweeps /
                                                           dinfo.sweep_seconds / 1e9, 2),
                                "same_scores_as_host_call": same,
                                "fp64_phase": ("one anchor sweep, then refinement sweeps gathering "
                                               "the FP32 correction" if refined else
                                               "FP64 sweeps"),
                                "roofline": {
                                    "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                                    "peak_kind": peak_kind, "unit": "GB/s",
                                    "frac": round(ach / hbm, 4),
                                    "bytes_per_sweep_avg": round(alg / max(dinfo.sweeps, 1)),
                                    "bytes": "offsets, indices and the gathered n x B block per "
                                             "sweep; previous, new and scaled iterate of each "
                                             "active column",
                                    "with_row_gathers": {
                                        "achieved": round(ach_rows, 1),
                                        "frac": round(ach_rows / hbm, 4),
                                        "bytes": "as above, but one gathered row of B values per "
                                                 "arc instead of the n x B block once"}}},
            "metric": "GTEPS*B per sweep", "unit": "GTEPS*B/sweep", "higher_is_better": True,
            "value": round(arcs * B * info.sweeps / sec / 1e9, 2),
            "solve_ms": round(sec * 1e3, 2),
            "sweeps_ms": round(info.sweep_seconds * 1e3, 2),
            "gteps_b_per_sweep_device": round(arcs * B * info.sweeps / info.sweep_seconds / 1e9, 2),
            "sweeps": int(info.sweeps),
            "sweeps_fp32": int(info.sweeps_fp32), "arcs": arcs,
            "l1_vs_oracle_sampled_columns": errs,
            "cpu_restatement_ms_per_vector": round(cpu / 2 * 1e3, 1),
            "cpu_restatement_ms_all_vectors_estimated": round(cpu / 2 * B * 1e3, 0),
            "cores": O.threads_for(0, n, arcs // 2)}


def run_c4b(args):
    """10,000 ego graphs, power-law sizes 50-50,000, mean degree 12, one
    persistent launch."""
    import knappnet_b200 as K
    from oracle import oracle as O
    sizes = K.power_law_sizes(10_000, 2.1, 50, 50_000, seed=20240705)
    m = np.minimum(6 * sizes, sizes * (sizes - 1) // 2)
    src, tgt = K.generate_gnm(sizes, m, False, False, seed=20240706)
    off = np.concatenate([[0], np.cumsum(sizes)])
    g = K.Graph(int(off[-1]), src, tgt, None, False)
    keep = {}

    def gpu():
        out, its, info = g.pagerank_graphs(off, tol=1e-12)
        keep["x"], keep["its"], keep["info"] = out, its, info
        return info.seconds
    sec = _median_device(gpu, args.steps, args.warmup)
    # the restatement, graph by graph, on a sample of 200 graphs, scaled by
    # nodes plus arcs
    rng = np.random.default_rng(9)
    pick = rng.choice(len(sizes), 200, replace=False)
    cpu, work, worst = 0.0, 0, 0.0
    for k in pick:
        lo, hi = off[k], off[k + 1]
        sel = (src >= lo) & (src < hi)
        og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, None, False)
        t0 = time.perf_counter()
        ref = og.pagerank(tol=1e-12)
        cpu += time.perf_counter() - t0
        work += int(hi - lo) + 2 * int(sel.sum())
        worst = max(worst, float(np.abs(keep["x"][lo:hi] - ref).sum()))
    total_work = int(off[-1]) + 2 * int(m.sum())
    return {"workload": "c4b: 10,000 undirected G(n, 6n) ego graphs, sizes power law "
                        "(exponent 2.1) on [50, 50000], PageRank FP64 tol 1e-12, one launch",
            "metric": "batch ms", "value": round(sec * 1e3, 3), "unit": "ms",
            "higher_is_better": False, "nodes": int(off[-1]), "edges": int(m.sum()),
            "kernel_launches": int(keep["info"].kernel_launches),
            "launch_graph_instantiations": int(keep["info"].long_row),
            "threads_per_cta": int(keep["info"].sweep_kernel),
            "ctas_per_cluster": int(keep["info"].hot_columns),
            "graphs_split_over_clusters": int(keep["info"].iterations_fp32),
            "max_iterations": int(keep["its"].max()),
            "l1_vs_oracle_worst_of_200": worst,
            "cpu_restatement_ms_estimated": round(cpu * total_work / work * 1e3, 1),
            "cores": 1}


def run_c4a_ranks(args):
    """C4a on N GPUs (torchrun, one process per GPU): the 256 teleport
    vectors split into contiguous column ranges (ranks.split_columns), each
    rank solving its range on its own copy of the graph with no exchange;
    the scores are then gathered on rank 0, which checks sampled columns
    against the oracle. Total work is fixed as N grows (strong scaling)."""
    import torch
    import knappnet_b200 as K
    from knappnet_b200 import ranks
    from oracle import oracle as O
    rank, world, local, dist = dist_setup(args.gpus)
    scale = args.scale if args.scale != SCALE else 22
    g = K.generate_rmat(scale, 16, seed=20240703, clean=True)
    n, B = g.n, 256
    rng = np.random.default_rng(20240704)
    P = np.zeros((B, n))
    for b in range(B):
        k = int(rng.integers(1, 65))
        P[b, rng.choice(n, size=k, replace=False)] = 1.0 / k
    ranges = [ranks.split_columns(B, world, r) for r in range(world)]
    lo, hi = ranges[rank]
    dP = torch.from_numpy(P[lo:hi].copy()).cuda()
    dX = torch.empty_like(dP)
    keep = {}

    def gpu():
        i = g.pagerank_batch_device(dP.data_ptr(), hi - lo, dX.data_ptr(),
                                    precision=K.PREC_MIXED, tol=1e-10)
        keep["info"] = i
        return i.seconds
    for _ in range(args.warmup):
        gpu()
    ranks.barrier(dist)
    times = [gpu() for _ in range(max(args.steps, 1))]
    sec = max_over_ranks(dist, statistics.median(times))
    arcs = int(g.csr(1)[0][-1])
    units = sum_over_ranks(dist, float(arcs) * (hi - lo) * keep["info"].sweeps)
    X = ranks.gather_rows(dist, dX, ranges)
    line = None
    if rank == 0:
        s_, t_, _ = g.edges()
        og = O.Graph(n, s_, t_, None, True)
        errs = [float(np.abs(X[b] - og.pagerank(personalization=P[b], tol=1e-10)).sum())
                for b in (0, ranges[-1][0], B - 1)]
        line = {"workload": f"c4a on {world} GPUs: R-MAT {scale} directed, 256 personalisation "
                            "vectors split by contiguous column ranges, no exchange; scores "
                            "gathered on rank 0 after the timed solves",
                "metric": "GTEPS*B per sweep", "unit": "GTEPS*B/sweep",
                "higher_is_better": True, "value": round(units / sec / 1e9, 2),
                "solve_ms_slowest_rank": round(sec * 1e3, 2), "n_gpus": world,
                "scaling": "strong", "columns_per_rank": [h - l for l, h in ranges],
                "l1_vs_oracle_sampled_columns": errs}
    if dist is not None:
        dist.destroy_process_group()
    return line


def run_c4b_ranks(args):
    """C4b on N GPUs (torchrun, one process per GPU): the 10,000 ego graphs
    split into contiguous graph ranges of nearly equal nodes plus arcs
    (ranks.split_graphs), each rank packing and solving its range in one
    launch with no exchange; the scores are gathered on rank 0, which checks
    sampled graphs against the oracle. Total work is fixed (strong scaling)."""
    import torch
    import knappnet_b200 as K
    from knappnet_b200 import ranks
    from oracle import oracle as O
    rank, world, local, dist = dist_setup(args.gpus)
    sizes = K.power_law_sizes(10_000, 2.1, 50, 50_000, seed=20240705)
    m = np.minimum(6 * sizes, sizes * (sizes - 1) // 2)
    src, tgt = K.generate_gnm(sizes, m, False, False, seed=20240706)
    off = np.concatenate([[0], np.cumsum(sizes)])
    cuts = [ranks.split_graphs(off, 2 * m, world, r) for r in range(world)]
    nodes = [(int(off[a]), int(off[b])) for a, b in cuts]
    g0, g1 = cuts[rank]
    a, b = nodes[rank]
    sel = (src >= a) & (src < b)
    g = K.Graph(b - a, src[sel] - a, tgt[sel] - a, None, False)
    loff = off[g0:g1 + 1] - a
    keep = {}

    def gpu():
        out, its, info = g.pagerank_graphs(loff, tol=1e-12)
        keep["x"], keep["info"] = out, info
        return info.seconds
    for _ in range(args.warmup):
        gpu()
    ranks.barrier(dist)
    times = [gpu() for _ in range(max(args.steps, 1))]
    sec = max_over_ranks(dist, statistics.median(times))
    X = ranks.gather_rows(dist, torch.from_numpy(keep["x"]).cuda(), nodes)
    line = None
    if rank == 0:
        rng = np.random.default_rng(9)
        worst = 0.0
        for k in rng.choice(len(sizes), 20, replace=False):
            lo, hi = off[k], off[k + 1]
            s2 = (src >= lo) & (src < hi)
            og = O.Graph(hi - lo, src[s2] - lo, tgt[s2] - lo, None, False)
            worst = max(worst, float(np.abs(X[lo:hi] - og.pagerank(tol=1e-12)).sum()))
        line = {"workload": f"c4b on {world} GPUs: 10,000 undirected G(n, 6n) ego graphs split "
                            "by contiguous graph ranges of nearly equal work, one launch per "
                            "rank, no exchange; scores gathered on rank 0",
                "metric": "batch ms (slowest rank)", "value": round(sec * 1e3, 3), "unit": "ms",
                "higher_is_better": False, "n_gpus": world, "scaling": "strong",
                "graphs_per_rank": [c1 - c0 for c0, c1 in cuts],
                "l1_vs_oracle_worst_of_20": worst}
    if dist is not None:
        dist.destroy_process_group()
    return line


def run_rows(args):
    """PageRank of the benchmark line's graph (R-MAT 24, lognormal weights,
    FP64) split by rows over N GPUs (torchrun, one process per GPU): each
    rank's shard holds rows of nearly equal rows plus arcs (net_shard_bounds),
    sweeps them into its payload, the ranks all-gather the payloads over
    NCCL (one collective per sweep, also for one rank under torchrun), and
    every rank finishes the sweep over all nodes. Total work is fixed (strong
    scaling). Rank 0 checks the scores against the single-GPU FP64 solve."""
    import torch
    import knappnet_b200 as K
    from knappnet_b200 import ranks
    rank, world, local, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    g = make_graph(args.scale)
    b = g.shard_bounds(world, directed=True, weighted=True)
    sh = K.Shard(g, b, rank, damping=0.85, directed=True, weighted=True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    keep = {}

    def solve():
        sh.restart(torch.empty(1, device=dev))
        ev0.record()
        keep["sweeps"] = ranks.pagerank_rows(dist, sh, device=dev, tol=1e-9)
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / 1e3
    for _ in range(args.warmup):
        solve()
    ranks.barrier(dist)
    times = [solve() for _ in range(max(args.steps, 1))]
    sec = max_over_ranks(dist, statistics.median(times))
    sweeps = keep["sweeps"]
    line = None
    if rank == 0:
        x = sh.scores()
        ref, info = g.pagerank_ex(directed=True, weighted=True, tol=1e-9, precision=K.PREC_FP64)
        arcs = int(g.m)  # a directed graph without loops: one pull arc per edge
        line = {"workload": f"rows on {world} GPUs: R-MAT {args.scale} directed, lognormal "
                            "weights, PageRank FP64, tol 1e-9, split by rows of the pull "
                            "operator; one all-gather of the payloads per sweep over NCCL",
                "metric": "GTEPS per iteration (whole job)",
                "value": round(arcs * sweeps / sec / 1e9, 3), "unit": "GTEPS",
                "higher_is_better": True, "n_gpus": world, "scaling": "strong",
                "ms_per_solve": round(sec * 1e3, 3), "sweeps": sweeps,
                "rows_per_rank": [int(b[k + 1] - b[k]) for k in range(world)],
                "payload_bytes_per_rank_per_sweep": sh.payload_len * 8,
                "exchange": "nccl all_gather_into_tensor" if dist is not None else "none",
                "l1_vs_single_gpu_fp64": float(np.abs(x - ref).sum()),
                "single_gpu_fp64_iterations": int(info.iterations)}
    sh.close()
    if dist is not None:
        dist.destroy_process_group()
    return line


def run_c5(args):
    """Differentiable PageRank on directed R-MAT 20 with lognormal weights:
    forward solve, adjoint solve and edge-gradient scatter through
    torch.autograd.Function."""
    import torch
    import knappnet_b200 as K
    from knappnet_b200 import autograd as AG
    g = K.generate_rmat(20, 16, seed=20240707, clean=True, lognormal=True, wseed=20240708)
    _, _, w = g.edges()
    rng = np.random.default_rng(20240709)
    wp = w * np.maximum(1 + 0.1 * rng.standard_normal(len(w)), 1e-3)
    target = AG.pagerank(torch.tensor(wp, device="cuda"), g, tol=1e-12).detach()
    wt = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)

    def step():
        wt.grad = None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        loss = ((AG.pagerank(wt, g, tol=1e-12) - target) ** 2).sum()
        loss.backward()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3
    sec = _median_device(step, args.steps, args.warmup)
    grad = wt.grad.detach().cpu().numpy()
    v = rng.standard_normal(len(w)) * w
    h = 1e-4

    def loss_at(x):
        y = AG.pagerank(torch.tensor(x, dtype=torch.float64, device="cuda"), g, tol=1e-13)
        return ((y - target) ** 2).sum().item()
    fd = (loss_at(w + h * v) - loss_at(w - h * v)) / (2 * h)
    an = float(grad @ v)
    return {"workload": "c5: R-MAT 20 directed, lognormal(0,1) FP32 weights, L = |x - x*|^2, "
                        "x* from weights perturbed by 10%, forward + adjoint + edge gradients",
            "metric": "forward+backward ms", "value": round(sec * 1e3, 3), "unit": "ms",
            "higher_is_better": False, "edges": int(len(w)),
            "directional_fd_rel_error": abs(fd - an) / abs(an)}


def run_next(args):
    """The measures built on the same kernels beyond PageRank and eigenvector
    centrality, one JSON line each: wall time of the C ABI call (host
    buffers; the median and minimum of the timed calls, which reuse the
    set-up kept per operator, and the first call on the handle, which builds
    it) against the oracle's time for the same call on this host, and the
    largest difference from the oracle."""
    import knappnet_b200 as K
    from oracle import oracle as O

    def timed(fn, release=None):
        """Median and minimum wall time of fn(); the previous call's result
        is released outside the timed region."""
        keep = {}
        times = []
        for i in range(args.warmup + max(args.steps, 1)):
            if "r" in keep and release is not None:
                release(keep["r"])
            keep.pop("r", None)
            t0 = time.perf_counter()
            keep["r"] = fn()
            dt = time.perf_counter() - t0
            if i == 0:
                timed.first = dt
            if i >= args.warmup:
                times.append(dt)
        timed.last_min = min(times)
        return statistics.median(times), keep["r"]

    def cpu(fn):
        t0 = time.perf_counter()
        r = fn()
        return time.perf_counter() - t0, r

    lines = []

    def line(name, what, sec, csec, extra):
        d = {"workload": name, "description": what, "metric": "call ms", "value": round(sec * 1e3, 3),
             "unit": "ms", "higher_is_better": False, "min_ms": round(timed.last_min * 1e3, 3),
             "first_call_ms": round(timed.first * 1e3, 3), "oracle_ms": round(csec * 1e3, 1)}
        d.update(extra)
        lines.append(d)

    # Katz and Bonacich power centrality, directed weighted R-MAT
    g = K.generate_rmat(20, 16, seed=20240711, clean=True, lognormal=True, wseed=20240712)
    s, t, w = g.edges()
    og = O.Graph(g.n, s, t, w, True)
    _, lam, _ = g.eigenvector(mode=2, weighted=True)
    alpha = 0.5 / lam
    sec, x = timed(lambda: g.katz(alpha=alpha, beta=1.0, mode=2, weighted=True))
    csec, ox = cpu(lambda: og.katz(alpha=alpha, beta=1.0, mode=2, weighted=True))
    line("katz", "R-MAT 20 directed, lognormal weights, mode in, alpha = 0.5 / lambda_max",
         sec, csec, {"nodes": g.n, "edges": g.m,
                     "max_rel_vs_oracle": float(np.abs(x - ox).max() / np.abs(ox).max())})
    sec, hv = timed(lambda: g.hits())
    csec, ohv = cpu(lambda: og.hits())
    line("hits", "R-MAT 20 directed, unweighted, scale max", sec, csec,
         {"nodes": g.n, "edges": g.m, "value_rel_vs_oracle": abs(hv[2] - ohv[2]) / ohv[2],
          "max_abs_vs_oracle": float(max(np.nanmax(np.abs(hv[0] - ohv[0])),
                                         np.nanmax(np.abs(hv[1] - ohv[1]))))})
    g.close()
    del og

    # strong and weak components
    g = K.generate_rmat(22, 16, seed=20240713, clean=True)
    s, t, _ = g.edges()
    og = O.Graph(g.n, s, t, None, True)
    for strong in (True, False):
        sec, (m, c) = timed(lambda: g.components(strong=strong))
        csec, (om, oc) = cpu(lambda: og.components(strong=strong))
        line("components_strong" if strong else "components_weak",
             "R-MAT 22 directed, cleaned", sec, csec,
             {"nodes": g.n, "edges": g.m, "components": int(c),
              "labels_identical": bool(c == oc and np.array_equal(m.astype(np.int64),
                                                                  om.astype(np.int64)))})
    g.close()
    del og

    # adjacency-matrix reading of a multigraph, then two-mode eigenvector
    g = K.generate_rmat(18, 16, seed=20240714, clean=False, lognormal=True, wseed=20240715)
    s, t, w = g.edges()
    og = O.Graph(g.n, s, t, w, True)
    sec, a = timed(lambda: g.simplify(undirected=True, keep=0), release=lambda h: h.close())
    csec, oa = cpu(lambda: og.simplify(undirected=True, keep=0))
    sa, ta, wa = a.edges()
    sb, tb, wb = oa.edges()
    line("simplify", "R-MAT 18 with loops and parallel arcs, lognormal weights, symmetrized, "
         "largest weight kept", sec, csec,
         {"edges_in": g.m, "edges_out": int(len(sa)),
          "identical": bool(np.array_equal(sa, sb) and np.array_equal(ta, tb)
                            and np.array_equal(wa, wb))})
    a.close()
    g.close()
    del og, oa
    rng = np.random.default_rng(20240716)
    n1, n2, mm = 200_000, 100_000, 2_000_000
    bs = rng.integers(0, n1, mm)
    bt = n1 + rng.integers(0, n2, mm)
    types = [0] * n1 + [1] * n2
    g = K.Graph(n1 + n2, bs, bt, None, False)
    og = O.Graph(n1 + n2, bs, bt, None, False)
    sec, (x, lam, _) = timed(lambda: g.twomode_eigenvector(types))
    csec, (ox, olam, _) = cpu(lambda: og.twomode_eigenvector(types))
    line("twomode_eigenvector", "random two-mode network, 200,000 + 100,000 nodes, 2,000,000 ties",
         sec, csec, {"singular_value_rel_vs_oracle": abs(lam - olam) / olam,
                     "max_abs_vs_oracle": float(np.nanmax(np.abs(x - ox)))})
    g.close()
    del og

    # leading eigenvector communities at the size limit's scale
    rng = np.random.default_rng(20240717)
    sizes = [250] * 8
    blk = np.repeat(np.arange(8), 250)
    iu, ju = np.triu_indices(2000, 1)
    p = np.where(blk[iu] == blk[ju], 0.05, 0.002)
    keep = rng.random(len(iu)) < p
    ls, lt = iu[keep].astype(np.int64), ju[keep].astype(np.int64)
    g = K.Graph(2000, ls, lt, None, False)
    og = O.Graph(2000, ls, lt, None, False)
    sec, (m, q, sp) = timed(lambda: g.leading_eigen())
    csec, (om, oq, osp) = cpu(lambda: og.leading_eigen())
    line("leading_eigen", "planted partition, 8 blocks of 250 nodes, p_in 0.05, p_out 0.002",
         sec, csec, {"edges": int(len(ls)), "splits": int(sp), "modularity": q,
                     "labels_identical": bool(np.array_equal(m, om) and sp == osp),
                     "modularity_rel_vs_oracle": abs(q - oq) / abs(oq)})
    g.close()
    return lines


SHARDED = {"c4a": run_c4a_ranks, "c4b": run_c4b_ranks, "rows": run_rows}
WORKLOADS = {"c1": run_c1, "c2": run_c2, "c4a": run_c4a, "c4b": run_c4b, "c5": run_c5,
             "next": run_next, "rows": run_rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-budget", type=float, default=15.0,
                    help="seconds of CPU work for the cpu_baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", choices=["c3", "c1", "c2", "c4a", "c4b", "c5", "next", "rows"],
                    default="c3",
                    help="c3 (default) is the benchmark line; the others print one JSON line "
                         "each for the other configurations (next: one per measure beyond "
                         "PageRank and eigenvector centrality)")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="R-MAT scale (the benchmark workload is 24; smaller scales "
                         "serve profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload != "c3":
        if args.impl == "reference":
            return
        if args.workload in SHARDED and "WORLD_SIZE" in os.environ:
            line = SHARDED[args.workload](args)  # every rank takes part; rank 0 reports
            if line is not None:
                line.update({"steps": args.steps, "warmup": args.warmup,
                             "data": "synthetic (seeded Philox generators)"})
                print(json.dumps(line), flush=True)
            return
        if int(os.environ.get("RANK", 0)) != 0:
            return
        result = WORKLOADS[args.workload](args)
        for line in (result if isinstance(result, list) else [result]):
            line.update({"n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                         "data": "synthetic (seeded Philox generators)"})
            print(json.dumps(line), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
