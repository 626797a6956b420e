"""Benchmark of the Kirchhoff engine (prints ONE JSON line on rank 0).

Default workload: the single large solve — 2^20 rays on a Gaussian aperture
(sigma 0.1 mm, R = 30 m, 10 keV) against a 512x512 screen grid of +-0.5 mm at
z = 1000 mm (2.75e11 ray x screen pairs per step), FP32 phase-reduced form.

  value  Gpair/s of the FP32 phase-reduced solve with inputs resident in HBM
         (CUDA events on the launching stream, L2 flushed between steps)
  e2e    the same through the host-buffer C ABI (pinned host inputs, H2D
         copies, solve, D2H of the field), wall clock per step
  fp64_plain  the plain FP64 solve on the same inputs (the 10x reference)
  roofline    the pair kernel against the FP32-FMA/SFU pair roofline
  cpu_baseline the CPU oracle (a restatement of src/waves/diffraction.rs) on
         a bounded sample of screen points, all host threads

`--impl reference` times the reference's CPU algorithm (the oracle port, the
reference's Rust cannot be built here) on the same workload's sample.

Multi-GPU (torchrun): by default the one solve's screen is split into
contiguous blocks, one per rank, and the blocks are all-gathered over NCCL
each step (strong scaling); `--shard replica` runs an independent copy of the
workload per rank instead (weak scaling). Timing is the max over ranks.

After the timed region the default run also reports served latency: the
serving mix as a Poisson stream through the continuous-batching server at a
rate one B200 sustains and at 200 req/s (`serve`).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "xrt-rs_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Gpair/s (ray x screen pair evaluations), FP32 phase-reduced vs FP64 plain"
UNIT = "Gpair/s"
# Algorithmic work per ray x screen pair of the reference formula
# (kirchhoff.wgsl:79-128 with per-ray terms amortised): 34 FP32 FMA-pipe
# operations and 4 SFU operations (rsqrt, rcp, sin, cos).
FMA_OPS_PER_PAIR = 34
SFU_OPS_PER_PAIR = 4
# DRAM bytes (read + write) of one pr_persistent_kernel launch on the 2^20 x
# 512^2 workload from an ncu capture of the full-size launch, by the number of
# amplitude columns summed (two-column kernel: key False).
DRAM_BYTES_CONFIG1 = {False: 502.3e6, True: 270.7e6}
# The same for one fresnel_pair_kernel launch on 2^20 rays x 512^2: the four
# ray columns read once (the FP64 split partials stay in L2).
FRESNEL_DRAM_BYTES_CONFIG = 33.8e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 plain comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--sweep", type=int, default=-1,
                    help="-1 auto, 0 SFU reciprocal, 1 packed (quadratic series), "
                         "2 packed (linear series)")
    ap.add_argument("--phase-budget", type=float, default=512.0,
                    help="cap on the FP32 residual phase [rad]")
    ap.add_argument("--tolerance", type=float, default=1e-4,
                    help="requested relative L2 error of the FP32 phase-reduced field; the "
                         "planner derives the residual-phase budget from it")
    ap.add_argument("--polarization", type=int, default=-1, choices=[-1, 0],
                    help="-1: one amplitude column when all rays share a polarization; "
                         "0: always sum Es and Ep separately")
    ap.add_argument("--workload", choices=["single", "batch", "sweep", "serve", "fresnel"],
                    default="single",
                    help="single: the 2^20 x 512^2 solve (default); batch: 64 uneven solves; "
                         "sweep: the energy x distance precision sweep; serve: Poisson "
                         "arrivals through the server; fresnel: 2-D Fresnel propagation")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: Poisson arrival rate [1/s]")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: arrival window [s]")
    ap.add_argument("--drain", type=float, default=60.0,
                    help="serve: seconds to wait for outstanding requests after the window")
    ap.add_argument("--sweep-sample", type=int, default=64,
                    help="screen points per cell checked against the CPU oracle")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--tune-budget-ms", type=float, default=100.0,
                    help="batch: device time the autotuner may spend per solve")
    ap.add_argument("--epoch-pairs", type=float, default=0.0,
                    help="serve: pairs per epoch (0 = the server's default)")
    ap.add_argument("--item-pairs", type=float, default=0.0,
                    help="serve: pairs per work item (0 = the server's default)")
    ap.add_argument("--serve-policy", type=int, default=0, choices=[0, 1],
                    help="server epoch sharing: 0 shortest remaining work first, aged "
                         "(default); 1 equal share per running request")
    ap.add_argument("--reserve-sms", type=int, default=0,
                    help="serve: SMs left to planning (0 = the server's default)")
    ap.add_argument("--shard", choices=["screen", "replica"], default="screen",
                    help="N > 1: 'screen' splits the one solve's screen across the ranks "
                         "(strong scaling, blocks all-gathered on the GPUs each step); "
                         "'replica' runs an independent copy of the workload per rank "
                         "(weak scaling)")
    ap.add_argument("--no-serve", action="store_true",
                    help="single workload: skip the served-latency block")
    ap.add_argument("--serve-window", type=float, default=30.0,
                    help="single workload: arrival window of each served-latency stream [s]")
    ap.add_argument("--serve-rate", type=float, default=25.0,
                    help="single workload: the sustainable stream's arrival rate [1/s]")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smmax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smmax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smmax)) if smmax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def balanced_count(count: int, threads: int, limit: int) -> int:
    """Screen points per CPU sample rounded up to a multiple of 4 x threads,
    so that the oracle's one-point-at-a-time OpenMP schedule ends with every
    thread busy (a sample of 92 points on 16 threads left 9 idle in its last
    round)."""
    unit = 4 * max(1, threads)
    return int(min(limit, max(unit, -(-count // unit) * unit)))


def cpu_baseline(rays, screen, seconds: float):
    """The oracle on a bounded sample of screen points, all host threads."""
    from oracle import oracle  # checker / baseline only
    from xrt_rs import synth

    rl = [rays[k] for k in ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re",
                            "ep_im", "energy")]
    threads = max(oracle.max_threads(), len(os.sched_getaffinity(0)))  # not torchrun's 1
    count = balanced_count(8, threads, len(screen["x"]))
    rate = None
    while True:
        sub, _ = synth.subsample_screen(screen, count, seed=7)
        t0 = time.perf_counter()
        oracle.kahan_f64(rl, [sub["x"], sub["y"], sub["z"]], threads=threads)
        dt = time.perf_counter() - t0
        rate = len(rl[0]) * count / dt
        if dt >= seconds * 0.5 or count >= len(screen["x"]):
            break
        count = int(min(len(screen["x"]), max(count * 2, count * seconds * 0.6 / max(dt, 1e-3))))
        count = balanced_count(count, threads, len(screen["x"]))
    return {"value": rate / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(rl[0])} rays x {count} seeded screen points of the workload "
                      f"({dt:.1f} s, C restatement of src/waves/diffraction.rs:56-117, "
                      f"OpenMP over screen points)"}


def single_workload(n_rays: int, grid: int) -> str:
    """Name of the single-solve workload (both arms)."""
    return (f"single solve: {n_rays} rays (Gaussian aperture sigma 0.1 mm, 10 keV) x "
            f"{grid}x{grid} screen +-0.5 mm at 1000 mm")


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle
    from xrt_rs import synth

    rays, screen = synth.config1(seed=0, n_rays=args.rays, grid=args.grid)
    rl = [rays[k] for k in ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re",
                            "ep_im", "energy")]
    # All the host's cores: rank 0 runs alone (torchrun sets OMP_NUM_THREADS=1
    # for every rank, which would otherwise leave the reference on one core).
    threads = max(oracle.max_threads(), len(os.sched_getaffinity(0)))
    # Size one step to ~2 s of CPU work.
    sub, _ = synth.subsample_screen(screen, 16, seed=7)
    t0 = time.perf_counter()
    oracle.kahan_f64(rl, [sub["x"], sub["y"], sub["z"]], threads=threads)
    per_point = (time.perf_counter() - t0) / 16
    count = int(max(16, min(len(screen["x"]), 2.0 / max(per_point, 1e-6))))
    count = balanced_count(count, threads, len(screen["x"]))
    sub, _ = synth.subsample_screen(screen, count, seed=7)
    pl = [sub["x"], sub["y"], sub["z"]]
    for _ in range(args.warmup):
        oracle.kahan_f64(rl, pl, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.kahan_f64(rl, pl, threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    pairs = len(rl[0]) * count
    value = pairs / (ms / 1e3) / 1e9
    sample = (f"{len(rl[0])} rays x {count} seeded screen points of the 512x512 grid per step; "
              f"C restatement of src/waves/diffraction.rs:56-117 (the Rust reference cannot be "
              f"built: no cargo), OpenMP over screen points")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        # The same scaling key as this arm's CUDA line for the same flags.
        "higher_is_better": True, "scaling": "strong" if args.shard == "screen" else "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": single_workload(args.rays, args.grid), "rays": args.rays,
                   "screen_points": args.grid ** 2,
                   "workload_pairs": float(args.rays) * float(args.grid ** 2),
                   "parallelism": "rank 0 only (host cores)",
                   "pairs_per_step": float(pairs)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """64 uneven solves: one persistent graph-captured launch vs a loop of
    per-solve calls, both on device-resident inputs."""
    import torch
    import xrt_rs
    from xrt_rs import synth

    torch.cuda.set_device(0)
    ctx = xrt_rs.GpuContext.new(0)
    ctx.set_option("sweep", args.sweep)
    ctx.set_option("phase_budget", args.phase_budget)
    ctx.set_option("tolerance", args.tolerance)
    ctx.set_option("polarization", args.polarization)
    solves = synth.config3(seed=0, count=args.batch_count)
    pairs = float(sum(len(r["x"]) * len(p["x"]) for r, p, _ in solves))
    dev = []
    for rays, screen, _ in solves:
        d_r = [torch.from_numpy(rays[k]).cuda() for k in xrt_rs.RAY_FIELDS]
        d_p = [torch.from_numpy(screen[k]).cuda() for k in "xyz"]
        d_o = [torch.zeros(len(screen["x"]), dtype=torch.float64, device="cuda") for _ in range(4)]
        dev.append((d_r, d_p, d_o))
    stream = torch.cuda.current_stream()

    def loop():
        for d_r, d_p, d_o in dev:
            xrt_rs.diffraction_integral_device(d_r, d_p, d_o, path="f32pr", ctx=ctx,
                                               stream=stream.cuda_stream)

    for _ in range(args.warmup):
        loop()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loop()
    torch.cuda.synchronize()
    loop_ms = 1e3 * (time.perf_counter() - t0) / args.steps

    # The first batch maps its memory from the driver; a batch planned after it
    # reuses that memory from the stream-ordered pool (the steady state of a
    # caller that plans batch after batch). Both planning times are reported.
    first = xrt_rs.Batch([(d_r, d_p) for d_r, d_p, _ in dev], path="f32pr", ctx=ctx,
                         device_outputs=[d_o for _, _, d_o in dev])
    first.run()
    plan_first_ms = first.stats["plan_ms"]
    first.close()
    batch = xrt_rs.Batch([(d_r, d_p) for d_r, d_p, _ in dev], path="f32pr", ctx=ctx,
                         device_outputs=[d_o for _, _, d_o in dev])
    plan_ms = None
    for _ in range(args.warmup):
        batch.run()
        plan_ms = batch.stats["plan_ms"]
    exec_ms, wall_ms = [], []
    for _ in range(args.steps):
        batch.run()
        exec_ms.append(batch.stats["exec_ms"])
        wall_ms.append(batch.stats["wall_ms"])
    ex = float(np.mean(exec_ms))
    batch_stats = dict(batch.stats)
    batch.close()

    # Autotuned: each solve's bucket tuned once (xk_autotune, settings kept in
    # the context's per-bucket cache), then the same batch and loop again.
    tune_t0 = time.perf_counter()
    tuned_buckets = 0
    for d_r, d_p, d_o in dev:
        res = xrt_rs.autotune(d_r, d_p, d_o, ctx=ctx, budget_ms=args.tune_budget_ms, apply=True)
        tuned_buckets += 1 if res["trials"] > 1 else 0
    tune_s = time.perf_counter() - tune_t0
    for _ in range(args.warmup):
        loop()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loop()
    torch.cuda.synchronize()
    loop_tuned_ms = 1e3 * (time.perf_counter() - t0) / args.steps
    tuned = xrt_rs.Batch([(d_r, d_p) for d_r, d_p, _ in dev], path="f32pr", ctx=ctx,
                         device_outputs=[d_o for _, _, d_o in dev])
    for _ in range(args.warmup):
        tuned.run()
    texec = []
    for _ in range(args.steps):
        tuned.run()
        texec.append(tuned.stats["exec_ms"])
    tplan_ms = tuned.stats["plan_ms"]
    tuned_plans = sum(1 for i in range(len(dev)) if tuned.plan(i).get("tuned", 0))
    tuned.close()
    tex = float(np.mean(texec))
    line = {
        "workload": "batch", "metric": "Gpair/s over 64 uneven solves", "unit": UNIT,
        "value": pairs / (ex / 1e3) / 1e9, "steps": args.steps, "warmup": args.warmup,
        "pairs_per_step": pairs, "n_solves": len(solves),
        "inputs": "device-resident for both arms",
        "batch_graph_exec_ms": ex, "batch_run_wall_ms": float(np.mean(wall_ms)),
        "batch_plan_ms": plan_ms, "batch_plan_first_ms": plan_first_ms,
        "loop_per_solve_calls_ms": loop_ms,
        "loop_gpair_s": pairs / (loop_ms / 1e3) / 1e9,
        "batch_plus_plan_gpair_s": pairs / ((ex + plan_ms) / 1e3) / 1e9,
        "speedup_graph_exec_vs_loop": loop_ms / ex,
        "autotuned": {
            "tune_s": tune_s, "solves_tuned": tuned_buckets, "batch_plans_tuned": tuned_plans,
            "batch_graph_exec_ms": tex, "batch_plan_ms": tplan_ms,
            "batch_gpair_s": pairs / (tex / 1e3) / 1e9,
            "loop_per_solve_calls_ms": loop_tuned_ms,
            "loop_gpair_s": pairs / (loop_tuned_ms / 1e3) / 1e9,
            "speedup_tuned_batch_vs_default_loop": loop_ms / tex,
            "speedup_tuned_batch_vs_tuned_loop": loop_tuned_ms / tex,
            "speedup_tuned_vs_default_batch": ex / tex},
        "routed_f64": batch_stats["routed_f64"], "kernels_per_run": batch_stats["kernels"],
        "data": "synthetic: N log-uniform [1e3,1e6], M log-uniform [64,262144], E U(5,25) keV, "
                "d U(500,10000) mm, sigma U(0.02,0.2) mm, R U(10,50) m",
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_sweep(args):
    """E in {1,5,10,20,30} keV x d in {100,1000,5000,20000} mm, 2^18 rays x 256^2.

    Per cell: the FP32 phase-reduced field and the FP64 field on the GPU (full
    screen, timed), and their errors on a seeded screen subsample against the
    oracle evaluated with an extended-precision phase (CPU)."""
    import torch
    import xrt_rs
    from oracle import oracle
    from xrt_rs import synth

    torch.cuda.set_device(0)
    ctx = xrt_rs.GpuContext.new(0)
    ctx.set_option("sweep", args.sweep)
    ctx.set_option("phase_budget", args.phase_budget)
    ctx.set_option("tolerance", args.tolerance)
    ctx.set_option("polarization", args.polarization)
    cells = []
    for e in synth.CONFIG2_ENERGIES:
        for d in synth.CONFIG2_DISTANCES:
            rays, screen, meta = synth.config2_cell(e, d, seed=int(e) + int(d))
            rl = [rays[k] for k in xrt_rs.RAY_FIELDS]
            d_r = [torch.from_numpy(a).cuda() for a in rl]
            d_p = [torch.from_numpy(screen[k]).cuda() for k in "xyz"]
            m = len(screen["x"])
            res = {}
            for path in ("f32pr", "f64"):
                d_o = [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in range(4)]
                xrt_rs.diffraction_integral_device(d_r, d_p, d_o, path=path, ctx=ctx)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                st = xrt_rs.diffraction_integral_device(d_r, d_p, d_o, path=path, ctx=ctx)
                e1.record()
                e1.synchronize()
                res[path] = ([t.cpu().numpy() for t in d_o], e0.elapsed_time(e1), st)
            sub, idx = synth.subsample_screen(screen, args.sweep_sample, seed=int(e + d))
            exact = oracle.kahan_ld(rl, [sub["x"], sub["y"], sub["z"]])

            def err(out):
                a = np.concatenate([out[0][idx] + 1j * out[1][idx], out[2][idx] + 1j * out[3][idx]])
                b = np.concatenate([exact[0] + 1j * exact[1], exact[2] + 1j * exact[3]])
                ia = np.abs(a[: len(idx)]) ** 2 + np.abs(a[len(idx):]) ** 2
                ib = np.abs(b[: len(idx)]) ** 2 + np.abs(b[len(idx):]) ** 2
                return (float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                        float(np.linalg.norm(ia - ib) / np.linalg.norm(ib)))

            pairs = float(len(rl[0])) * m
            f32, f64 = res["f32pr"], res["f64"]
            e32, e32i = err(f32[0])
            e64, e64i = err(f64[0])
            cells.append({
                "energy_ev": e, "dist_mm": d, "sigma_mm": meta["sigma_mm"],
                "radius_mm": meta["radius_mm"], "path": "f32pr" if f32[2]["path"] == 1 else "f64",
                "n_chunks": f32[2]["n_chunks"], "sweep": f32[2]["sweep"],
                "amplitude_columns": 1 if f32[2]["one_polarization"] else 2,
                "rel_l2_field": e32, "rel_l2_intensity": e32i,
                "fp64_formula_rel_l2_field": e64, "fp64_formula_rel_l2_intensity": e64i,
                "f32pr_gpair_s": pairs / f32[1] / 1e6, "fp64_gpair_s": pairs / f64[1] / 1e6,
                "speedup": f64[1] / f32[1]})
            print(json.dumps(cells[-1]), file=sys.stderr, flush=True)
    worst = max(c["rel_l2_field"] for c in cells)
    line = {"workload": "sweep", "metric": "rel L2 vs the extended-precision oracle per (E, d) cell",
            "n_rays": 1 << 18, "screen": "256x256 grid +-1 mm", "sample_points": args.sweep_sample,
            "worst_rel_l2_field": worst,
            "worst_rel_l2_intensity": max(c["rel_l2_intensity"] for c in cells),
            "min_speedup": min(c["speedup"] for c in cells), "cells": cells}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_fresnel(args):
    """2-D Fresnel propagation (src/waves/fresnel.rs:53-106): the aperture's
    2^20 rays (x, z) with complex amplitudes onto a 512x512 screen of
    +-0.5 mm at 1000 mm, 10 keV. The separable tensor-core product against the
    FP64 direct sum on the same inputs, the oracle on one screen row as the
    CPU baseline; the product kernel against the measured bf16 tensor peak."""
    import torch
    import xrt_rs
    from oracle import oracle
    from xrt_rs import synth

    torch.cuda.set_device(0)
    ctx = xrt_rs.GpuContext.new(0)
    rays, _ = synth.config1(seed=0, n_rays=args.rays, grid=8)
    # Host inputs in pinned memory (the end-to-end time copies them every step).
    x = torch.from_numpy(rays["x"]).pin_memory().numpy()
    z = torch.from_numpy(rays["y"]).pin_memory().numpy()
    es = (torch.from_numpy(rays["es_re"]).pin_memory().numpy(),
          torch.from_numpy(rays["es_im"]).pin_memory().numpy())
    g = args.grid
    sc = xrt_rs.FresnelScreen(-0.5, 0.5, g, -0.5, 0.5, g)
    energy, dist = 10000.0, 1000.0
    pairs = float(len(x)) * g * g
    for _ in range(args.warmup):
        xrt_rs.fresnel_propagate(x, z, es, energy, dist, sc, ctx=ctx)
    clocks = ClockSampler(0)
    clocks.start()
    dev_ms, wall_ms, gemm_ms = [], [], []
    for _ in range(args.steps):
        res, st = xrt_rs.fresnel_propagate(x, z, es, energy, dist, sc, ctx=ctx, return_stats=True)
        dev_ms.append(st["gpu_ms"])
        wall_ms.append(st["wall_ms"])
        gemm_ms.append(st["main_kernel_ms"])
    clk = clocks.stop()
    ref64, st64 = xrt_rs.fresnel_propagate(x, z, es, energy, dist, sc, path="f64", ctx=ctx,
                                           return_stats=True)
    err = float(np.linalg.norm(res.amplitude - ref64.amplitude) / np.linalg.norm(ref64.amplitude))
    # Tensor work: per pair one complex multiply-add (8 real flops) in each of
    # the three f16 partial products.
    algo_flops = 24.0 * pairs
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    if "bf16_tflops" in peaks:
        peak = float(peaks["bf16_tflops"])
        peak_source = "MEASURED_PEAKS.json bf16_tflops (burst; f16 runs at the bf16 rate)"
    else:
        peak = 1590.0
        peak_source = ("fallback: 1590 TFLOP/s, an earlier burst cuBLAS bf16 measurement on "
                       "this pool (MEASURED_PEAKS.json absent; f16 runs at the bf16 rate)")
    gemm = float(np.mean(gemm_ms))
    achieved = algo_flops / (gemm / 1e3) / 1e12
    # Screens of more than 128 rows run on CTA pairs (stats sweep = 1).
    fr_kernel = "fresnel_pair_kernel" if st["sweep"] == 1 else "fresnel_fused_kernel"
    # DRAM bytes (read + write) of one fresnel_pair_kernel launch on the
    # 2^20-ray 512x512 workload, from a single-pass ncu capture of full-size
    # launches; other sizes report null.
    fr_traffic = (FRESNEL_DRAM_BYTES_CONFIG
                  if (args.rays == 1 << 20 and args.grid == 512 and st["sweep"] == 1) else None)
    cpu = None
    if not args.no_cpu:
        row = xrt_rs.FresnelScreen(-0.5, 0.5, g, 0.0, 0.0, 1)
        t0 = time.perf_counter()
        oracle.fresnel(x, z, es[0], es[1], energy, dist, row.x_min, row.x_max, g, 0.0, 0.0, 1)
        dt = time.perf_counter() - t0
        cpu = {"value": len(x) * g / dt / 1e9, "unit": UNIT, "cores": oracle.max_threads(),
               "kind": "port",
               "sample": f"{len(x)} rays x one {g}-point screen row ({dt:.1f} s, C restatement "
                         f"of src/waves/fresnel.rs:53-106, OpenMP over screen points)"}
    dev = float(np.mean(dev_ms))
    line = {
        "workload": "fresnel", "metric": "Gpair/s (ray x screen pair evaluations)",
        "value": pairs / (dev / 1e3) / 1e9, "unit": UNIT, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev, "dtype": "f16x3 products, f32/f64 accumulation",
        "data": "synthetic",
        "config": {"workload": f"fresnel: {len(x)} rays x {g}x{g} screen +-0.5 mm at 1000 mm, "
                               "10 keV", "rays": len(x), "screen_points": g * g,
                   "pairs_per_step": pairs, "chunks": st["n_chunks"],
                   "tiles": st["n_tiles"], "k_splits": st["groups"]},
        "e2e": {"value": pairs / (float(np.mean(wall_ms)) / 1e3) / 1e9, "unit": UNIT,
                "ms_per_step": float(np.mean(wall_ms)), "h2d_bytes_per_step": st["h2d_bytes"],
                "d2h_bytes_per_step": st["d2h_bytes"]},
        "fp64_direct": {"value": pairs / (st64["gpu_ms"] / 1e3) / 1e9, "unit": UNIT,
                        "ms_per_step": st64["gpu_ms"],
                        "speedup_separable_vs_f64": st64["gpu_ms"] / dev,
                        "rel_l2_separable_vs_f64": err},
        "roofline": {"bound": "tensor", "kernel": fr_kernel,
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": fr_traffic, "kernel_ms": gemm,
                     "peak_source": peak_source,
                     "algorithmic_flops": algo_flops,
                     # The sum itself is one complex multiply-add (8 flops) per
                     # pair; the three f16 partial products that carry its
                     # precision are counted above.
                     "single_product_equivalent": {
                         "flops": 8.0 * pairs, "achieved": achieved / 3.0,
                         "frac": achieved / 3.0 / peak}},
        "cpu_baseline": cpu, "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def serve_session(ctx, rate_hz: float, duration_s: float, drain_s: float, seed: int = 0,
                  epoch_pairs: float = 0.0, item_pairs: float = 0.0, reserve_sms: int = 0,
                  policy: int = 0):
    """One Poisson request stream through the continuous-batching server.

    Request sizes follow the serving configuration (rays log-uniform in
    [1e4, 2e6], screen points log-uniform in [256, 1e6], E ~ U(1, 30) keV,
    d ~ U(100, 20000) mm, 30 % reuse a resident ray set). Rays are slices of a
    shared 2e6-ray Gaussian aperture with the request's energy, so requests
    can be produced at the arrival rate; screens are square grids. Requests
    still unfinished `drain_s` after the arrival window are cancelled by the
    shutdown and counted as unfinished; latencies are those of completed
    requests."""
    import threading

    import xrt_rs
    from xrt_rs import synth
    from xrt_rs.serve import Server

    reqs = synth.config4_requests(seed=seed, rate_hz=rate_hz, duration_s=duration_s)
    base = synth.gaussian_aperture(2_000_000, 0.1, 10_000.0, 30_000.0, seed=1)
    srv = Server(ctx, hbm_budget_bytes=120e9, epoch_pairs=epoch_pairs,
                 item_pairs=item_pairs, reserve_sms=reserve_sms, policy=policy)
    sets = {}
    lat, done_pairs, failures = [], [0.0], [0]
    lock = threading.Lock()
    pending = []

    def rays_for(r):
        n = r["n_rays"]
        out = {k: v[:n] for k, v in base.items() if k != "energy"}
        out["energy"] = np.full(n, r["energy_ev"])
        return out

    grids = {}

    def screen_for(r):
        side = max(16, int(round(np.sqrt(r["n_pix"]))))
        if side not in grids:
            g = synth.grid_screen(side, side, 1.0, 0.0)
            grids[side] = (g["x"], g["y"])
        x, y = grids[side]
        return {"x": x, "y": y, "z": np.full(len(x), r["dist_mm"])}

    def waiter():
        while True:
            with lock:
                item = pending.pop(0) if pending else None
            if item is None:
                if stop.is_set():
                    return
                time.sleep(0.001)
                continue
            t, pairs = item
            try:
                srv.wait(t, timeout_ms=max(1.0, 1e3 * (deadline - time.perf_counter())))
                st = srv.last_stats
                with lock:
                    lat.append(st["total_ms"])
                    done_pairs[0] += st["pairs"]
            except xrt_rs.XkError:
                with lock:
                    failures[0] += 1

    stop = threading.Event()
    deadline = time.perf_counter() + duration_s + drain_s
    waiters = [threading.Thread(target=waiter, daemon=True) for _ in range(8)]
    for w in waiters:
        w.start()
    t0 = time.perf_counter()
    submitted = 0
    for i, r in enumerate(reqs):
        now = time.perf_counter() - t0
        if r["t"] > now:
            time.sleep(r["t"] - now)
        screen = screen_for(r)
        if r["reuse_of"] >= 0 and sets:
            # A new screen on a ray set already resident on the device.
            key = list(sets)[r["reuse_of"] % len(sets)]
            handle, n = sets[key]
            t = srv.submit(screen, rayset=handle)
        else:
            rays = rays_for(r)
            n = r["n_rays"]
            if i % 4 == 0:  # keep up to 32 ray sets resident for later screens
                if len(sets) >= 32:
                    old = next(iter(sets))
                    srv.release_rays(sets.pop(old)[0])
                sets[i] = (srv.upload_rays(rays), n)
                t = srv.submit(screen, rayset=sets[i][0])
            else:
                t = srv.submit(screen, rays=rays)
        with lock:
            pending.append((t, float(n) * len(screen["x"])))
        submitted += 1
    window = time.perf_counter() - t0
    launched_in_window = srv.stats()["pairs_launched"]
    stop.set()
    for w in waiters:
        w.join(timeout=drain_s + 30)
    elapsed = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat_a = np.array(lat) if lat else np.array([np.nan])
    offered = sum(r["n_rays"] * max(16, int(round(np.sqrt(r["n_pix"])))) ** 2
                  for r in reqs) / duration_s / 1e9
    return {
        "rate_hz": rate_hz, "window_s": window, "elapsed_s": elapsed, "submitted": submitted,
        "completed": len(lat), "unfinished": submitted - len(lat),
        "p50_ms": float(np.percentile(lat_a, 50)), "p90_ms": float(np.percentile(lat_a, 90)),
        "p99_ms": float(np.percentile(lat_a, 99)),
        "gpair_s_served": done_pairs[0] / elapsed / 1e9,
        # Pairs of all work items launched during the arrival window (partly
        # served requests included): the device throughput under this load.
        "gpair_s_launched_in_window": launched_in_window / window / 1e9,
        "offered_gpair_s": offered,
        "epochs": st["epochs"], "peak_bytes": st["peak_bytes"], "hbm_budget_bytes": 120e9,
    }


def run_serve(args):
    import torch
    import xrt_rs

    torch.cuda.set_device(0)
    ctx = xrt_rs.GpuContext.new(0)
    res = serve_session(ctx, args.rate, args.duration, args.drain, epoch_pairs=args.epoch_pairs,
                        item_pairs=args.item_pairs, reserve_sms=args.reserve_sms,
                        policy=args.serve_policy)
    ctx.close()
    line = {"workload": "serve", "metric": "served latency and throughput", **res,
            "data": "synthetic: rays sliced from one 2e6-ray aperture, square-grid screens"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "sweep":
        return run_sweep(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "fresnel":
        return run_fresnel(args)

    import torch
    import xrt_rs
    from xrt_rs import synth

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if world > 1 else 0)
    ctx = xrt_rs.GpuContext.new(dev.index)
    if ctx is None:
        raise RuntimeError("no CUDA device")
    ctx.set_option("sweep", args.sweep)
    ctx.set_option("phase_budget", args.phase_budget)
    ctx.set_option("tolerance", args.tolerance)
    ctx.set_option("polarization", args.polarization)

    from xrt_rs import parallel

    # Screen sharding: every rank holds the same rays and solves a contiguous
    # block of the one screen; replicas: every rank its own seeded copy.
    shard = args.shard == "screen"
    rays, screen = synth.config1(seed=0 if shard else rank, n_rays=args.rays, grid=args.grid)
    fields = xrt_rs.RAY_FIELDS
    m_total = len(screen["x"])
    blk0, blk1 = parallel.shard_range(m_total, rank, world) if shard else (0, m_total)
    d_rays = [torch.from_numpy(rays[k]).to(dev) for k in fields]
    d_pix_full = [torch.from_numpy(screen[k]).to(dev) for k in "xyz"]
    d_pix = [t[blk0:blk1] for t in d_pix_full]  # contiguous views of this rank's block
    m = blk1 - blk0
    n = len(rays["x"])
    d_out = [torch.zeros(m, dtype=torch.float64, device=dev) for _ in range(4)]
    gather = shard and world > 1
    d_full = ([torch.zeros(m_total, dtype=torch.float64, device=dev) for _ in range(4)]
              if gather else None)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    pairs = float(n) * float(m)  # this rank's
    pairs_job = float(n) * float(m_total) if shard else pairs * world

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def solve(path):
        return xrt_rs.diffraction_integral_device(d_rays, d_pix, d_out, path=path, ctx=ctx,
                                                  stream=stream.cuda_stream)

    def step():
        st = solve("f32pr")
        if gather:  # the field's blocks, GPU to GPU over NCCL
            parallel.gather_field_device(d_out, m_total, out=d_full)
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(dev.index)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, kern_ms, launches = [], [], 0
    stats = None
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stats = step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        kern_ms.append(stats["main_kernel_ms"])
        launches += stats["kernels"]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = float(np.mean(step_ms))
    if world > 1:
        ms = parallel.max_over_ranks(ms)
    value = pairs_job / (ms / 1e3) / 1e9
    out32 = [t.cpu().numpy() for t in d_out]

    # The same solve with Es and Ep summed separately (what any input without
    # one common polarization runs), for comparison.
    two_col = None
    if stats["one_polarization"]:
        ctx.set_option("polarization", 0)
        solve("f32pr")
        tms = []
        for _ in range(3):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solve("f32pr")
            e1.record(stream)
            e1.synchronize()
            tms.append(e0.elapsed_time(e1))
        ctx.set_option("polarization", args.polarization)
        o2 = [t.cpu().numpy() for t in d_out]
        a = np.concatenate([out32[0] + 1j * out32[1], out32[2] + 1j * out32[3]])
        b = np.concatenate([o2[0] + 1j * o2[1], o2[2] + 1j * o2[3]])
        tms_mean = float(np.mean(tms))
        if world > 1:
            tms_mean = parallel.max_over_ranks(tms_mean)
        two_col = {"value": pairs_job / (tms_mean / 1e3) / 1e9, "unit": UNIT,
                   "ms_per_step": tms_mean, "steps": 3,
                   "rel_l2_field_vs_one_column": float(np.linalg.norm(a - b) / np.linalg.norm(b))}

    # End to end through the host C ABI: pinned host inputs -> field on host.
    # With screen sharding on N > 1 ranks each rank solves its block from
    # host memory and the field is all-gathered (xrt_rs.parallel.solve_sharded).
    e2e = None
    if not args.no_e2e:
        h_rays = {k: torch.from_numpy(rays[k]).pin_memory().numpy() for k in fields}
        h_pix = {k: torch.from_numpy(screen[k]).pin_memory().numpy() for k in "xyz"}
        h_blk = {k: v[blk0:blk1] for k, v in h_pix.items()}

        def e2e_step():
            if gather:
                parallel.solve_sharded(h_rays, h_pix, path="f32pr", ctx=ctx)
                return None
            return xrt_rs.diffraction_integral(h_rays, h_blk, path="f32pr", ctx=ctx,
                                               return_stats=True)[1]

        e2e_step()
        times = []
        st = None
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            st = e2e_step()
            times.append(time.perf_counter() - t0)
        e2e_ms = 1e3 * float(np.mean(times))
        if world > 1:
            e2e_ms = parallel.max_over_ranks(e2e_ms)
        if st is not None:
            h2d, d2h = int(st["h2d_bytes"]), int(st["d2h_bytes"])
        else:  # rays + this rank's block up, its field down, and the gather
            width = max(b - a for a, b in (parallel.shard_range(m_total, r, world)
                                           for r in range(world)))
            h2d = 96 * n + 24 * m + 32 * width
            d2h = 32 * m + 32 * width * world
        e2e = {"value": pairs_job / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
               "ms_per_step": e2e_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # The plain FP64 form on the same inputs, and the FP32 form's error vs it.
    fp64 = None
    if not args.no_fp64:
        solve("f64")
        torch.cuda.synchronize()
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st64 = solve("f64")
        e1.record(stream)
        e1.synchronize()
        ms64 = e0.elapsed_time(e1)
        out64 = [t.cpu().numpy() for t in d_out]
        a = np.concatenate([out32[0] + 1j * out32[1], out32[2] + 1j * out32[3]])
        b = np.concatenate([out64[0] + 1j * out64[1], out64[2] + 1j * out64[3]])
        ia = np.abs(a[:m]) ** 2 + np.abs(a[m:]) ** 2
        ib = np.abs(b[:m]) ** 2 + np.abs(b[m:]) ** 2
        # The same FP64 path with the FMA-based phase reduction (opt-in).
        ctx.set_option("f64_reduction", 1)
        solve("f64")
        torch.cuda.synchronize()
        flush.zero_()
        e0.record(stream)
        solve("f64")
        e1.record(stream)
        e1.synchronize()
        ms64r = e0.elapsed_time(e1)
        ctx.set_option("f64_reduction", 0)
        fp64 = {"value": pairs / (ms64 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms64,
                "reduced_phase_option": {"value": pairs / (ms64r / 1e3) / 1e9, "unit": UNIT,
                                         "ms_per_step": ms64r},
                "speedup_f32pr_vs_f64": (pairs / (ms / 1e3)) / (pairs / (ms64 / 1e3)),
                "rel_l2_field_f32pr_vs_f64": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                "rel_l2_intensity_f32pr_vs_f64": float(np.linalg.norm(ia - ib) / np.linalg.norm(ib))}

    # Roofline of the pair kernel. It is bound by the FP32 FMA pipe and the
    # MUFU unit; both peak rates are measured on this GPU (xk_probe_pipes:
    # lane operations and MUFU results per SM clock) and scaled by the SM
    # clock sampled during the timed region.
    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    clk_mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    pipes = xrt_rs.probe_pipes(ctx)
    fma_rate = pipes["fma_lane_ops_per_clk_sm"]
    mufu_rate = pipes["mufu_ops_per_clk_sm"]
    one_col = bool(stats["one_polarization"])
    # The sweep as issued, per ray x screen pair: FMA-pipe lane cycles (an
    # f32x2 instruction holds the pipe for two lanes' worth) and MUFU results.
    # One amplitude column in the unfolded kernels is carried in polar form:
    # the sums take one f32x2 multiply and two FMAs per pair of points instead
    # of two multiplies and four FMAs (3 lane cycles fewer per pair).
    polar = one_col and not stats["folded"]
    if stats["sweep"] == 1:
        cyc, mufu = (14 if polar else 17) if one_col else 21, 2
    elif stats["sweep"] == 2:  # one f32x2 FMA fewer per pair of points
        cyc, mufu = (13 if polar else 16) if one_col else 20, 2
    else:
        cyc, mufu = (12 if polar else 16) if one_col else 20, 3
    ceiling = sms * min(fma_rate / cyc, mufu_rate / mufu) * clk_mhz * 1e6 / 1e9
    kms = float(np.mean(kern_ms))
    achieved = pairs / (kms / 1e3) / 1e9
    # The reference formula's operation count (kirchhoff.wgsl:79-128, per-ray
    # terms amortised): 34 FMA-pipe and 4 SFU operations per pair, 4 FMA-pipe
    # fewer with one amplitude column. The kernel's phase decomposition needs
    # fewer, so the ratio against this count can exceed 1.
    fma_ops = FMA_OPS_PER_PAIR - (4 if one_col else 0)
    algo_peak = sms * min(fma_rate / fma_ops, mufu_rate / SFU_OPS_PER_PAIR) * clk_mhz * 1e6 / 1e9
    # DRAM bytes of one launch of this workload are not computed from sizes:
    # they come from a single-pass ncu capture of the full-size launch of the
    # default configuration, and are reported for that configuration only.
    full_size = n == 1 << 20 and m == 512 * 512 and stats["phase_bound_rad"] <= 512.0 + 1e-9
    traffic = (DRAM_BYTES_CONFIG1[one_col] if full_size else None)
    roofline = {"bound": "fp32_fma_pipe+mufu", "achieved": achieved, "peak": ceiling,
                "unit": UNIT, "frac": achieved / ceiling, "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
                                   "full-size launch, this workload only" if traffic else None),
                "kernel": "pr_persistent_kernel", "kernel_ms": kms,
                "peak_source": (f"measured pipe rates {fma_rate:.1f} FMA-pipe lane ops and "
                                f"{mufu_rate:.2f} MUFU results per SM clock (xk_probe_pipes) "
                                f"x {sms} SMs x {clk_mhz:.0f} MHz median SM clock in the timed "
                                f"region, over {cyc} FMA-pipe lane cycles and {mufu} MUFU "
                                f"results per pair as the sweep issues them"),
                "kernel_ops_per_pair": {"fma_pipe_lane_cycles": cyc, "mufu": mufu},
                "measured_pipes": pipes,
                "algorithmic_count_equivalent": {
                    "fma_pipe_ops_per_pair": fma_ops, "sfu_ops_per_pair": SFU_OPS_PER_PAIR,
                    "peak": algo_peak, "ratio": achieved / algo_peak}}

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(rays, screen, args.cpu_seconds)

    # Served latency (after the timed region, one GPU): the serving mix as a
    # Poisson stream at a rate one B200 sustains and at the configuration's
    # 200 req/s (about 8x what one B200 computes), each for a bounded window.
    serve = None
    if rank == 0 and world == 1 and not args.no_serve:
        sust = serve_session(ctx, args.serve_rate, args.serve_window, 10.0, seed=0,
                             policy=args.serve_policy)
        over = serve_session(ctx, 200.0, args.serve_window, 10.0, seed=1,
                             policy=args.serve_policy)
        serve = {
            "mix": "rays log-uniform [1e4, 2e6], screen points log-uniform [256, 1e6], "
                   "E ~ U(1, 30) keV, d ~ U(100, 20000) mm, 30 % resident ray sets, "
                   "HBM budget 120 GB, FP32 phase-reduced",
            "policy": ("equal share per running request" if args.serve_policy == 1 else
                       "shortest remaining work first, aged (1 s)"),
            "p99_ms": sust["p99_ms"], "sustainable": sust, "offered_200_req_s": over}
        if fp64:
            # The FP64 path serves at most its single-solve rate: the offered
            # work over that rate is how far its queue would fall behind.
            serve["fp64_plain"] = {
                "capacity_gpair_s": fp64["value"],
                "sustainable_stream_load": sust["offered_gpair_s"] / fp64["value"],
                "offered_200_load": over["offered_gpair_s"] / fp64["value"]}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": single_workload(n, args.grid),
                   "rays": n, "screen_points": m_total, "pairs_per_step": pairs_job,
                   "parallelism": (f"screen-sharded x{world}" if shard else f"replica x{world}"),
                   "l2": "flushed between steps (256 MiB write)",
                   "path": "f32pr", "phase_bound_rad": stats["phase_bound_rad"],
                   "n_tiles": stats["n_tiles"], "n_chunks": stats["n_chunks"],
                   "groups": stats["groups"], "sweep": ["sfu_rcp", "packed_f32x2", "packed_f32x2_linear_series"][stats["sweep"]],
                   "amplitude_columns": 1 if stats["one_polarization"] else 2},
        "e2e": e2e, "fp64_plain": fp64, "two_amplitude_columns": two_col,
        "roofline": roofline, "cpu_baseline": cpu, "serve": serve,
        "clocks": clk, "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
