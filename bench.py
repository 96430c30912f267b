"""Benchmark of the D3Q19 time step (MLUPS) on B200.

Workload (one "step" = one lattice update of the whole lattice): D3Q19 Couette flow on a
512^3 lattice in FP64, BGK tau = 0.6, periodic in x and y, bounce-back at z = 0 and a wall
moving along x at z = 511 (pre_bounce_back + cavity_z_l + post_bounce_back), populations at
rest equilibrium.  MLUPS counts every node of the lattice per step, as the reference's log
operator does (log.cpp:74-88).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision f64|f64_strict|f32|f16|bf16] [--collision bgk|mrt] [--n 512]
    python bench.py --workload precision|batch|serve [...]

Other workloads, one JSON line each: `precision` (MRT flow past a sphere in a 1024x256x256
channel, 20000 steps, at FP64 / FP32 / FP16 / BF16 storage: velocity L2 error, mass drift and drag
against the FP64 run), `batch` (256 independent lattices of mixed sizes and decks in FP32, one
launch per step for all of them, against the same lattices stepped one at a time) and `serve`
(Poisson request streams served by continuous batching with FP16 storage against the plain FP64
path serving the same stream, one request at a time).

The default arm prints one JSON line with the device-timed throughput (`value`), the end-to-end
figure through the C-ABI with host buffers (`e2e`: populations in from pinned memory, the solve,
rho and u of every node back out), the fused kernel's roofline against the measured HBM copy
bandwidth, the CPU baseline (the reference's own functors, all host cores, the median of three
segments on a 128^3 sample), the SM clocks sampled during the timed region, the number of kernel
launches, and two summaries: `tiers` (the same 512^3 workload in FP64 MRT, FP32 and FP16 / BF16
storage, BGK and MRT: ms per step, MLUPS, fraction of the copy bandwidth, kernel) and `serve` (16
requests at 100 req/s served by continuous batching in FP16 against the plain FP64 path one at a
time: p50 / p99 time to solution, aggregate MLUPS).  `--impl reference` times the reference
functors alone (oracle/_ref) on the host, on the same 512^3 workload.
Multi-GPU (torchrun): independent replicas, one lattice per rank, throughput summed over ranks
and timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_POP = {"f64": 8, "f64_strict": 8, "f32": 4, "f16": 2, "bf16": 2}
DEFAULT_VARIANT = {("f64", "bgk"): 4, ("f64", "mrt"): 4, ("f64_strict", "bgk"): 4, ("f64_strict", "mrt"): 4,
                   ("f32", "bgk"): 1, ("f32", "mrt"): 1, ("f16", "bgk"): 9, ("f16", "mrt"): 9,
                   ("bf16", "bgk"): 9, ("bf16", "mrt"): 9}
DTYPE = {"f64": "f64", "f64_strict": "f64", "f32": "f32", "f16": "f32 (f16 storage)", "bf16": "f32 (bf16 storage)"}
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f64", choices=list(BYTES_PER_POP))
    ap.add_argument("--collision", default="bgk", choices=["bgk", "mrt"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--tau", type=float, default=0.6)
    ap.add_argument("--e2e-steps", type=int, default=500, help="time steps per end-to-end solve")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-n", type=int, default=128, help="lattice edge of the CPU baseline sample")
    ap.add_argument("--variant", type=int, default=-1,
                    help="step-kernel variant; -1: the tier's default (the autotuner's pick on 512^3 Couette)")
    ap.add_argument("--autotune", action="store_true", help="time every variant on the lattice and keep the fastest")
    ap.add_argument("--rounding", default="stochastic", choices=["stochastic", "nearest"],
                    help="16-bit storage rounding")
    ap.add_argument("--workload", default="couette", choices=["couette", "precision", "batch", "serve", "parity", "solve"])
    ap.add_argument("--parity-steps", type=int, default=500, help="parity workload: time steps")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="precision workload: linear scale of the 1024x256x256 channel (steps scale alike)")
    ap.add_argument("--tiers", default="f64,f32,f16,f16:nearest,bf16",
                    help="precision workload: storage tiers (\":nearest\": round-to-nearest storage)")
    ap.add_argument("--members", type=int, default=256, help="batch workload: lattices")
    ap.add_argument("--policy", default="fifo", choices=["fifo", "sjf"], help="serve workload: admission order")
    ap.add_argument("--max-active-nodes", type=int, default=0,
                    help="serve workload, sjf: admit while the active lattices hold fewer nodes (0: no cap)")
    ap.add_argument("--batch-variant", type=int, default=-1,
                    help="batch workload: hlbm_batch_tune variant (-1: 8, 9 and 10, report the fastest); "
                         "serve workload: the batch variant (-1: 10)")
    ap.add_argument("--member-steps", type=int, default=2000, help="batch workload: steps of every lattice")
    ap.add_argument("--alone-steps", type=int, default=200,
                    help="batch workload: steps per lattice of the one-at-a-time comparison")
    ap.add_argument("--requests", type=int, default=64, help="serve workload: requests per stream")
    ap.add_argument("--no-tiers", action="store_true",
                    help="default workload: skip the other storage tiers and collisions of the `tiers` object")
    ap.add_argument("--no-serve", action="store_true", help="default workload: skip the `serve` summary")
    ap.add_argument("--serve-requests", type=int, default=16, help="default workload: requests of the serve summary")
    ap.add_argument("--serve-rate", type=float, default=100.0, help="default workload: arrival rate (req/s) of it")
    ap.add_argument("--rates", default="10,100,1000", help="serve workload: arrival rates (req/s)")
    ap.add_argument("--solve", default="channel", choices=["cavity", "channel", "sphere"],
                    help="solve workload: the kind of serving solve stepped alone")
    ap.add_argument("--edges", default="181,150,170", help="solve workload: nodes along x, y, z")
    return ap.parse_args()


def workload_name(a) -> str:
    return f"couette_{a.n}^3_{a.collision}_tau{a.tau}_{a.precision}"


def make_case(a, n=None):
    from hippolbm_b200 import deck

    return deck.couette_case(n or a.n, tau=a.tau, u_wall=0.05, steps=500, collision=a.collision)


# ------------------------------------------------------------------ distributed plumbing
def dist_init(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def dist_max(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device):
    if world > 1:
        import torch.distributed as dist

        dist.barrier(device_ids=[device.index])


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, index: int):
        self.proc = None
        self.index = index
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={CLOCK_FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            p = [s.strip() for s in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ roofline inputs
def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def step_kernel_name(variant: int) -> str:
    """The fused step kernel a single-lattice variant runs on a lattice without wall obstacles
    whose rows split into at least 32 vectors (the Couette workload)."""
    if variant >= 8:
        return "k_step_rows"
    if variant >= 6:
        return "k_step_tma"
    return "k_step_vec" if variant % 2 == 1 else "k_step"


def ncu_traffic_per_node(precision: str, collision: str, kernel: str):
    """DRAM bytes per node per launch of the fused step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d[f"{precision}_{collision}_{kernel}"]["dram_bytes_per_node"])
    except (OSError, KeyError, ValueError):
        return None


# ------------------------------------------------------------------ CPU baseline
def cpu_reference_mlups(n: int, steps, warmup: int, collision: str, tau: float, runs: int = 3):
    """The reference's own functors (oracle/_ref) on all host cores; falls back to the C
    restatement (oracle/_build) when the harness library is absent.  After `warmup` steps, `runs`
    timed segments of `steps` steps each (or of the step counts in the list `steps`); returns the
    median segment's MLUPS with every segment's MLUPS, the kind, the thread count and the total
    timed seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hippolbm_b200 import deck

    kind = "reference" if oracle.available("reference") else "port"
    counts = list(steps) if isinstance(steps, (list, tuple)) else [int(steps)] * runs
    case = deck.couette_case(n, tau=tau, u_wall=0.05, steps=sum(counts), collision=collision)
    lat = oracle.OracleLattice(case, kind).initialize()
    lat.step(warmup)
    segs = []
    for k in counts:
        t0 = time.perf_counter()
        lat.step(k)
        segs.append(time.perf_counter() - t0)
    lat.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", "0")) or (os.cpu_count() or 1)
    mlups = [n ** 3 * k / dt / 1e6 for k, dt in zip(counts, segs)]
    return statistics.median(mlups), mlups, kind, cores, sum(segs)


# ------------------------------------------------------------------ reference arm
def run_reference(a):
    """The reference's functors on the headline workload itself (512^3 by default): W warm-up
    steps, then K steps timed as three segments; the median segment is the value."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = a.n
    segs = [a.steps // 3 + (1 if i < a.steps % 3 else 0) for i in range(3)]  # K steps in three segments
    segs = [k for k in segs if k > 0]
    mlups, runs, kind, cores, dt = cpu_reference_mlups(n, segs, a.warmup, a.collision, a.tau)
    sample = (f"couette {n}^3 {a.collision} tau={a.tau} FP64 in the reference's ghosted layout: {a.warmup} "
              f"warm-up steps, then {a.steps} steps timed as segments of {segs} steps, median segment; OpenMP "
              f"static over {cores} host threads")
    line = {"metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(n ** 3 / (mlups * 1e6) * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name(a), "nodes": [n, n, n], "collision": a.collision, "tau": a.tau,
                       "segments_mlups": [round(v, 3) for v in runs]},
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ tiers and serving summaries
TIERS = [("f64", "mrt"), ("f32", "bgk"), ("f32", "mrt"), ("f16", "bgk"), ("f16", "mrt"), ("bf16", "bgk")]


def measure_tier(a, precision: str, collision: str, local: int, peak: float) -> dict:
    """The headline workload at another storage tier / collision: the tier's default kernel
    variant, W warm-up steps, K steps timed by CUDA events on the lattice's stream."""
    import torch

    from hippolbm_b200 import deck
    from hippolbm_b200.lattice import Lattice

    case = deck.couette_case(a.n, tau=a.tau, u_wall=0.05, steps=500, collision=collision)
    variant = DEFAULT_VARIANT[(precision, collision)]
    with Lattice.from_case(case, precision, device=local) as lat:
        lat.tune(variant)
        stream = torch.cuda.ExternalStream(lat.stream_handle(), device=torch.device("cuda", local))
        lat.step(a.warmup)
        lat.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lat.step(a.steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        nodes = lat.ncell
    alg = 38 * BYTES_PER_POP[precision] + 1
    gbs = nodes * alg / (ms * 1e-3) / 1e9
    return {"precision": precision, "collision": collision, "ms_per_step": round(ms, 4),
            "mlups": round(nodes / (ms * 1e-3) / 1e6, 1), "algorithmic_gbs": round(gbs, 1),
            "frac": round(gbs / peak, 4), "algorithmic_bytes_per_node": alg,
            "kernel": f"hlbm::{step_kernel_name(variant)}", "variant": variant}


def serve_summary(a) -> dict:
    """Continuous batching of a Poisson request stream (FP16 storage, HBM admission budget 160 GB)
    against the plain FP64 path serving the same stream one request at a time."""
    from hippolbm_b200 import serve

    fast = serve.serve_batched(serve.make_stream(a.serve_rate, a.serve_requests), "f16", hbm_budget=160e9, variant=10)
    plain = serve.serve_plain(serve.make_stream(a.serve_rate, a.serve_requests), "f64")
    keep = ("p50_s", "p99_s", "mean_s", "wall_s", "aggregate_mlups", "converged")
    return {"rate_per_s": a.serve_rate, "requests": a.serve_requests, "edges": [24, 192], "budgets": [500, 20000],
            "batched_f16": {k: fast[k] for k in keep}, "plain_f64": {k: plain[k] for k in keep},
            "mlups_ratio": round(fast["aggregate_mlups"] / plain["aggregate_mlups"], 3)}


# ------------------------------------------------------------------ our arm
def run_ours(a):
    import numpy as np
    import torch

    from hippolbm_b200.lattice import Lattice

    rank, world, local = dist_init(a)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    case = make_case(a)
    lat = Lattice.from_case(case, a.precision, device=local)
    lat.rounding(a.rounding)
    stream = torch.cuda.ExternalStream(lat.stream_handle(), device=device)
    nodes = lat.ncell
    # the tier's default step-kernel variant (the autotuner's pick on this workload), or the
    # autotuner's pick on this lattice (state unchanged)
    if a.autotune:
        variant, variant_ms = lat.autotune(reps=3)
    else:
        variant, variant_ms = (a.variant if a.variant >= 0 else DEFAULT_VARIANT[(a.precision, a.collision)]), {}
        lat.tune(variant)
    # warm-up
    lat.step(a.warmup)
    lat.sync()
    launches0 = lat.info()["launches"]
    barrier(world, device)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lat.step(a.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world, device)
    launches = lat.info()["launches"] - launches0
    ms = e0.elapsed_time(e1)
    ms_max = dist_max(ms, world, device)
    ms_per_step = ms_max / a.steps
    mlups_total = world * nodes * a.steps / (ms_max * 1e-3) / 1e6
    state = lat.simulation_state()
    lat.close()
    del lat

    # end to end through the C-ABI with host buffers: one solve = H2D of the initial populations
    # from pinned memory, e2e_steps time steps, and D2H of the result -- the macroscopic fields
    # rho and u of every node (macro_variables) and simulation_state -- into pinned memory.
    e2e = None
    lat = Lattice.from_case(case, a.precision, device=local)
    lat.rounding(a.rounding)
    lat.tune(variant)
    init = torch.empty(19 * nodes, dtype=torch.float64, pin_memory=True)
    rho_out = torch.empty(nodes, dtype=torch.float64, pin_memory=True)
    u_out = torch.empty(3 * nodes, dtype=torch.float64, pin_memory=True)
    w = [1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12  # rest equilibrium, rho = 1
    iv = init.numpy().reshape(19, nodes)
    for i in range(19):
        iv[i] = w[i]
    stats = (C.c_double * 3)()
    L = lat.L
    dp = C.POINTER(C.c_double)

    def solve():
        rc = L.hlbm_put_populations(lat.h, C.cast(init.data_ptr(), dp))
        rc = rc or L.hlbm_step(lat.h, a.e2e_steps)
        rc = rc or L.hlbm_macro_variables(lat.h, C.cast(rho_out.data_ptr(), dp), C.cast(u_out.data_ptr(), dp))
        rc = rc or L.hlbm_simulation_state(lat.h, stats)
        if rc:
            raise RuntimeError(L.hlbm_last_error().decode())

    solve()  # warm-up solve
    barrier(world, device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solve()
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    t_e2e = dist_max(t_e2e, world, device)
    h2d = 19 * nodes * 8
    d2h = 4 * nodes * 8 + 24
    e2e = {"value": round(world * nodes * a.e2e_steps / t_e2e / 1e6, 3), "unit": "MLUPS",
           "h2d_bytes_per_step": int(h2d / a.e2e_steps), "d2h_bytes_per_step": int(d2h / a.e2e_steps),
           "steps_per_solve": a.e2e_steps, "h2d_bytes_per_solve": h2d, "d2h_bytes_per_solve": d2h,
           "step": f"one solve: put_populations (pinned host) + {a.e2e_steps} time steps + macro_variables "
                   f"(rho, u to pinned host) + simulation_state"}
    lat.close()
    del init, rho_out, u_out

    out = None
    if rank == 0:
        bpp = BYTES_PER_POP[a.precision]
        alg_bytes_per_node = 38 * bpp + 1
        achieved = nodes * alg_bytes_per_node / (ms_per_step * 1e-3) / 1e9
        peak, peak_kind = measured_hbm_peak()
        kname = step_kernel_name(variant)
        tpn = ncu_traffic_per_node(a.precision, a.collision, kname)
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} copy bandwidth",
                "traffic": round(tpn * nodes) if tpn else None,
                "algorithmic_bytes_per_node": alg_bytes_per_node, "kernel": f"hlbm::{kname} (MODE_FUSED)"}
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            cpu_steps = 50  # three segments: about 10 s of host work on 16 cores
            mlups_c, runs_c, kind, cores, dt = cpu_reference_mlups(a.cpu_n, cpu_steps, 2, a.collision, a.tau)
            cpu = {"value": round(mlups_c, 3), "unit": "MLUPS", "cores": cores, "kind": kind,
                   "sample": f"couette {a.cpu_n}^3 {a.collision} tau={a.tau} FP64 (a {a.cpu_n}^3 sample of the "
                             f"{a.n}^3 workload): 3 segments of {cpu_steps} steps ({dt:.1f} s), median segment, "
                             f"through the reference functors, OpenMP over {cores} threads",
                   "segments_mlups": [round(v, 3) for v in runs_c]}
        tiers = None
        if not a.no_tiers and world == 1:
            tiers = [measure_tier(a, prec, coll, local, peak) for prec, coll in TIERS]
            for t in tiers:
                t["vs_f64_bgk"] = round(t["mlups"] / (nodes / (ms_per_step * 1e-3) / 1e6), 3)
        serving = None if (a.no_serve or world > 1) else serve_summary(a)
        out = {"metric": "MLUPS", "value": round(mlups_total, 3), "unit": "MLUPS", "n_gpus": world,
               "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 5),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[a.precision],
               "data": "synthetic",
               "config": {"workload": workload_name(a), "nodes": [a.n] * 3, "collision": a.collision,
                          "tau": a.tau, "u_wall": 0.05, "precision": a.precision, "rounding": a.rounding,
                          "l2": f"inputs larger than L2: {2 * 19 * nodes * bpp / 1e9:.1f} GB of populations",
                          "parallelism": f"replicas x{world}", "state_after": list(state),
                          "kernel_variant": variant,
                          "autotune_ms": {str(k): round(v, 4) for k, v in variant_ms.items()}},
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches) * world,
               "clocks": clk, "tiers": tiers, "serve": serving}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ other workloads
def run_precision(a):
    from hippolbm_b200.deck import sphere_channel_case
    from hippolbm_b200.precision import precision_study

    k = a.scale
    nodes = (int(round(1024 * k)), int(round(256 * k)), int(round(256 * k)))
    steps = int(round(20000 * k))
    case = sphere_channel_case(nodes, (256 * k, 128 * k, 128 * k), 24 * k, tau=0.56, u_in=0.04, steps=steps)
    t0 = time.perf_counter()
    recs = precision_study(case, tuple(a.tiers.split(",")), steps)
    by = {r["precision"]: r for r in recs}
    low = by.get("f16") or recs[-1]
    line = {"workload": "precision", "metric": "rel_l2_velocity_error", "value": low["l2_u"], "unit": "1",
            "tier": low["precision"], "higher_is_better": False, "n_gpus": 1, "steps": steps,
            "data": "synthetic", "dtype": "f64 / f32 / f32 (f16 storage) / f32 (bf16 storage)",
            "config": {"workload": f"sphere_channel_{nodes[0]}x{nodes[1]}x{nodes[2]}_mrt_tau0.56_u0.04",
                       "sphere": {"center": [256 * k, 128 * k, 128 * k], "radius": 24 * k},
                       "mrt_rates": list(case.mrt_rates), "outlet": "zero_gradient", "inlet": "neumann u_x=0.04"},
            "tiers": recs, "wall_s": round(time.perf_counter() - t0, 1)}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(a):
    """The batch workload with each batch kernel (--batch-variant, or 8, 9 and 10 with -1); the
    line's value is the fastest, the others are listed."""
    import torch

    from hippolbm_b200.batch import Batch
    from hippolbm_b200.deck import mixed_batch_cases
    from hippolbm_b200.lattice import Lattice

    torch.cuda.set_device(0)
    cases = mixed_batch_cases(a.members, steps=a.member_steps)
    variants = [8, 9, 10] if a.batch_variant < 0 else [a.batch_variant]
    runs = {}
    for variant in variants:
        lats = [Lattice.from_case(c, "f32") for c in cases]
        nodes = sum(l.ncell for l in lats)
        batch = Batch("f32")
        batch.tune(variant)
        for l in lats:
            batch.add(l)
        stream = torch.cuda.ExternalStream(batch.stream_handle(), device=torch.device("cuda", 0))
        batch.step(a.warmup)
        torch.cuda.synchronize()
        info0 = batch.info()
        clocks = ClockSampler(0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.step(a.member_steps - a.warmup)
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1)
        timed = a.member_steps - a.warmup
        info = batch.info()
        runs[variant] = {"mlups": round(nodes * timed / (ms * 1e-3) / 1e6, 1), "ms_per_step": round(ms / timed, 4),
                         "gpu_launches": info["launches"] - info0["launches"],
                         "graph_replays": info["graph_replays"] - info0["graph_replays"], "clocks": clk}
        batch.close()
        for l in lats:
            l.close()
    best = max(runs, key=lambda v: runs[v]["mlups"])
    # the batch autotuner's pick on the same members (timed one step per kernel, state unchanged)
    lats = [Lattice.from_case(c, "f32") for c in cases]
    with Batch("f32") as tb:
        for l in lats:
            tb.add(l)
        tb.step(2)
        auto_pick, auto_ms = tb.autotune(reps=3)
    for l in lats:
        l.close()
    # the same lattices one at a time, each with its own launches (its default kernel, no graph)
    alone_ms = 0.0
    for c in cases:
        with Lattice.from_case(c, "f32") as l:
            l.step(3)
            s = torch.cuda.ExternalStream(l.stream_handle(), device=torch.device("cuda", 0))
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(s)
            l.step(a.alone_steps)
            f1.record(s)
            f1.synchronize()
            alone_ms += f0.elapsed_time(f1)
    alone = nodes * a.alone_steps / (alone_ms * 1e-3) / 1e6
    kinds = {}
    for c in cases:
        kinds[c.name.split("_")[1]] = kinds.get(c.name.split("_")[1], 0) + 1
    r = runs[best]
    timed = a.member_steps - a.warmup
    line = {"workload": "batch", "metric": "MLUPS", "value": r["mlups"], "unit": "MLUPS", "n_gpus": 1,
            "steps": timed, "warmup": a.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"mixed_batch_{a.members}", "members": a.members, "nodes": nodes,
                       "kinds": kinds, "seed": 20261203, "kernel_variant": best},
            "by_variant": {str(v): runs[v]["mlups"] for v in runs},
            "autotune": {"chosen": auto_pick, "ms_per_step": {str(k): round(v, 4) for k, v in auto_ms.items()}},
            "one_at_a_time_mlups": round(alone, 1), "speedup_vs_one_at_a_time": round(r["mlups"] / alone, 2),
            "gpu_launches": r["gpu_launches"], "graph_replays": r["graph_replays"], "clocks": r["clocks"]}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(a):
    from hippolbm_b200 import serve

    lines = []
    for rate in [float(r) for r in a.rates.split(",")]:
        fast = serve.serve_batched(serve.make_stream(rate, a.requests), "f16", hbm_budget=160e9,
                                   variant=a.batch_variant if a.batch_variant >= 0 else 10, policy=a.policy,
                                   max_active_nodes=a.max_active_nodes or None)
        plain = serve.serve_plain(serve.make_stream(rate, a.requests), "f64")
        lines.append({"rate": rate, "batched_f16": fast, "plain_f64": plain,
                      "mlups_ratio": round(fast["aggregate_mlups"] / plain["aggregate_mlups"], 2)})
    top = lines[-1]
    line = {"workload": "serve", "metric": "aggregate MLUPS", "value": top["batched_f16"]["aggregate_mlups"],
            "unit": "MLUPS", "n_gpus": 1, "higher_is_better": True, "dtype": "f32 (f16 storage)",
            "data": "synthetic",
            "config": {"workload": f"poisson_stream_{a.requests}_requests", "requests": a.requests,
                       "rates": a.rates, "hbm_budget_gb": 160, "edges": [24, 192], "budgets": [500, 20000],
                       "residual_tol": 1e-6},
            "sweep": lines}
    print(json.dumps(line), flush=True)
    return 0


def run_solve(a):
    """One solve of the serving mix (--solve, --edges: every face non-periodic, the operators of
    serve.solve_case) stepped alone at FP64 (variant 4) and at FP16 storage (the pair kernel,
    variant 4, and the row / span pipeline, variant 9): W warm-up steps, K steps timed by CUDA
    events on the lattice's stream, for each."""
    import numpy as np
    import torch

    from hippolbm_b200 import serve
    from hippolbm_b200.lattice import Lattice

    edges = tuple(int(e) for e in a.edges.split(","))
    case = serve.solve_case(a.solve, edges, a.tau, np.random.default_rng(20261203))
    peak, peak_kind = measured_hbm_peak()
    out = []
    for precision, variant in (("f64", 4), ("f16", 4), ("f16", 9)):
        with Lattice.from_case(case, precision) as lat:
            lat.tune(variant)
            stream = torch.cuda.ExternalStream(lat.stream_handle(), device=torch.device("cuda", 0))
            lat.step(a.warmup)
            lat.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lat.step(a.steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / a.steps
            nodes = lat.ncell
        alg = 38 * BYTES_PER_POP[precision] + 1
        out.append({"precision": precision, "variant": variant, "ms_per_step": round(ms, 4),
                    "mlups": round(nodes / (ms * 1e-3) / 1e6, 1),
                    "frac": round(nodes * alg / (ms * 1e-3) / 1e9 / peak, 4)})
    line = {"workload": "solve", "metric": "MLUPS", "value": out[-1]["mlups"], "unit": "MLUPS", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": f"{a.solve}_{edges[0]}x{edges[1]}x{edges[2]}", "tau": a.tau},
            "frac_of": f"{peak_kind} copy bandwidth {peak} GB/s", "by_tier": out}
    print(json.dumps(line), flush=True)
    return 0


def run_parity(a):
    """The Couette workload (--n, --collision, --tau) on the CPU oracle and on the GPU in strict FP64
    and FP64: strict FP64 must equal the oracle in every population, FP64 stay within 1e-12 of it
    relative to each population.  The oracle is the C restatement of the reference (bit-exact
    against the reference functors on every golden case), OpenMP over all host threads."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hippolbm_b200 import deck
    from hippolbm_b200.lattice import Lattice

    case = deck.couette_case(a.n, tau=a.tau, u_wall=0.05, steps=a.parity_steps, collision=a.collision)
    t0 = time.perf_counter()
    ref = oracle.OracleLattice(case, "port").initialize().step(a.parity_steps)
    t_oracle = time.perf_counter() - t0
    f_ref = ref.real(ref.f())
    out = {}
    for precision in ("f64_strict", "f64"):
        with Lattice.from_case(case, precision) as lat:
            lat.step(a.parity_steps)
            f = lat.populations()
        mismatches, worst = 0, 0.0
        for i in range(19):
            a_i, b_i = f[i], f_ref[i]
            mismatches += int(np.count_nonzero(a_i != b_i))
            worst = max(worst, float((np.abs(a_i - b_i) / np.abs(b_i)).max()))
        out[precision] = {"populations_differing": mismatches, "max_rel_diff": worst}
        del f
    ref.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", "0")) or (os.cpu_count() or 1)
    line = {"workload": "parity", "metric": "max relative population difference (FP64 vs oracle)",
            "value": out["f64"]["max_rel_diff"], "unit": "1", "higher_is_better": False, "n_gpus": 1,
            "steps": a.parity_steps, "data": "synthetic",
            "config": {"workload": workload_name(a), "nodes": [a.n] * 3, "collision": a.collision, "tau": a.tau},
            "tolerance": 1e-12, "pass": out["f64_strict"]["populations_differing"] == 0
            and out["f64"]["max_rel_diff"] <= 1e-12,
            "by_precision": out, "oracle": {"kind": "port", "cores": cores, "seconds": round(t_oracle, 1)}}
    print(json.dumps(line), flush=True)
    return 0 if line["pass"] else 1


def main():
    a = parse_args()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "precision":
        return run_precision(a)
    if a.workload == "batch":
        return run_batch(a)
    if a.workload == "serve":
        return run_serve(a)
    if a.workload == "parity":
        return run_parity(a)
    if a.workload == "solve":
        return run_solve(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
