"""Benchmark of the D3Q19 time step (MLUPS) on B200.

Workload (one "step" = one lattice update of the whole lattice): D3Q19 Couette flow on a
512^3 lattice in FP64, BGK tau = 0.6, periodic in x and y, bounce-back at z = 0 and a wall
moving along x at z = 511 (pre_bounce_back + cavity_z_l + post_bounce_back), populations at
rest equilibrium.  MLUPS counts every node of the lattice per step, as the reference's log
operator does (log.cpp:74-88).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision f64|f64_strict|f32|f16|bf16] [--collision bgk|mrt] [--n 512]

The default arm prints one JSON line with the device-timed throughput (`value`), the end-to-end
figure through the C-ABI with host buffers (`e2e`), the fused kernel's roofline against the
measured HBM copy bandwidth, the CPU baseline (the reference's own functors, all host cores, a
bounded sample), the SM clocks sampled during the timed region, and the number of kernel
launches.  `--impl reference` times the reference functors alone (oracle/_ref) on the host.
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
    ap.add_argument("--variant", type=int, default=-1, help="step-kernel variant; -1: autotune")
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


def ncu_traffic_per_node(precision: str, collision: str):
    """DRAM bytes per node per launch of the fused step from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d[f"{precision}_{collision}"]["dram_bytes_per_node"])
    except (OSError, KeyError, ValueError):
        return None


# ------------------------------------------------------------------ CPU baseline
def cpu_reference_mlups(n: int, steps: int, warmup: int, collision: str, tau: float):
    """The reference's own functors (oracle/_ref) on all host cores; falls back to the C
    restatement (oracle/_build) when the harness library is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hippolbm_b200 import deck

    kind = "reference" if oracle.available("reference") else "port"
    case = deck.couette_case(n, tau=tau, u_wall=0.05, steps=steps, collision=collision)
    lat = oracle.OracleLattice(case, kind).initialize()
    lat.step(warmup)
    t0 = time.perf_counter()
    lat.step(steps)
    dt = time.perf_counter() - t0
    lat.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", "0")) or (os.cpu_count() or 1)
    return n ** 3 * steps / dt / 1e6, kind, cores, dt


# ------------------------------------------------------------------ reference arm
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = a.cpu_n
    mlups, kind, cores, dt = cpu_reference_mlups(n, a.steps, a.warmup, a.collision, a.tau)
    sample = (f"couette {n}^3 {a.collision} tau={a.tau} FP64 in the reference's ghosted layout, "
              f"{a.steps} steps after {a.warmup} warm-up, OpenMP static over {cores} host threads")
    line = {"metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(dt / a.steps * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name(a), "sample_nodes": [n, n, n], "collision": a.collision,
                       "tau": a.tau},
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


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
    stream = torch.cuda.ExternalStream(lat.stream_handle(), device=device)
    nodes = lat.ncell
    # the project's autotuner picks the step-kernel variant on this lattice (state unchanged)
    if a.variant >= 0:
        variant, variant_ms = a.variant, {}
        lat.tune(variant)
    else:
        variant, variant_ms = lat.autotune(reps=3)
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

    # end to end through the C-ABI with host buffers: H2D of the initial populations from
    # pinned memory, one solve of e2e_steps time steps, D2H of simulation_state.
    e2e = None
    lat = Lattice.from_case(case, a.precision, device=local)
    lat.tune(variant)
    init = torch.empty(19 * nodes, dtype=torch.float64, pin_memory=True)
    w = [1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12  # rest equilibrium, rho = 1
    iv = init.numpy().reshape(19, nodes)
    for i in range(19):
        iv[i] = w[i]
    stats = (C.c_double * 3)()
    L = lat.L

    def solve():
        L.hlbm_put_populations(lat.h, C.cast(init.data_ptr(), C.POINTER(C.c_double)))
        L.hlbm_step(lat.h, a.e2e_steps)
        L.hlbm_simulation_state(lat.h, stats)

    solve()  # warm-up solve
    barrier(world, device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solve()
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    t_e2e = dist_max(t_e2e, world, device)
    e2e = {"value": round(world * nodes * a.e2e_steps / t_e2e / 1e6, 3), "unit": "MLUPS",
           "h2d_bytes_per_step": int(19 * nodes * 8), "d2h_bytes_per_step": 24,
           "step": f"one solve: put_populations (pinned host) + {a.e2e_steps} time steps + simulation_state"}
    lat.close()
    del init

    out = None
    if rank == 0:
        bpp = BYTES_PER_POP[a.precision]
        alg_bytes_per_node = 38 * bpp + 1
        achieved = nodes * alg_bytes_per_node / (ms_per_step * 1e-3) / 1e9
        peak, peak_kind = measured_hbm_peak()
        tpn = ncu_traffic_per_node(a.precision, a.collision)
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} copy bandwidth",
                "traffic": round(tpn * nodes) if tpn else None,
                "algorithmic_bytes_per_node": alg_bytes_per_node, "kernel": "hlbm::k_step (MODE_FUSED)"}
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            cpu_steps = 10
            mlups_c, kind, cores, dt = cpu_reference_mlups(a.cpu_n, cpu_steps, 2, a.collision, a.tau)
            cpu = {"value": round(mlups_c, 3), "unit": "MLUPS", "cores": cores, "kind": kind,
                   "sample": f"couette {a.cpu_n}^3 {a.collision} tau={a.tau} FP64, {cpu_steps} steps "
                             f"({dt:.1f} s) through the reference functors, OpenMP over {cores} threads"}
        out = {"metric": "MLUPS", "value": round(mlups_total, 3), "unit": "MLUPS", "n_gpus": world,
               "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 5),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[a.precision],
               "data": "synthetic",
               "config": {"workload": workload_name(a), "nodes": [a.n] * 3, "collision": a.collision,
                          "tau": a.tau, "u_wall": 0.05, "precision": a.precision,
                          "l2": f"inputs larger than L2: {2 * 19 * nodes * bpp / 1e9:.1f} GB of populations",
                          "parallelism": f"replicas x{world}", "state_after": list(state),
                          "kernel_variant": variant,
                          "autotune_ms": {str(k): round(v, 4) for k, v in variant_ms.items()}},
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches) * world,
               "clocks": clk}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    a = parse_args()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
