"""Continuous-batching solve server (no reference counterpart).

Requests arrive over time (a Poisson stream).  Each is a D3Q19 solve -- lid-driven cavity,
channel with a velocity inlet, or channel around a sphere -- with a step budget and, optionally, a
steady-state target: the relative L2 change of the velocity field between checks
(`hlbm_residual`, FP64 on the device) below a tolerance.  The server admits waiting requests in
arrival order (or, with the "sjf" policy, smallest work first, up to a cap on the active nodes)
while their HBM footprint fits the budget, keeps their populations resident, and
advances every admitted lattice together: one batched kernel launch per time step
(`hlbm_batch_step`), in chunks.  Between chunks it retires finished solves, frees their memory
and admits new ones, so requests that arrive while others run join the next chunk.  Time to
solution = finish - arrival.

The plain path serves the same stream one request at a time, each lattice on its own (`Lattice`),
with the same chunking and residual checks.
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from .batch import Batch
from .deck import Case, Op
from .lattice import Lattice

BYTES = {"f64": 8, "f64_strict": 8, "f32": 4, "f16": 2, "bf16": 2}


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float
    case: Case
    budget: int
    tol: float | None = None
    admitted: float | None = None
    finished: float | None = None
    steps: int = 0
    residual: float = math.inf
    lat: Lattice | None = None
    result: np.ndarray | None = None  # final populations, when the server keeps them

    @property
    def nodes(self) -> int:
        return int(np.prod(self.case.nodes))


def footprint_bytes(case: Case, precision: str) -> int:
    """Device bytes a resident solve holds: two population lattices, flags, velocity snapshot."""
    n = int(np.prod(case.nodes))
    stride = (n + 127) // 128 * 128
    return 2 * 19 * stride * BYTES[precision] + n + 3 * 4 * n + (1 << 16)


def solve_case(kind: str, edges, tau: float, rng) -> Case:
    nx, ny, nz = (int(e) for e in edges)
    c = Case(name=f"{kind}_{nx}x{ny}x{nz}", cell_dims=(nx - 1, ny - 1, nz - 1), bmin=(0, 0, 0),
             bmax=(nx - 1, ny - 1, nz - 1), tau=tau, nuth=(tau - 0.5) / 3, collision="bgk", steps=0)
    if kind == "cavity":
        c.periodic = (False, False, False)
        c.pre_stream_bcs = [Op("pre_bounce_back")]
        c.post_stream_bcs = [Op("post_bounce_back"),
                             Op("lid_driven_cavity", {"U": [float(rng.uniform(0.02, 0.1)), 0.0, 0.0],
                                                      "regions": ["plan_xy_l"]})]
    else:
        c.periodic = (False, False, False)
        u = float(rng.uniform(0.01, 0.05))
        c.pre_stream_bcs = [Op("pre_bounce_back")]
        c.post_stream_bcs = [Op("post_bounce_back")]
        c.boundary_conditions = [Op("neumann", {"U": [u, 0.0, 0.0], "regions": ["plan_yz_0", "plan_yz_l"]})]
        if kind == "sphere":
            r = float(rng.uniform(0.1, 0.2)) * min(nx, ny, nz)
            c.obstacles = [("ball", 0, ((nx / 3.0, ny / 2.0, nz / 2.0), r))]
            c.pre_stream_bcs.append(Op("wall_bounce_back"))
    return c


def make_stream(rate: float, count: int, seed: int = 20261203, edge_range=(24, 192), budget_range=(500, 20000),
                tol: float = 1e-6, tol_fraction: float = 0.5) -> list[Request]:
    """Poisson arrivals at `rate` per second; cavity / channel / sphere solves with log-uniform edge
    lengths, tau uniform in [0.55, 1.0], a step budget uniform in budget_range, and (for
    tol_fraction of them) a steady-state residual target."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = np.log(edge_range[0]), np.log(edge_range[1])
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        kind = str(rng.choice(["cavity", "channel", "sphere"]))
        edges = np.round(np.exp(rng.uniform(lo, hi, size=3))).astype(int)
        tau = float(rng.uniform(0.55, 1.0))
        case = solve_case(kind, edges, tau, rng)
        budget = int(rng.integers(budget_range[0], budget_range[1] + 1))
        out.append(Request(i, t, case, budget, tol if rng.random() < tol_fraction else None))
    return out


def _done(r: Request, check_every: int) -> bool:
    if r.steps >= r.budget:
        return True
    if r.tol is not None and r.steps % check_every == 0:
        r.residual = r.lat.residual()
        return r.residual < r.tol
    return False


def _stats(reqs: list[Request], t_end: float, precision: str, mode: str) -> dict:
    tts = np.array([r.finished - r.arrival for r in reqs])
    updates = float(sum(r.nodes * r.steps for r in reqs))
    return {"mode": mode, "precision": precision, "requests": len(reqs), "wall_s": round(t_end, 3),
            "p50_s": round(float(np.percentile(tts, 50)), 4), "p99_s": round(float(np.percentile(tts, 99)), 4),
            "mean_s": round(float(tts.mean()), 4), "node_updates": updates,
            "aggregate_mlups": round(updates / t_end / 1e6, 1),
            "converged": int(sum(1 for r in reqs if r.tol is not None and r.residual < r.tol))}


def admit(arrived: list[Request], active: list[Request], used: int, precision: str, hbm_budget: float,
          policy: str = "fifo", max_active_nodes: int | None = None) -> list[Request]:
    """The requests to admit now, in order, from those that have arrived (in arrival order).

    "fifo": arrival order while the HBM footprint fits; a request that does not fit blocks the
    ones behind it.  "sjf": smallest work (nodes x step budget) first, skipping requests that do
    not fit, and, with `max_active_nodes`, only while the active lattices hold fewer nodes than
    that (enough work to fill the GPU; more only shares it and lengthens every solve).  With
    nothing active, the first candidate is always admitted."""
    if policy not in ("fifo", "sjf"):
        raise ValueError(f"unknown admission policy {policy!r}")
    order = arrived if policy == "fifo" else sorted(arrived, key=lambda r: (r.nodes * r.budget, r.arrival))
    nodes = sum(r.nodes for r in active)
    out = []
    for r in order:
        lone = not active and not out
        need = footprint_bytes(r.case, precision)
        if policy == "sjf" and max_active_nodes is not None and nodes >= max_active_nodes and not lone:
            break
        if used + need > hbm_budget and not lone:
            if policy == "fifo":
                break
            continue
        out.append(r)
        used += need
        nodes += r.nodes
    return out


def serve_batched(requests: list[Request], precision: str = "f16", device: int = 0, hbm_budget: float = 160e9,
                  chunk: int = 100, check_every: int = 500, clock=time.perf_counter, keep_results: bool = False,
                  variant: int | None = None, policy: str = "fifo", max_active_nodes: int | None = None) -> dict:
    """Continuous batching: admit (`admit`: policy and cap) while memory allows, advance all
    admitted solves together (`variant`: the batch kernel, hlbm_batch_tune)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    active: list[Request] = []
    finished: list[Request] = []
    used = 0
    batch = Batch(precision, device)
    if variant is not None:
        batch.tune(variant)
    start = clock()
    try:
        while pending or active:
            now = clock() - start
            arrived = [r for r in pending if r.arrival <= now]
            for r in admit(arrived, active, used, precision, hbm_budget, policy, max_active_nodes):
                pending.remove(r)
                r.lat = Lattice.from_case(r.case, precision, device)
                batch.add(r.lat)
                r.admitted = now
                used += footprint_bytes(r.case, precision)
                active.append(r)
            if not active:
                time.sleep(max(0.0, pending[0].arrival - (clock() - start)))
                continue
            k = min(chunk, min(r.budget - r.steps for r in active))
            if any(r.tol is not None for r in active):
                k = min(k, min(check_every - r.steps % check_every for r in active if r.tol is not None))
            batch.step(k)
            for r in active:
                r.steps += k
            for r in list(active):
                if _done(r, check_every):
                    r.finished = clock() - start
                    if keep_results:
                        r.result = r.lat.populations()
                    batch.remove(r.lat)
                    r.lat.close()
                    r.lat = None
                    used -= footprint_bytes(r.case, precision)
                    active.remove(r)
                    finished.append(r)
    finally:
        for r in active:
            if r.lat is not None:
                r.lat.close()
        batch.close()
    out = _stats(finished, clock() - start, precision, "continuous batching")
    out["batch_variant"] = 8 if variant is None else variant
    out["policy"] = policy if max_active_nodes is None else f"{policy}, max {max_active_nodes} active nodes"
    return out


def serve_plain(requests: list[Request], precision: str = "f64", device: int = 0, chunk: int = 100,
                check_every: int = 500, clock=time.perf_counter) -> dict:
    """The plain path: one request at a time, in arrival order, each lattice on its own."""
    pending = sorted(requests, key=lambda r: r.arrival)
    start = clock()
    for r in pending:
        now = clock() - start
        if r.arrival > now:
            time.sleep(r.arrival - now)
        r.lat = Lattice.from_case(r.case, precision, device)
        r.admitted = clock() - start
        while True:
            k = min(chunk, r.budget - r.steps)
            if r.tol is not None:
                k = min(k, check_every - r.steps % check_every)
            r.lat.step(k)
            r.steps += k
            if _done(r, check_every):
                break
        r.lat.sync()
        r.finished = clock() - start
        r.lat.close()
        r.lat = None
    return _stats(pending, clock() - start, precision, "plain, one at a time")
