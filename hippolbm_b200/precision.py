"""Precision study: one deck run at several storage/compute tiers, compared with the FP64 run.

For each tier the deck is initialised, stepped in chunks and read back once at the end.  Against
the FP64 run it reports
  - l2_u:  relative L2 velocity error over fluid nodes, ||u - u_64|| / ||u_64||;
  - mass drift: (M_end - M_0) / M_0 with M = sum of rho over fluid nodes (FP64 device reduction),
    and its difference from the FP64 run's drift;
  - drag: x-force on the wall obstacles by momentum exchange (hlbm_wall_force), and its relative
    difference from the FP64 drag;
  - the run's throughput (MLUPS, wall clock around the synchronised steps).
The tiers are the library's precisions: "f64", "f32" (FP32 storage and arithmetic), "f16" /
"bf16" (FP32 arithmetic in deviation form, 16-bit storage of f_i minus the collision's rest
equilibrium, stochastic rounding); the suffix ":nearest" selects round-to-nearest storage.
"""
from __future__ import annotations

import time

import numpy as np

from .deck import Case
from .lattice import Lattice


def run_tier(case: Case, tier: str, steps: int, chunk: int = 1000, device: int = 0, variant: int | None = None):
    """Run `case` for `steps` at one tier -- a precision, with ":nearest" for round-to-nearest
    storage -- and return (u (3, nz, ny, nx) FP64, fluid mask, record)."""
    precision, _, opts = tier.partition(":")
    opts = [o for o in opts.split("+") if o]
    with Lattice.from_case(case, precision, device) as lat:
        if "nearest" in opts:
            lat.rounding("nearest")
        if variant is not None:
            lat.tune(variant)
        m0 = lat.moments()[0]
        lat.step(1)  # the first launch includes the prologue; time the rest
        lat.sync()
        t0 = time.perf_counter()
        done = 1
        while done < steps:
            k = min(chunk, steps - done)
            lat.step(k)
            done += k
        lat.sync()
        dt = time.perf_counter() - t0
        m1 = lat.moments()[0]
        force = lat.wall_force()
        _, u = lat.macro()
        fluid = lat.flags() == -1
        ncell = lat.ncell
    rec = {"precision": tier, "steps": steps, "mass_start": m0, "mass_end": m1,
           "mass_drift": (m1 - m0) / m0, "drag": force[0], "lift": (force[1], force[2]),
           "mlups": round(ncell * (steps - 1) / dt / 1e6, 1) if steps > 1 else None}
    return u, fluid, rec


def compare(u, u64, fluid, rec, rec64) -> dict:
    du = (u - u64)[:, fluid]
    ref = u64[:, fluid]
    out = dict(rec)
    out["l2_u"] = float(np.sqrt(np.sum(du * du) / np.sum(ref * ref)))
    out["mass_drift_diff"] = rec["mass_drift"] - rec64["mass_drift"]
    out["drag_rel_diff"] = (rec["drag"] - rec64["drag"]) / rec64["drag"] if rec64["drag"] != 0 else None
    return out


def precision_study(case: Case, precisions=("f64", "f32", "f16"), steps: int | None = None, chunk: int = 1000,
                    device: int = 0) -> list[dict]:
    """Run `case` at FP64 first, then at every other tier; one record per tier."""
    steps = case.steps if steps is None else steps
    u64, fluid, rec64 = run_tier(case, "f64", steps, chunk, device)
    out = [compare(u64, u64, fluid, rec64, rec64)]
    for p in precisions:
        if p == "f64":
            continue
        u, _, rec = run_tier(case, p, steps, chunk, device)
        out.append(compare(u, u64, fluid, rec, rec64))
        del u
    return out
