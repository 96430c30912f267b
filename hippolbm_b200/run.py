"""Run a hippoLBM deck end to end on one B200: the `simulation` sequence of main-config.msp.

    python -m hippolbm_b200.run DECK.msp [--precision f64] [--device 0]
                                [--checkpoint-every N] [--restart FILE] [--quiet]

The sequence, as the reference's graph runs it (main-config.msp, config_initialize.msp,
config_compute_loop.msp, config_io.msp, config_analysis.msp, config_verification.msp):

  initialize:  domain, lbm_parameters, set_distributions, obstacles, macro_variables,
               simulation_state, write_paraview (display_paraview_first_timestep), log, analysis
  compute_loop, timestep t = 1 .. simulation_end_iteration:
               one fused time step, then end_iteration: write_paraview when t % paraview_freq == 0,
               simulation_state + log when t % print_log_freq == 0, analysis when
               t % analysis_freq == 0 (a frequency <= 0 disables the trigger)
  write_paraview, then the checker: simulation_state + check_macro_quantities.

Time steps between two triggers run as one `hlbm_step(n)` call (n fused launches, no host work in
between).  The log line is the reference's (log.cpp:92-99), MLUPS measured between log lines.
Analysis operators: plane_velocity_profile (CSV as plane_velocity_profile.cu:214-257); others are
reported and skipped.  Like the reference, log, analysis and the checker at timestep t see the
macro fields of the iteration's start (the state after t - 1 steps); write_paraview recomputes
them (config_io.msp:12-17), so it shows the state after t steps.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from .deck import Case, load_msp
from .lattice import Lattice

LOG_HEADER = "     Step     Time          Mesh Size   Sum(density)   min(||V||)   max(||V||)     MLUPS"


class CheckFailed(RuntimeError):
    pass


def check_macro_quantities(stats: tuple, density=None, tol=None, vmin=0.0, vmax=None) -> str:
    """check_marco_quantities.cpp:71-114 on (sum rho, min |u|, max |u|); returns "Test Pass." or
    raises CheckFailed with the reference's message."""
    sum_density, min_v, max_v = stats
    errors = []
    if min_v < vmin - 1e-15:
        errors.append(f"min vel (simulation): {min_v:f} is below (user-defined check): {vmin:f}")
    if vmax is not None and max_v > vmax + 1e-15:
        errors.append(f"max vel (simulation): {max_v:f} is upper (user-defined check): {vmax:f}")
    if density is not None:
        if tol is None:
            raise CheckFailed("Please add a tolerance if you use the density INPUT slot.")
        if abs(sum_density - density) > tol:
            errors.append(f"Sum of densities (simulation): {sum_density:f} is not closed to (user-defined check): "
                          f"{density:f} +/- {tol:f}")
    if errors:
        raise CheckFailed("Regression test checker [macro quantities]\n" + "\n".join(errors) + "\n")
    return "Test Pass."


def format_log_line(step: int, time_phys: float, size: int, stats: tuple, celerity: float, mlups: float) -> str:
    """log.cpp:92-99 (velocities converted to physical units, log.cpp:89-90)."""
    return "%9d % .6e %13d       %.2e     %.2e     %.2e   %.2e" % (
        step, time_phys, size, stats[0], stats[1] * celerity, stats[2] * celerity, mlups)


def write_profile_csv(path: str, origin: float, dx: float, avg, vmin, vmax):
    """plane_velocity_profile.cu:236-257: fixed-width columns position avg min max, 8 digits."""
    w = 16
    lines = ["%*s%*s%*s%*s" % (w, "position", w, "avg", w, "min", w, "max")]
    for i in range(len(avg)):
        vals = [origin + i * dx, avg[i], vmin[i], vmax[i]]
        lines.append("".join("%*s" % (w, "%.8g" % v) for v in vals))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


class Runner:
    def __init__(self, case: Case, precision: str = "f64", device: int = 0, out=sys.stdout, quiet=False,
                 paraview: bool = True):
        self.case = case
        self.write_output = paraview
        self.precision = precision
        self.out = out
        self.quiet = quiet
        self.lat = Lattice.from_case(case, precision, device)
        self.prm = self.lat.parameters()
        self.run = {"paraview_freq": -1, "analysis_freq": -1, "print_log_freq": 1,
                    "display_paraview_first_timestep": True, "output_directory": "hippoLBMOutputDir"}
        self.run.update(case.run or {})
        self.size = int(np.prod(case.nodes))
        self.timestep = 0
        self.log_header = True
        self.last_log = None  # (timestep, wall clock)
        self.files: list[str] = []
        self.check_stats = None

    # --------------------------------------------------------------- operators
    def say(self, s: str):
        if not self.quiet:
            print(s, file=self.out, flush=True)

    def log(self, stats: tuple | None = None):
        """simulation_state + log; `stats` are those of the iteration's start state."""
        stats = self.lat.simulation_state() if stats is None else stats
        now = time.perf_counter()
        if self.last_log is None or self.timestep == self.last_log[0]:
            mlups = 0.0
        else:
            mlups = self.size * (self.timestep - self.last_log[0]) / (1e6 * (now - self.last_log[1]))
        self.last_log = (self.timestep, now)
        if self.log_header:
            self.say(LOG_HEADER)
            self.log_header = False
        self.say(format_log_line(self.timestep, self.timestep * self.prm["dtLB"], self.size, stats,
                                 self.prm["celerity"], mlups))
        return stats

    def paraview(self):
        from .output import write_paraview

        if not self.write_output:
            return
        path = write_paraview(self.lat, self.timestep, self.run["output_directory"])
        self.files.append(path)
        self.say(f"writing paraview file: {path}")

    def profiles(self) -> list:
        """plane_velocity_profile of every analysis operator on the current state."""
        out = []
        for op in self.case.analysis:
            if op.name != "plane_velocity_profile":
                out.append((op, None))
                continue
            dim = str(op.slots.get("dimension", "Z")).upper()
            out.append((op, self.lat.plane_velocity_profile(dim) if dim in ("X", "Y", "Z") else None))
        return out

    def analysis(self, results: list | None = None):
        for op, prof in (self.profiles() if results is None else results):
            if op.name != "plane_velocity_profile":
                self.say(f"[analysis] {op.name}: not available in this runner, skipped")
                continue
            if prof is None:
                self.say('[plane_velocity_profile] Please, select a valid dimension "X", "Y", or "Z".')
                continue
            avg, vmin, vmax, _ = prof
            dim = str(op.slots.get("dimension", "Z")).upper()
            base = os.path.join(str(op.slots.get("output_directory", self.run["output_directory"])), "Profile")
            os.makedirs(base, exist_ok=True)
            path = os.path.join(base, str(op.slots.get("dump_file", "profile_%010d.csv")) % self.timestep)
            axis = "XYZ".index(dim)
            write_profile_csv(path, self.case.bmin[axis], self.case.dx, avg, vmin, vmax)
            self.files.append(path)
            self.say(f"writing profile file: {path}")

    @staticmethod
    def due(t: int, freq: int) -> bool:
        return freq > 0 and t % freq == 0

    # --------------------------------------------------------------------- run
    def initialize(self):
        if self.run["display_paraview_first_timestep"]:  # config_io.msp:20-27
            self.paraview()
        self.log()
        self.analysis()

    def compute_loop(self, checkpoint_every: int = 0, checkpoint_path: str | None = None):
        """Timesteps up to simulation_end_iteration.  Log, analysis and the final check read the
        statistics of the iteration's start state S_{t-1}, as the reference's operators read the
        macro fields computed at the start of iteration t; write_paraview recomputes them (S_t)."""
        end = self.case.steps
        run = self.run
        freqs = [run["paraview_freq"], run["print_log_freq"], run["analysis_freq"], checkpoint_every]
        t = self.timestep
        while t < end:
            nxt = end
            for f in freqs:
                if f and f > 0:
                    nxt = min(nxt, (t // f + 1) * f)
            want_log = self.due(nxt, run["print_log_freq"])
            want_ana = self.due(nxt, run["analysis_freq"]) and bool(self.case.analysis)
            want_chk = nxt == end and bool(self.case.checks)
            stats = prof = None
            if want_log or want_ana or want_chk:
                if nxt - 1 > t:
                    self.lat.step(nxt - 1 - t)
                    t = nxt - 1
                stats = self.lat.simulation_state()
                prof = self.profiles() if want_ana else None
            self.lat.step(nxt - t)
            t = self.timestep = nxt
            if self.due(t, run["paraview_freq"]):
                self.paraview()
            if want_log:
                self.log(stats)
            if want_ana:
                self.analysis(prof)
            if want_chk:
                self.check_stats = stats
            if checkpoint_path and self.due(t, checkpoint_every):
                self.lat.save_checkpoint(checkpoint_path)
        self.lat.sync()

    def finish(self) -> list[str]:
        self.paraview()  # main-config.msp: write_paraview after compute_loop
        messages = []
        if self.case.checks:
            stats = self.check_stats if self.check_stats is not None else self.lat.simulation_state()
            for chk in self.case.checks:
                messages.append(check_macro_quantities(stats, density=chk.get("density"), tol=chk.get("tol"),
                                                       vmin=chk.get("vmin", 0.0), vmax=chk.get("vmax")))
            for m in messages:
                self.say(m)
        return messages

    def restart(self, path: str):
        self.lat.load_checkpoint(path)
        self.timestep = self.lat.info()["steps"]

    def close(self):
        self.lat.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m hippolbm_b200.run")
    ap.add_argument("deck")
    ap.add_argument("--precision", default="f64", choices=["f64", "f64_strict", "f32", "f16", "bf16"])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--checkpoint-every", type=int, default=0)
    ap.add_argument("--checkpoint", default=None, help="checkpoint file (written every --checkpoint-every steps)")
    ap.add_argument("--restart", default=None, help="continue from this checkpoint")
    ap.add_argument("--quiet", action="store_true")
    ap.add_argument("--no-paraview", action="store_true", help="skip the write_paraview operators")
    a = ap.parse_args(argv)
    case = load_msp(a.deck)
    r = Runner(case, a.precision, a.device, quiet=a.quiet, paraview=not a.no_paraview)
    try:
        if a.restart:
            r.restart(a.restart)
        else:
            r.initialize()
        ckpt = a.checkpoint or (os.path.join(r.run["output_directory"], "checkpoint.bin") if a.checkpoint_every else None)
        if ckpt:
            os.makedirs(os.path.dirname(os.path.abspath(ckpt)), exist_ok=True)
        r.compute_loop(a.checkpoint_every, ckpt)
        r.finish()
    except CheckFailed as e:
        print(str(e), file=sys.stdout, flush=True)
        return 1
    finally:
        r.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
