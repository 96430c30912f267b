"""Generate tests/golden/golden.json from the reference's own functors.

Run in a container that has the reference tree (read-only) and oracle/_ref/libhlbm_ref.so
(`make -C oracle`).  For every case it records:
  - the case itself, as this package's Case JSON (regression decks are parsed with
    hippolbm_b200.deck, not copied);
  - the SHA-256 of the real-box populations (float64, (19, nz, ny, nx) C order) and flags
    (int32) after `steps` reference steps, computed by the reference harness;
  - simulation_state after steps-1 and after `steps` (what check_macro_quantities reads is the
    macro of the state at the start of the last step);
  - the deck's check_macro_quantities pins.
Small cases also store the real-box populations in golden_<name>.npz.

    HIPPOLBM_REFERENCE=<reference tree> python tests/golden/make_golden.py [--reference <reference tree>]
"""
import argparse
import glob
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from hippolbm_b200 import deck  # noqa: E402
from hippolbm_b200.deck import Case, Op  # noqa: E402


def builtin_cases():
    """Cases exercising every operator on the step path, in lattice units."""
    cases = []
    c = deck.couette_case(64, tau=0.8, u_wall=0.05, steps=1000)
    c.name = "couette64_bgk_tau0.8"
    cases.append(c)
    c = deck.couette_case(24, tau=0.6, u_wall=0.05, steps=200, collision="mrt")
    c.name = "couette24_mrt_tau0.6"
    cases.append(c)
    c = deck.couette_case(12, tau=0.6, u_wall=0.05, steps=50, collision="mrt")
    c.name = "couette12_mrt_small"
    cases.append(c)
    # channel with a sphere: bounce-back on y/z faces and the sphere, Zou/He velocity inlet
    cases.append(Case(
        name="sphere_channel_64x24x24_mrt", cell_dims=(63, 23, 23), bmin=(0, 0, 0), bmax=(63, 23, 23),
        periodic=(False, False, False), tau=0.8, nuth=(0.8 - 0.5) / 3, collision="mrt",
        obstacles=[("ball", 0, ((16.0, 11.5, 11.5), 4.0))],
        pre_stream_bcs=[Op("pre_bounce_back"), Op("wall_bounce_back")],
        post_stream_bcs=[Op("post_bounce_back")],
        boundary_conditions=[Op("neumann", {"U": [0.01, 0.0, 0.0], "regions": ["plan_yz_0", "plan_yz_l"]})],
        steps=120))
    # Poiseuille: body force, Zou/He no-slip planes, BGK
    cases.append(Case(
        name="poiseuille_20_force", cell_dims=(9, 9, 19), bmin=(0, 0, 0), bmax=(9, 9, 19),
        periodic=(True, True, False), tau=0.9, nuth=(0.9 - 0.5) / 3, Fext=(1e-5, 0.0, 0.0),
        boundary_conditions=[Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_xy_0", "plan_xy_l"]})],
        steps=120))
    # lid-driven cavity, all faces Zou/He-free: BB + lid on the top plane, BGK and MRT
    for col in ("bgk", "mrt"):
        cases.append(Case(
            name=f"lid_cavity_16_{col}", cell_dims=(15, 15, 15), bmin=(0, 0, 0), bmax=(15, 15, 15),
            periodic=(False, False, False), tau=0.7, nuth=(0.7 - 0.5) / 3, collision=col,
            pre_stream_bcs=[Op("pre_bounce_back")],
            post_stream_bcs=[Op("post_bounce_back"), Op("lid_driven_cavity", {"U": [0.05, 0.0, 0.0],
                                                                                "regions": ["plan_xy_l"]})],
            steps=100))
    # cavity_z_0 and cavity_z_l together, Zou/He on x faces, walls + start_iteration reset
    cases.append(Case(
        name="mixed_ops_18x14x12", cell_dims=(17, 13, 11), bmin=(0, 0, 0), bmax=(17, 13, 11),
        periodic=(False, True, False), tau=0.65, nuth=(0.65 - 0.5) / 3,
        init_distributions=[(1.02, (0, 0, 0, 4, 13, 11))],
        obstacles=[("wall", 0, ((7.5, 0.0, 3.5), (9.5, 13.0, 6.5))), ("ball", 1, ((13.0, 7.0, 6.0), 2.2))],
        start_iteration=[Op("set_distribution", {"value": 1.01, "bounds": [[0, 0, 0], [1, 13, 11]]})],
        pre_stream_bcs=[Op("pre_bounce_back"), Op("cavity_z_0", {"U": [0.0, 0.01, 0.0]}),
                        Op("cavity_z_l", {"U": [0.03, 0.0, 0.0]}), Op("wall_bounce_back")],
        post_stream_bcs=[Op("post_bounce_back")],
        boundary_conditions=[Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_yz_l"]})], steps=80))
    # init_double_couette (lbm_prepro_double_couette.msp shape): linear profile along Z / X, Zou/He
    # planes moving in opposite directions
    cases.append(Case(
        name="double_couette_z_20x12x24", cell_dims=(19, 11, 23), bmin=(0, 0, 0), bmax=(0.19, 0.11, 0.23),
        periodic=(True, True, False), nuth=1e-2, celerity=1.0, double_couette={"U": [0.001, 0.0, 0.0], "dimension": "Z"},
        boundary_conditions=[Op("neumann", {"U": [-0.001, 0.0, 0.0], "regions": ["plan_xy_l"]}),
                             Op("neumann", {"U": [0.001, 0.0, 0.0], "regions": ["plan_xy_0"]})],
        steps=20))
    cases.append(Case(
        name="double_couette_x_18x10x8", cell_dims=(17, 9, 7), bmin=(0, 0, 0), bmax=(17, 9, 7),
        periodic=(False, True, True), tau=0.8, nuth=0.1, double_couette={"U": [0.0, 0.02, 0.01], "dimension": "X"},
        boundary_conditions=[Op("neumann", {"U": [0.0, -0.02, -0.01], "regions": ["plan_yz_l"]}),
                             Op("neumann", {"U": [0.0, 0.02, 0.01], "regions": ["plan_yz_0"]})],
        steps=15))
    return cases


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_reference(case):
    lat = oracle.OracleLattice(case, "reference").initialize()
    lat.step(case.steps - 1)
    lat.lib.orc_macro_variables(lat.h)
    st_prev = lat.simulation_state()
    lat.step(1)
    lat.lib.orc_macro_variables(lat.h)
    st = lat.simulation_state()
    f = lat.real(lat.f()).copy()
    obst = lat.real(lat.obst()).copy()
    lat.close()
    return f, obst, st_prev, st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("HIPPOLBM_REFERENCE"),
                    help="the reference tree (default: $HIPPOLBM_REFERENCE)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set HIPPOLBM_REFERENCE to the reference tree")
    if not oracle.available("reference"):
        oracle.build("reference")
    cases = []
    for path in sorted(glob.glob(os.path.join(args.reference, "regression-test", "*.msp"))):
        c = deck.load_msp(path)
        cases.append(c)
    # the reference's double-Couette example deck (init_double_couette), parsed as a user deck
    c = deck.load_msp(os.path.join(args.reference, "example", "lbm_prepro_double_couette.msp"))
    c.name = "example_prepro_double_couette"
    cases.append(c)
    cases += builtin_cases()
    out = {}
    for c in cases:
        f, obst, st_prev, st = run_reference(c)
        entry = {"case": c.to_dict(), "steps": c.steps, "sha_f": sha(f), "sha_obst": sha(obst.astype(np.int32)),
                 "state_prev": list(st_prev), "state": list(st), "pins": c.checks,
                 "shape": list(f.shape), "n_wall": int((obst == -2).sum())}
        if f.size * 8 <= 300_000:
            np.savez_compressed(os.path.join(HERE, f"golden_{c.name}.npz"), f=f, obst=obst.astype(np.int8))
            entry["npz"] = f"golden_{c.name}.npz"
        out[c.name] = entry
        print(c.name, st, entry["sha_f"][:16])
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
