"""The deck runner (`python -m hippolbm_b200.run`): run controls, log line, checker and profile
output of the reference's operators, and whole regression decks on the GPU against the reference's
own statistics and check_macro_quantities pins."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from hippolbm_b200.deck import Case, loads_msp
from hippolbm_b200.run import CheckFailed, check_macro_quantities, format_log_line, write_profile_csv

with open(os.path.join(GOLDEN, "golden.json")) as fh:
    GOLD = json.load(fh)

DECK = """
do_domain:
  - domain:
     bounds:    [ [0, 0, 0],[0.1 m, 0.1 m, 0.1 m] ]
     cell_dims: [ 10 , 10 , 10 ]
     periodic:  [ true, true, false ]
set_lbm_parameters:
  - lbm_parameters:
     nuth: 1e-3
     tau: 0.7
boundary_conditions:
  - neumann: {U: [0.001,0,0], regions: [plan_xy_l]}
  - neumann: {U: [0,0,0], regions: [plan_xy_0]}
analysis:
  - plane_velocity_profile:
     dimension: Z
  - plot_line_velocity:
     line: [[0.05,0.05,0],[0.05,0.05,0.1]]
global:
   simulation_paraview_freq: 100
   simulation_end_iteration: 30
   simulation_analysis_freq: 10
   simulation_print_log_freq: 5
   output_directory: "CouetteTestDir"
"""


def test_run_controls_are_parsed():
    c = loads_msp(DECK)
    assert c.run == {"paraview_freq": 100, "analysis_freq": 10, "print_log_freq": 5,
                     "display_paraview_first_timestep": True, "output_directory": "CouetteTestDir"}
    assert [op.name for op in c.analysis] == ["plane_velocity_profile", "plot_line_velocity"]
    assert c.steps == 30
    c2 = Case.from_dict(json.loads(json.dumps(c.to_dict())))
    assert c2.run == c.run and c2.analysis[0].slots == {"dimension": "Z"}


def test_check_macro_quantities_semantics():
    assert check_macro_quantities((29791.0, 0.0, 0.001), density=29791, tol=1e-6, vmax=0.001) == "Test Pass."
    with pytest.raises(CheckFailed, match="max vel"):
        check_macro_quantities((29791.0, 0.0, 0.0011), vmax=0.001)
    with pytest.raises(CheckFailed, match="Sum of densities"):
        check_macro_quantities((29791.5, 0.0, 0.0), density=29791, tol=0.1)
    with pytest.raises(CheckFailed, match="tolerance"):
        check_macro_quantities((1.0, 0.0, 0.0), density=1.0)
    # min velocity and the 1e-15 slack of check_marco_quantities.cpp:82-96
    assert check_macro_quantities((1.0, 0.0, 0.001 + 5e-16), vmax=0.001) == "Test Pass."
    with pytest.raises(CheckFailed, match="min vel"):
        check_macro_quantities((1.0, 0.01, 0.02), vmin=0.02)


def test_log_line_and_profile_format(tmp_path):
    line = format_log_line(100, 0.05, 1030301, (1030301.0, 0.0, 0.001), 2.0, 1234.5)
    assert line == "      100  5.000000e-02       1030301       1.03e+06     0.00e+00     2.00e-03   1.23e+03"
    p = tmp_path / "p.csv"
    write_profile_csv(str(p), 0.0, 0.01, [0.5, 0.0], [0.25, 1.79769313486231570815e308],
                      [1.0, -1.79769313486231570815e308])
    rows = p.read_text().splitlines()
    assert rows[0] == "        position             avg             min             max"
    assert rows[1] == "               0             0.5            0.25               1"
    assert rows[2].split() == ["0.01", "0", "1.7976931e+308", "-1.7976931e+308"]


REGRESSION = sorted(k for k in GOLD if k.startswith("regression_"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", REGRESSION)
def test_regression_deck_runs_and_passes_its_pins(name, tmp_path, monkeypatch):
    from hippolbm_b200.run import Runner

    monkeypatch.chdir(tmp_path)
    g = GOLD[name]
    case = Case.from_dict(g["case"])
    r = Runner(case, "f64_strict", quiet=True, paraview=False)
    try:
        r.initialize()
        r.compute_loop()
        msgs = r.finish()
        assert r.timestep == case.steps
        st = r.check_stats
    finally:
        r.close()
    assert all(m == "Test Pass." for m in msgs) and len(msgs) == len(case.checks)
    ref = g["state_prev"]  # what the reference's checker reads: the macro of the last iteration's start
    assert abs(st[0] - ref[0]) <= 1e-12 * abs(ref[0])
    assert st[1] == ref[1] and st[2] == ref[2]


@pytest.mark.gpu
@pytest.mark.parametrize("dim", ["X", "Y", "Z"])
def test_plane_velocity_profile_matches_oracle(dim, oracle_mod):
    from hippolbm_b200.lattice import Lattice

    case = Case.from_dict(GOLD["mixed_ops_18x14x12"]["case"])
    ref = oracle_mod.OracleLattice(case).initialize().step(case.steps)
    a_ref, lo_ref, hi_ref, n_ref = ref.plane_velocity_profile(dim)
    ref.close()
    with Lattice.from_case(case, "f64_strict") as lat:
        lat.step(case.steps)
        a, lo, hi, n = lat.plane_velocity_profile(dim)
    assert np.array_equal(n, n_ref)
    assert np.array_equal(lo, lo_ref) and np.array_equal(hi, hi_ref)
    assert np.allclose(a, a_ref, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_runner_writes_outputs_and_restarts(tmp_path, monkeypatch):
    from hippolbm_b200.run import main

    monkeypatch.chdir(tmp_path)
    deck = tmp_path / "couette.msp"
    deck.write_text(DECK)
    assert main([str(deck), "--quiet", "--checkpoint-every", "10", "--checkpoint", "ck.bin"]) == 0
    prof = tmp_path / "CouetteTestDir" / "Profile" / "profile_0000000030.csv"
    assert prof.exists() and len(prof.read_text().splitlines()) == 12
    assert (tmp_path / "CouetteTestDir" / "ParaviewOutput" / "hippoLBM_0000000000.pvtr").exists()
    assert (tmp_path / "CouetteTestDir" / "ParaviewOutput" / "hippoLBM_0000000030.pvtr").exists()
    assert (tmp_path / "ck.bin").exists()
    assert main([str(deck), "--quiet", "--restart", "ck.bin", "--no-paraview"]) == 0
