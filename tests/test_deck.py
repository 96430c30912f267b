"""The .msp reader: Onika YAML subset, units, includes, errors the reference raises."""
import os

import pytest

from hippolbm_b200 import deck
from hippolbm_b200.deck import DeckError

DECK = """
do_domain:
  - domain:
     bounds: [[0 m, 0 m, 0 m], [0.2 m, 0.1 m, 0.1 m]]
     cell_dims: [ 20, 10, 10 ]
     periodic: [true, false, false]
set_lbm_parameters:
  - lbm_parameters:
     Fext: [1e-5, 0, 0]
     nuth: 1e-4
     celerity: 2
set_obstacles:
  - register_solid_ball:
     id: 0
     center: [0.05, 0.05, 0.05]
     radius: 0.02
  - register_solid_wall:
     id: 1
     bounds: [[0.1, 0, 0], [0.12, 0.1, 0.04]]
pre_stream_bcs:
  - pre_bounce_back
  - cavity_z_l:
     U: [0.01, 0, 0]
  - wall_bounce_back
post_stream_bcs:
  - post_bounce_back
boundary_conditions:
  - neumann:
     U: [0.001, 0, 0]
     regions: [plan_xy_l, plan_xy_0]
collision: mrt
global:
  simulation_end_iteration: 42
"""


def test_parse_full_deck():
    c = deck.loads_msp(DECK)
    assert c.nodes == (21, 11, 11)
    assert c.dx == pytest.approx(0.01)
    assert c.periodic == (True, False, False)
    assert c.Fext == (1e-5, 0.0, 0.0) and c.nuth == 1e-4 and c.celerity == 2.0
    assert c.collision == "mrt" and c.steps == 42
    assert [op.name for op in c.pre_stream_bcs] == ["pre_bounce_back", "cavity_z_l", "wall_bounce_back"]
    assert c.boundary_conditions[0].slots["regions"] == ["plan_xy_l", "plan_xy_0"]
    assert c.obstacles[0][0] == "ball" and c.obstacles[1][0] == "wall"


def test_parameters_follow_define_by_c():
    c = deck.loads_msp(DECK)
    p = deck.lbm_parameters(c)
    dt = c.dx / 2.0
    assert p["dtLB"] == dt
    assert p["tau"] == 3.0 * (1e-4 * dt / (c.dx * c.dx)) + 0.5


def test_stale_grid_dims_deck_is_rejected():
    """The perf decks use `grid_dims`; `domain` requires `cell_dims` (domain_lbm.cpp:47)."""
    text = "do_domain:\n  - domain:\n     bounds: [[0,0,0],[1,1,1]]\n     grid_dims: [8,8,8]\n     periodic: [true,true,true]\n"
    with pytest.raises(DeckError, match="cell_dims"):
        deck.loads_msp(text)


def test_inconsistent_dx_is_rejected():
    text = "do_domain:\n  - domain:\n     bounds: [[0,0,0],[1,1,2]]\n     cell_dims: [8,8,8]\n     periodic: [true,true,true]\n"
    with pytest.raises(DeckError, match="Dx"):
        deck.loads_msp(text)


def test_unknown_region_is_rejected():
    text = DECK.replace("plan_xy_0]", "plan_zz_0]")
    with pytest.raises(DeckError, match="Traversal"):
        deck.loads_msp(text)


def test_includes(tmp_path):
    (tmp_path / "common.msp").write_text("set_lbm_parameters:\n  - lbm_parameters:\n     tau: 0.7\n     nuth: 0.1\n")
    (tmp_path / "main.msp").write_text(
        "includes:\n  - common.msp\ndo_domain:\n  - domain:\n     bounds: [[0,0,0],[4,4,4]]\n"
        "     cell_dims: [4,4,4]\n     periodic: [true,true,true]\n")
    c = deck.load_msp(str(tmp_path / "main.msp"))
    assert c.tau == 0.7 and c.nuth == 0.1


def test_case_roundtrip():
    c = deck.loads_msp(DECK)
    c2 = deck.Case.from_dict(c.to_dict())
    assert c2 == c
