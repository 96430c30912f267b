"""The CPU oracle reproduces the reference functors bit for bit (golden hashes made by
tests/golden/make_golden.py from oracle/_ref), and the regression decks' own pins hold."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from hippolbm_b200.deck import Case

with open(os.path.join(GOLDEN, "golden.json")) as fh:
    GOLD = json.load(fh)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_matches_reference_functors(name, oracle_mod):
    g = GOLD[name]
    case = Case.from_dict(g["case"])
    lat = oracle_mod.OracleLattice(case, "port").initialize()
    lat.step(case.steps - 1)
    lat.lib.orc_macro_variables(lat.h)
    st_prev = lat.simulation_state()
    lat.step(1)
    f = lat.real(lat.f()).copy()
    obst = lat.real(lat.obst()).astype(np.int32)
    assert sha(obst) == g["sha_obst"], "flag field differs from the reference rasteriser"
    assert sha(f) == g["sha_f"], "populations differ from the reference functors"
    assert st_prev[0] == pytest.approx(g["state_prev"][0], rel=1e-13)
    if "npz" in g:
        z = np.load(os.path.join(GOLDEN, g["npz"]))
        assert np.array_equal(z["f"], f)
    lat.close()


@pytest.mark.parametrize("name", sorted(n for n in GOLD if GOLD[n]["pins"]))
def test_regression_pins(name):
    """check_macro_quantities (check_marco_quantities.cpp:71-114) on the golden state."""
    g = GOLD[name]
    s, vmin, vmax = g["state_prev"]
    for pin in g["pins"]:
        assert vmin >= pin.get("vmin", 0.0) - 1e-15
        if "vmax" in pin:
            assert vmax <= pin["vmax"] + 1e-15
        if "density" in pin:
            assert abs(s - pin["density"]) <= pin["tol"]


def test_reference_harness_agrees_when_available(oracle_mod):
    """With the reference tree present (this container), the harness itself reproduces a hash."""
    if not oracle_mod.available("reference"):
        pytest.skip("oracle/_ref not built")
    g = GOLD["regression_lbm_cavite_wall"]
    case = Case.from_dict(g["case"])
    lat = oracle_mod.OracleLattice(case, "reference").initialize().step(case.steps)
    assert sha(lat.real(lat.f()).copy()) == g["sha_f"]


def test_port_equals_reference_functors_256(oracle_mod):
    """The restatement against the reference's own functors on the 256^3 Couette lattice of the
    large parity test (BGK and MRT, tau = 0.6, 5 steps): equal bit for bit at a size where
    indices pass 2^24."""
    from hippolbm_b200 import deck

    if not oracle_mod.available("reference"):
        pytest.skip("oracle/_ref (the reference functors) not built")
    for collision in ("bgk", "mrt"):
        case = deck.couette_case(256, tau=0.6, u_wall=0.05, steps=5, collision=collision)
        a = oracle_mod.OracleLattice(case, "port").initialize().step(5)
        b = oracle_mod.OracleLattice(case, "reference").initialize().step(5)
        fa, fb = a.real(a.f()), b.real(b.f())
        for i in range(19):
            assert np.array_equal(fa[i], fb[i]), f"{collision}: direction {i} differs"
        a.close()
        b.close()
