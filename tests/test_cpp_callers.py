"""C++ callers of the C-ABI: a host program that runs regression_lbm_cavite.msp through
include/hippolbm.h alone (tests/cpp/run_cavite.cpp), and the Onika plugin a hippoLBM maintainer
installs (hippolbm_b200/host/onika_plugin.cpp), compiled against a stand-in for Onika's operator
API (tests/cpp/onika_stub) and driven through its operator factory in the deck's operator order
(tests/cpp/run_plugin.cpp).  Both build here; on a GPU both run the deck and meet its
check_macro_quantities pins, and the host program's populations hash to the reference's."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

CXX = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT}/include"]
LINK = [f"-L{ROOT}/hippolbm_b200", "-lhippolbm", f"-Wl,-rpath,{ROOT}/hippolbm_b200"]


def build(out_dir):
    cavite = os.path.join(out_dir, "run_cavite")
    plugin = os.path.join(out_dir, "run_plugin")
    subprocess.run(CXX + [os.path.join(ROOT, "tests", "cpp", "run_cavite.cpp"), "-o", cavite] + LINK, check=True)
    subprocess.run(CXX + [f"-I{ROOT}/tests/cpp/onika_stub", os.path.join(ROOT, "tests", "cpp", "run_plugin.cpp"),
                          os.path.join(ROOT, "hippolbm_b200", "host", "onika_plugin.cpp"), "-o", plugin] + LINK,
                   check=True)
    return cavite, plugin


def test_cpp_callers_build(tmp_path):
    cavite, plugin = build(str(tmp_path))
    assert os.access(cavite, os.X_OK) and os.access(plugin, os.X_OK)


@pytest.mark.gpu
def test_cpp_callers_run_the_cavite_deck(tmp_path):
    with open(os.path.join(GOLDEN, "golden.json")) as fh:
        g = json.load(fh)["regression_lbm_cavite"]
    cavite, plugin = build(str(tmp_path))
    dump = os.path.join(str(tmp_path), "f.bin")
    r = subprocess.run([cavite, "1", dump], capture_output=True, text=True)  # HLBM_F64_STRICT
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Test Pass." in r.stdout
    state = [float(v) for v in r.stdout.split()[:3]]
    assert state[0] == pytest.approx(g["state"][0], rel=1e-13)
    assert state[1] == pytest.approx(g["state"][1], rel=1e-12) and state[2] == pytest.approx(g["state"][2], rel=1e-12)
    f = np.fromfile(dump, dtype=np.float64).reshape(g["shape"])
    assert hashlib.sha256(np.ascontiguousarray(f).tobytes()).hexdigest() == g["sha_f"]
    p = subprocess.run([plugin, "1"], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "Test Pass." in p.stdout
    assert [float(v) for v in p.stdout.split()[:3]] == state  # the same deck, the same library: same numbers
