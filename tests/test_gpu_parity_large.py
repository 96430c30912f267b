"""Parity on the headline configuration: D3Q19 Couette flow on a 256^3 lattice (periodic in x and
y, bounce-back at z = 0, a wall moving along x at z = 255 with u = 0.05), BGK at tau = 0.6 and MRT
with the reference's rates (mrt.hpp:43-47, s_nu = 1/tau), 500 time steps from rest.

  - HLBM_F64_STRICT (the reference's operation order, no FMA): every population equal in value to
    the oracle's;
  - HLBM_F64 (FMA, reciprocal multiplies): |f - f_ref| <= 1e-12 * |f_ref| for every population.

The oracle is the C restatement (oracle/hlbm_oracle.c), which reproduces the reference's own
functors bit for bit on every golden case and, at this size, over the first steps
(tests/test_oracle_golden.py::test_port_equals_reference_functors_256).  Sizes above 2^24 nodes per lattice
exercise the 64-bit source indices, the stride padding and the linear node decomposition that
the golden cases (64^3 and smaller) do not reach.
"""
import numpy as np
import pytest

from conftest import per_population_rel_err
from hippolbm_b200 import deck

pytestmark = pytest.mark.gpu
N = 256
STEPS = 500
F64_RTOL = 1e-12


@pytest.fixture(scope="module", params=["bgk", "mrt"])
def reference(request, oracle_mod):
    case = deck.couette_case(N, tau=0.6, u_wall=0.05, steps=STEPS, collision=request.param)
    lat = oracle_mod.OracleLattice(case, "port").initialize().step(STEPS)
    yield case, lat.real(lat.f())  # (19, nz, ny, nx) view into the oracle's populations
    lat.close()


def gpu_populations(case, precision):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.step(case.steps)
        return lat.populations()


def test_strict_f64_equals_oracle_256(reference):
    case, f_ref = reference
    f = gpu_populations(case, "f64_strict")
    for i in range(19):  # one direction at a time: no full-size temporaries
        bad = np.count_nonzero(f[i] != f_ref[i])
        assert bad == 0, f"{case.collision}: direction {i}: {bad} populations differ"


def test_f64_every_population_within_1e12_256(reference):
    case, f_ref = reference
    f = gpu_populations(case, "f64")
    err = per_population_rel_err(f, f_ref)
    assert err <= F64_RTOL, f"{case.collision}: max relative difference {err:.3e}"
