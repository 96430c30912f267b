"""Couette flow from rest against its analytic solution (the 64^3 plain-method configuration).

D3Q19 BGK, tau = 0.8 (nu = 0.1), 64^3 nodes, periodic in x and y, bounce-back at z = 0 and a wall
moving along x at z = 63 with u = 0.05; 1000 steps from rest equilibrium.  Half-way bounce-back
puts the walls half a node outside the end planes, at zeta = z + 1/2 = 0 and H = 64, and
cavity_z_l moves the wall at U_w = u * (1 + 0.5 / (L - 1)), L = 64 nodes along z
(cavity.hpp:57-65).  The flow is the transient, far from steady (H^2 / nu = 41k steps), so u_x(z)
is compared with the finite-gap solution of u_t = nu u_zz, u(0) = 0, u(H) = U_w, u(., 0) = 0:

    u(zeta, t) = U_w zeta / H + (2 U_w / pi) sum_n (-1)^n / n sin(n pi zeta / H) exp(-nu n^2 pi^2 t / H^2)

(the reference plots the semi-infinite startup solution U (1 - erf((L - z) / (2 sqrt(nu t)))),
script/profile/plot_line_couette.py:56-57, which differs from this one by at most 2.6e-7 at
t = 1000: the stationary wall's image term).
The lattice solution is second-order accurate: the largest deviation is 8.7e-6 = 1.7e-4 U; the
bound is 2e-5.
"""
import numpy as np
import pytest

from hippolbm_b200 import deck

N, STEPS, TAU, U = 64, 1000, 0.8, 0.05
BOUND = 2e-5


def analytic_profile(t: float) -> np.ndarray:
    nu, H = (TAU - 0.5) / 3.0, float(N)
    uw = U * (1.0 + 0.5 / (N - 1))
    zeta = np.arange(N) + 0.5
    k = np.arange(1, 4001)[:, None]
    series = np.sum(((-1.0) ** k / k) * np.sin(k * np.pi * zeta / H) * np.exp(-nu * k**2 * np.pi**2 * t / H**2), axis=0)
    return uw * zeta / H + (2.0 * uw / np.pi) * series


def case():
    return deck.couette_case(N, tau=TAU, u_wall=U, steps=STEPS)


def test_analytic_profile_limits():
    """Long times give the steady linear profile; at t = 1000 the finite gap and the semi-infinite
    startup solution the reference plots agree to well within the bound."""
    from math import erf, sqrt

    uinf = analytic_profile(1e9)
    assert np.allclose(uinf, U * (1.0 + 0.5 / (N - 1)) * (np.arange(N) + 0.5) / N, atol=1e-15)
    uw, nu = U * (1.0 + 0.5 / (N - 1)), (TAU - 0.5) / 3.0
    rayleigh = np.array([uw * (1.0 - erf((N - 0.5 - z) / (2.0 * sqrt(nu * STEPS)))) for z in range(N)])
    assert np.abs(analytic_profile(STEPS) - rayleigh).max() < 5e-7  # the stationary wall's image term


def test_oracle_profile_matches_analytic(oracle_mod):
    lat = oracle_mod.OracleLattice(case(), "port").initialize().step(STEPS)
    avg, vmin, vmax, count = lat.plane_velocity_profile("Z")
    lat.close()
    assert (count == N * N).all() and np.abs(vmax - vmin).max() < 1e-15  # uniform planes
    assert np.abs(avg - analytic_profile(STEPS)).max() <= BOUND


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32", "f16"])
def test_gpu_profile_matches_analytic(precision, oracle_mod):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case(), precision) as lat:
        lat.step(STEPS)
        avg, vmin, vmax, count = lat.plane_velocity_profile("Z")
    assert np.abs(avg - analytic_profile(STEPS)).max() <= BOUND
    if precision == "f64":  # and the reference's own arithmetic, to 1e-12
        ref = oracle_mod.OracleLattice(case(), "port").initialize().step(STEPS)
        ravg = ref.plane_velocity_profile("Z")[0]
        ref.close()
        # u near the resting wall is ~1e-7, a difference of O(1) populations: compare to 1e-12 U
        assert np.abs(avg - ravg).max() <= 1e-12 * U
