"""Stochastic rounding of the 16-bit storage tiers.

A periodic box at rest with rho = 1 + delta: every node carries the same FP32 post-collision value
in each direction, generally between two storage grid points.  Round to nearest stores the same
grid point everywhere; stochastic rounding stores the two neighbouring grid points in proportion,
so the node average recovers the FP32 value.  Results are reproducible (the random bits hash the
node, the step number and the direction) and differ from round-to-nearest.
"""
import numpy as np
import pytest

from hippolbm_b200.deck import Case

pytestmark = pytest.mark.gpu
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def box(n=32, delta=0.0123, tau=0.8):
    return Case(name="rest_box", cell_dims=(n - 1,) * 3, bmin=(0.0,) * 3, bmax=(float(n - 1),) * 3,
                periodic=(True, True, True), tau=tau, nuth=(tau - 0.5) / 3.0, collision="bgk",
                init_distributions=[(1.0 + delta, None)], steps=1)


def run(precision, mode, steps=1, case=None, initial=False):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case or box(), precision) as lat:
        lat.rounding(mode)
        f0 = lat.populations() if initial else None
        lat.step(steps)
        f = lat.populations()
    return (f0, f) if initial else f


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_stochastic_rounding_splits_between_neighbours(precision):
    """A uniform box: round to nearest stores one grid point per direction everywhere; stochastic
    rounding stores the two neighbouring points, the nearer one on most nodes."""
    near = run(precision, "nearest")
    sto = run(precision, "stochastic")
    n_split = 0
    for i in range(19):
        a = near[i].ravel()
        b = sto[i].ravel()
        assert np.unique(a).size == 1
        vals, counts = np.unique(b, return_counts=True)
        assert vals.size <= 2
        if vals.size == 2:
            n_split += 1
            assert a[0] in vals
            share = counts[int(np.argmin(np.abs(vals - a[0])))] / b.size
            assert share >= 0.5 - 5 / np.sqrt(b.size)
    assert n_split >= 7, n_split


def shear_wave(n=64, amp=1e-3, tau=0.8):
    """Periodic box, u_y(x) = amp sin(2 pi x / n), equilibrium populations (FP64)."""
    c = Case(name="shear_wave", cell_dims=(n - 1, 3, 3), bmin=(0.0,) * 3, bmax=(float(n - 1), 3.0, 3.0),
             periodic=(True, True, True), tau=tau, nuth=(tau - 0.5) / 3.0, collision="bgk", steps=0)
    x = np.arange(n)
    uy = amp * np.sin(2 * np.pi * x / n)
    ey = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
    eu = ey[:, None] * uy[None, :]
    feq = W[:, None] * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * uy[None, :] ** 2)
    f = np.broadcast_to(feq[:, None, None, :], (19, 4, 4, n)).copy()
    return c, f, ey


def decayed_amplitude(case, f_init, ey, precision, mode, steps):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.rounding(mode)
        lat.put_populations(f_init)
        lat.step(steps)
        f = lat.populations()
    uy = (ey[:, None, None, None] * f).sum(0) / f.sum(0)
    n = f.shape[-1]
    return 2.0 / n * (uy.mean(axis=(0, 1)) * np.sin(2 * np.pi * np.arange(n) / n)).sum()


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_stochastic_rounding_removes_stagnation(precision):
    """A decaying shear wave whose per-step change is about one storage quantum: round to nearest
    loses most updates and the amplitude stalls; stochastic rounding follows the FP64 decay."""
    case, f0, ey = shear_wave()
    steps = 1500
    a64 = decayed_amplitude(case, f0, ey, "f64", "nearest", steps)
    a_sto = decayed_amplitude(case, f0, ey, precision, "stochastic", steps)
    a_near = decayed_amplitude(case, f0, ey, precision, "nearest", steps)
    err_sto, err_near = abs(a_sto - a64) / a64, abs(a_near - a64) / a64
    assert err_sto < 0.5 * err_near or err_sto < 1e-3, (a64, a_sto, a_near)
    assert err_sto < 0.05, (a64, a_sto)


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_stochastic_rounding_is_reproducible(precision):
    from hippolbm_b200.deck import couette_case

    case = couette_case(24, 0.7, 0.05, 40)
    a = run(precision, "stochastic", 40, case)
    b = run(precision, "stochastic", 40, case)
    c = run(precision, "nearest", 40, case)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    scale = np.abs(c).max()
    assert np.abs(a - c).max() < 1e-2 * scale


def test_rounding_mode_is_validated():
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(box(8), "f16") as lat:
        assert lat.L.hlbm_storage_rounding(lat.h, 2) == -1
        assert lat.L.hlbm_storage_rounding(lat.h, 0) == 0
