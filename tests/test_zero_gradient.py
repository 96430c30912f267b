"""The zero-gradient outlet (an operator this project adds; the reference has none).

On a face plane, the populations that enter from outside take the streamed values of the interior
neighbour one node inside along the face normal.  Parity is against the oracle's restatement of that
rule (orc_zero_gradient), which no reference test pins.
"""
import numpy as np
import pytest

from conftest import per_population_rel_err
from hippolbm_b200.deck import sphere_channel_case

POST = [(1, 9, 7, 11, 13), (2, 10, 8, 12, 14), (3, 7, 10, 15, 17),
        (4, 8, 9, 16, 18), (5, 14, 11, 18, 15), (6, 13, 12, 17, 16)]


def small_channel(collision="mrt", steps=40):
    return sphere_channel_case((40, 18, 16), (10.0, 9.0, 8.0), 3.0, steps=steps, collision=collision)


@pytest.mark.parametrize("face", range(6))
def test_oracle_copies_interior_neighbour(face, oracle_mod):
    case = small_channel(steps=0)
    lat = oracle_mod.OracleLattice(case).initialize()
    f = lat.f()
    rng = np.random.default_rng(face)
    f[...] = rng.random(f.shape)
    obst = lat.obst().copy()
    lat.lib.orc_snapshot_streamed(lat.h)
    before = f.copy()
    assert lat.lib.orc_zero_gradient(lat.h, face) == 0
    after = lat.f()
    axis, side = face // 2, face % 2
    L = lat.L[axis]
    plane = 2 if side == 0 else L - 3
    nb = plane + 1 if side == 0 else plane - 1
    ax = 2 - axis  # (z, y, x) array axes
    sl = [slice(None)] * 3
    sl_nb = [slice(None)] * 3
    sl[ax], sl_nb[ax] = plane, nb
    fluid = obst[tuple(sl)] == -1
    for c in range(19):
        got, src, old = after[c][tuple(sl)], before[c][tuple(sl_nb)], before[c][tuple(sl)]
        if c in POST[face]:
            assert np.array_equal(got[fluid], src[fluid])
            assert np.array_equal(got[~fluid], old[~fluid])
        else:
            assert np.array_equal(got, old)
    rest = np.ones(after.shape[1:], bool)
    rest[tuple(sl)] = False
    assert np.array_equal(after[:, rest], before[:, rest])
    lat.close()


def test_oracle_sphere_channel_stays_bounded(oracle_mod):
    lat = oracle_mod.OracleLattice(small_channel(steps=300)).initialize().step(300)
    f = lat.real(lat.f())
    rho = f.sum(0)
    assert np.isfinite(f).all()
    assert 0.8 < rho.min() and rho.max() < 1.4
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("collision", ["bgk", "mrt"])
def test_gpu_strict_f64_equals_oracle(collision, oracle_mod):
    from hippolbm_b200.lattice import Lattice

    case = small_channel(collision)
    ref = oracle_mod.OracleLattice(case).initialize().step(case.steps)
    f_ref = ref.real(ref.f()).copy()
    fluid = ref.real(ref.obst()) != -2
    ref.close()
    with Lattice.from_case(case, "f64_strict") as lat:
        lat.step(case.steps)
        f = lat.populations()
    bad = np.argwhere((f != f_ref)[:, fluid])
    assert bad.size == 0, f"{len(bad)} populations differ; first (dir, node) {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1, 6])
@pytest.mark.parametrize("precision,rtol", [("f64", 1e-12), ("f32", 1e-5)])
def test_gpu_kernel_variants_follow_oracle(variant, precision, rtol, oracle_mod):
    from hippolbm_b200.lattice import Lattice

    case = small_channel("mrt", steps=20)
    ref = oracle_mod.OracleLattice(case).initialize().step(case.steps)
    f_ref = ref.real(ref.f()).copy()
    fluid = ref.real(ref.obst()) != -2
    ref.close()
    with Lattice.from_case(case, precision) as lat:
        lat.tune(variant)
        lat.step(case.steps)
        f = lat.populations()
    if precision == "f64":  # every population to 1e-12 relative
        err = per_population_rel_err(f, f_ref, fluid)
        assert err <= rtol, err
    else:  # FP32: 1e-5 of the largest population
        err = np.abs(f - f_ref)[:, fluid].max()
        assert err <= rtol * np.abs(f_ref[:, fluid]).max(), err


@pytest.mark.gpu
def test_gpu_rejects_unknown_region():
    from hippolbm_b200 import capi
    from hippolbm_b200.lattice import Lattice

    with Lattice((8, 8, 8), (0, 0, 0), (8, 8, 8), (True, True, False), "f64") as lat:
        assert lat.L.hlbm_zero_gradient(lat.h, capi.HOOK_POST, capi.ivec([6]), 1) == -1  # HLBM_EINVAL
        assert lat.L.hlbm_zero_gradient(lat.h, capi.HOOK_POST, capi.ivec([5]), 1) == 0
