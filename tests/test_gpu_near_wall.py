"""The near-wall map: the step kernels test a pull's source for a wall node only where the map
says a wall is one step away, so the map must follow every change of the flags.  A lattice whose
walls arrive by hlbm_put_flags or by a checkpoint restore steps exactly like the same lattice whose
walls were rasterised from obstacles, in every precision tier, and in strict FP64 both equal the
oracle."""
import numpy as np
import pytest

from hippolbm_b200.deck import sphere_channel_case

pytestmark = pytest.mark.gpu


def cases():
    with_ball = sphere_channel_case((48, 20, 18), (14.0, 10.0, 9.0), 4.0, steps=30, collision="mrt")
    bare = sphere_channel_case((48, 20, 18), (14.0, 10.0, 9.0), 4.0, steps=30, collision="mrt")
    bare.obstacles = []  # same operators (wall_bounce_back included), no rasterised walls
    return with_ball, bare


@pytest.mark.parametrize("precision", ["f64_strict", "f64", "f32", "f16"])
def test_walls_from_put_flags_step_like_rasterised_walls(precision):
    from hippolbm_b200.lattice import Lattice

    with_ball, bare = cases()
    with Lattice.from_case(with_ball, precision) as a, Lattice.from_case(bare, precision) as b:
        flags = a.flags()
        assert (flags == -2).any()
        b.put_flags(flags)
        a.step(with_ball.steps)
        b.step(with_ball.steps)
        fluid = flags != -2
        assert np.array_equal(a.populations()[:, fluid], b.populations()[:, fluid])


def test_walls_from_a_checkpoint_step_like_rasterised_walls():
    from hippolbm_b200.lattice import Lattice

    with_ball, bare = cases()
    with Lattice.from_case(with_ball, "f16") as a, Lattice.from_case(bare, "f16") as b:
        a.step(7)
        b.restore(a.checkpoint())
        a.step(20)
        b.step(20)
        fluid = a.flags() != -2
        assert np.array_equal(a.populations()[:, fluid], b.populations()[:, fluid])


def test_strict_walls_equal_the_oracle(oracle_mod):
    from hippolbm_b200.lattice import Lattice

    with_ball, _ = cases()
    ref = oracle_mod.OracleLattice(with_ball).initialize().step(with_ball.steps)
    f_ref = ref.real(ref.f()).copy()
    fluid = ref.real(ref.obst()) != -2
    ref.close()
    with Lattice.from_case(with_ball, "f64_strict") as lat:
        lat.step(with_ball.steps)
        assert np.array_equal(lat.populations()[:, fluid], f_ref[:, fluid])


def wide_channel(collision="mrt", steps=25):
    return sphere_channel_case((128, 20, 18), (30.0, 10.0, 9.0), 4.5, steps=steps, collision=collision)


@pytest.mark.parametrize("collision", ["bgk", "mrt"])
def test_vectorised_kernel_with_walls_equals_the_oracle(collision, oracle_mod):
    """The vectorised kernel pulls without the wall test; the wall fix-up pass restores it at the
    nodes the near-wall map marks (strict FP64: every value equal to the oracle's)."""
    from hippolbm_b200.lattice import Lattice

    case = wide_channel(collision)
    ref = oracle_mod.OracleLattice(case).initialize().step(case.steps)
    f_ref = ref.real(ref.f()).copy()
    fluid = ref.real(ref.obst()) != -2
    ref.close()
    with Lattice.from_case(case, "f64_strict") as lat:
        lat.tune(1)
        lat.step(case.steps)
        f = lat.populations()
    assert np.array_equal(f[:, fluid], f_ref[:, fluid])


@pytest.mark.parametrize("precision", ["f32", "f16", "bf16"])
def test_vectorised_kernel_with_walls_matches_one_node_kernel(precision):
    from hippolbm_b200.lattice import Lattice

    case = wide_channel("mrt")
    out = {}
    for variant in (4, 5):
        with Lattice.from_case(case, precision) as lat:
            lat.rounding("nearest")
            lat.tune(variant)
            lat.step(case.steps)
            out[variant] = lat.populations()
            fluid = lat.flags() != -2
    tol = (1e-6 if precision == "f32" else 0.0) * np.abs(out[4]).max()
    assert np.abs(out[4] - out[5])[:, fluid].max() <= tol
