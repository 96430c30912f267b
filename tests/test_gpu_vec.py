"""The vectorised step kernel (NPT x-nodes per thread, vector loads, warp-shuffled x pulls) gives
the same populations as the one-node-per-thread kernel.  Without FMA contraction (strict FP64)
and after rounding to 16-bit storage the two agree bit for bit; the FMA tiers may contract a
product differently in the two kernels, so FP64 agrees to 1e-12 and FP32 to 1e-6 of the
largest population (16-bit storage rounds to nearest for the bitwise check; with stochastic
rounding the kernels agree to a few storage quanta).  In strict FP64 both equal the oracle.  Row lengths cover partial warps,
several blocks per row, periodic x and bounce-back x ends."""
import numpy as np
import pytest

from hippolbm_b200.deck import Case, Op

pytestmark = pytest.mark.gpu

NPT = {"f64": 2, "f64_strict": 2, "f32": 4, "f16": 8, "bf16": 8}  # variant 1: one 16-byte vector per plane
RTOL = {"f64": 1e-12, "f64_strict": 0.0, "f32": 1e-6, "f16": 0.0, "bf16": 0.0}
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def case_for(nx, periodic_x, collision):
    ops = dict(pre_stream_bcs=[Op("pre_bounce_back"), Op("cavity_z_l", {"U": [0.04, 0.01, 0.0]}),
                               Op("cavity_z_0", {"U": [0.0, -0.02, 0.0]})],
               post_stream_bcs=[Op("post_bounce_back")],
               boundary_conditions=[Op("neumann", {"U": [0.0, 0.001, 0.0], "regions": ["plan_xz_0"]}),
                                    Op("lid_driven_cavity", {"U": [0.01, 0.0, 0.0], "regions": ["plan_xz_l"]})])
    if not periodic_x:
        ops["boundary_conditions"].append(Op("neumann", {"U": [0.005, 0.0, 0.0], "regions": ["plan_yz_0"]}))
    return Case(name=f"vec_{nx}_{periodic_x}_{collision}", cell_dims=(nx - 1, 5, 7), bmin=(0, 0, 0),
                bmax=(nx - 1, 5, 7), periodic=(periodic_x, False, False), tau=0.75, nuth=0.25 / 3,
                collision=collision, init_distributions=[(1.01, (3.0, 0, 0, 9.0, 5, 7))],
                start_iteration=[Op("set_distribution", {"value": 1.005, "bounds": [[0, 0, 0], [1, 5, 7]]})],
                steps=25, **ops)


def run(case, precision, variant, rounding="nearest"):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.rounding(rounding)
        lat.tune(variant)
        lat.step(case.steps)
        return lat.populations()


@pytest.mark.parametrize("precision", ["f64", "f64_strict", "f32", "f16", "bf16"])
@pytest.mark.parametrize("vectors", [32, 48, 160])
@pytest.mark.parametrize("periodic_x", [True, False])
def test_vector_kernel_matches_scalar_kernel(precision, vectors, periodic_x):
    nx = vectors * NPT[precision]
    for collision in ("bgk", "mrt"):
        case = case_for(nx, periodic_x, collision)
        f0 = run(case, precision, 0)
        f1 = run(case, precision, 1)
        assert np.isfinite(f1).all()
        tol = RTOL[precision] * np.abs(f0).max()
        diff = np.argwhere(np.abs(f0 - f1) > tol)
        assert diff.size == 0, f"{len(diff)} values differ beyond {tol}, first {diff[:4]}"
        if NPT[precision] == 8:
            # stochastic rounding turns a one-ulp FP32 difference between the kernels into a
            # one-quantum difference with probability ulp / quantum: a few quanta at most
            g0 = run(case, precision, 0, "stochastic")
            g1 = run(case, precision, 1, "stochastic")
            dev = np.abs(g0 - W[:, None, None, None]).max()
            quantum = dev * (2.0 ** -10 if precision == "f16" else 2.0 ** -7)
            assert np.abs(g0 - g1).max() <= 8 * quantum


@pytest.mark.parametrize("periodic_x", [True, False])
def test_vector_kernel_strict_equals_oracle(periodic_x, oracle_mod):
    case = case_for(96, periodic_x, "mrt")
    ref = oracle_mod.OracleLattice(case, "port").initialize().step(case.steps)
    f_ref = ref.real(ref.f()).copy()
    f = run(case, "f64_strict", 1)
    assert np.array_equal(f, f_ref)


@pytest.mark.parametrize("variant", range(6))
def test_every_variant_strict_equals_oracle(variant, oracle_mod):
    """All six step-kernel variants (kernel x occupancy target) give the oracle's populations."""
    from hippolbm_b200.lattice import Lattice

    case = case_for(96, False, "bgk")
    ref = oracle_mod.OracleLattice(case, "port").initialize().step(case.steps)
    with Lattice.from_case(case, "f64_strict") as lat:
        lat.tune(variant)
        lat.step(case.steps)
        assert np.array_equal(lat.populations(), ref.real(ref.f()))


def test_autotune_keeps_the_state():
    from hippolbm_b200.lattice import Lattice

    case = case_for(128, True, "mrt")
    with Lattice.from_case(case, "f64") as a, Lattice.from_case(case, "f64") as b:
        a.step(7)
        b.step(7)
        chosen, times = a.autotune(reps=2)
        assert chosen in times and all(t > 0 for t in times.values())
        a.tune(0)
        a.step(5)
        b.step(5)
        assert np.array_equal(a.populations(), b.populations())
