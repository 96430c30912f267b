"""The row pipeline of the 16-bit tiers (variants 8 and 9: bulk copies of source rows into shared
memory, node pairs updated from there) gives the same populations as the pair kernel (variant 4),
bit for bit and with stochastic rounding on: both update the same node pairs with the same packed
FP32 arithmetic and round them with the same random bits.  The cases cover periodic and bounced
x ends, bounced y / z rows, tiles of one and of several rows, a tile that wraps a periodic y edge,
boundary operators on every face kind (face pass), wall obstacles (wall fix-up), both collisions,
and rows longer than a tile (the vectorised kernel runs instead)."""
import numpy as np
import pytest

from hippolbm_b200.deck import Case, Op, couette_case, sphere_channel_case

pytestmark = pytest.mark.gpu


def cases():
    out = []
    for coll in ("bgk", "mrt"):
        out.append(couette_case(64, tau=0.7, u_wall=0.05, steps=12, collision=coll))
        # an even z-plane (97 x 42) with MRT: the reference variant 4 is then the pair kernel
        c = sphere_channel_case((96, 41 if coll == "mrt" else 40, 36), (30.0, 20.0, 18.0), 5.0, tau=0.6, u_in=0.02,
                                steps=12, collision=coll)
        out.append(c)
        out.append(Case(name=f"lid_{coll}", cell_dims=(31, 29, 27), bmin=(0, 0, 0), bmax=(31, 29, 27),
                        periodic=(False, True, False), tau=0.8, nuth=0.1, collision=coll,
                        pre_stream_bcs=[Op("pre_bounce_back")], post_stream_bcs=[Op("post_bounce_back")],
                        boundary_conditions=[Op("lid_driven_cavity", {"U": [0.05, 0.0, 0.0],
                                                                      "regions": ["plan_xy_l"]}),
                                             Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_yz_0"]})],
                        steps=12))
    # rows longer than a tile of variant 8 (1024 nodes) but not of variant 9 (1536), and longer than
    # both: variant 8 (and then 9) runs the vectorised kernel instead
    out.append(Case(name="long_rows_1088", cell_dims=(1087, 5, 4), bmin=(0, 0, 0), bmax=(1087, 5, 4),
                    periodic=(True, True, False), tau=0.7, nuth=0.1, collision="bgk",
                    pre_stream_bcs=[Op("pre_bounce_back")], post_stream_bcs=[Op("post_bounce_back")],
                    boundary_conditions=[Op("lid_driven_cavity", {"U": [0.05, 0.0, 0.0], "regions": ["plan_xy_l"]})],
                    steps=12))
    out.append(Case(name="long_rows_1600", cell_dims=(1599, 3, 2), bmin=(0, 0, 0), bmax=(1599, 3, 2),
                    periodic=(True, True, True), tau=0.7, nuth=0.1, collision="mrt", steps=12))
    return out


def run(case, precision, variant, rounding):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.rounding(rounding)
        lat.tune(variant)
        lat.step(case.steps)
        info = lat.info()
        return lat.populations(), info


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("rounding", ["stochastic", "nearest"])
def test_row_pipeline_equals_pair_kernel(precision, variant, rounding):
    for case in cases():
        f_ref, _ = run(case, precision, 4, rounding)
        f, info = run(case, precision, variant, rounding)
        assert np.isfinite(f).all()
        diff = np.argwhere(f != f_ref)
        assert diff.size == 0, f"{case.name}: {len(diff)} values differ, first (dir, z, y, x) {diff[:4]}"


def test_row_pipeline_is_chosen_by_the_autotuner_or_timed():
    """On a 256^3 Couette lattice variants 8 and 9 are timed (not skipped) by hlbm_autotune."""
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(couette_case(256, tau=0.6, u_wall=0.05, steps=10), "f16") as lat:
        lat.step(2)
        chosen, ms = lat.autotune(reps=2)
        assert 8 in ms and 9 in ms and ms[8] > 0 and ms[9] > 0
