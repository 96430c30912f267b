"""The span pipeline of the 16-bit tiers (variants 8 and 9 on lattices whose rows are not whole
16-byte chunks: tiles are spans of the linear node index, bulk-copied per direction) gives the same
populations as the pair kernel (variant 4), bit for bit, with stochastic rounding and with
rounding to nearest.  The cases cover odd row lengths (groups of four nodes across row ends and
node pairs across rows and planes), rows of 4 to 7 nodes, a node count that is no multiple of four
(the last group is partial), a lattice smaller than one tile, periodic wrap on every axis (face
nodes gather from global memory), non-periodic faces left to the face pass, boundary operators,
wall obstacles (the wall fix-up), both collisions, and the serving mix's cavity, channel and
sphere solves.

Variant 4 runs the pair kernel on lattices with even z-planes and the one-node kernel on odd ones.
The MRT cases use even planes: there the node-pair form and the one-node form of the FP32 MRT can
differ by one ulp in rare values (the code generator evaluates one product of the packed form in
a different order), which stochastic rounding then carries into the stored state; every node-pair
kernel (pair, row and span pipelines) agrees with every other bit for bit."""
import numpy as np
import pytest

from hippolbm_b200.deck import Case, Op
from hippolbm_b200.serve import solve_case

pytestmark = pytest.mark.gpu


def cases():
    out = []
    for coll, ny in (("bgk", 23), ("mrt", 24)):  # odd z-planes with BGK, even ones with MRT
        # every axis periodic: no face pass, every face node wraps through the global gather
        d = (36, ny - 1, 18)
        out.append(Case(name=f"periodic_37x{ny}x19_{coll}", cell_dims=d, bmin=(0, 0, 0), bmax=d,
                        periodic=(True, True, True), tau=0.7, nuth=0.2 / 3, collision=coll,
                        obstacles=[("ball", 0, ((18.0, 11.0, 9.0), 4.0))],
                        pre_stream_bcs=[Op("wall_bounce_back")], steps=12))
        # Couette with odd rows: x, y wrap; z faces in the face pass (moving wall)
        d = (44, ny + 7, 25)
        out.append(Case(name=f"couette_45x{ny + 8}x26_{coll}", cell_dims=d, bmin=(0, 0, 0), bmax=d,
                        periodic=(True, True, False), tau=0.6, nuth=0.1 / 3, collision=coll,
                        pre_stream_bcs=[Op("pre_bounce_back"), Op("cavity_z_l", {"U": [0.05, 0.0, 0.0]})],
                        post_stream_bcs=[Op("post_bounce_back")], steps=12))
    # rows of 5 nodes: most groups of four cross a row end; x periodic, y / z bounced
    out.append(Case(name="rows5", cell_dims=(4, 9, 7), bmin=(0, 0, 0), bmax=(4, 9, 7), periodic=(True, False, False),
                    tau=0.8, nuth=0.1, collision="bgk", pre_stream_bcs=[Op("pre_bounce_back")],
                    post_stream_bcs=[Op("post_bounce_back")], steps=12))
    # rows of 7 nodes, y periodic, x / z bounced with a lid and a Zou/He plane; 7 x 6 x 5 = 210 nodes
    # (one partial tile; 210 is no multiple of four)
    out.append(Case(name="rows7_lid", cell_dims=(6, 5, 4), bmin=(0, 0, 0), bmax=(6, 5, 4), periodic=(False, True, False),
                    tau=0.75, nuth=0.25 / 3, collision="mrt", pre_stream_bcs=[Op("pre_bounce_back")],
                    post_stream_bcs=[Op("post_bounce_back")],
                    boundary_conditions=[Op("lid_driven_cavity", {"U": [0.05, 0.0, 0.0], "regions": ["plan_xy_l"]}),
                                         Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_yz_0"]})],
                    steps=12))
    # x periodic with rows of 24 (8-element but not 16-element rows) and a sphere near the y faces
    out.append(Case(name="rows24_sphere", cell_dims=(23, 40, 33), bmin=(0, 0, 0), bmax=(23, 40, 33),
                    periodic=(True, False, False), tau=0.65, nuth=0.05, collision="bgk",
                    obstacles=[("ball", 0, ((12.0, 3.0, 16.0), 5.0))],
                    pre_stream_bcs=[Op("pre_bounce_back"), Op("wall_bounce_back")],
                    post_stream_bcs=[Op("post_bounce_back")], steps=12))
    # the serving mix: every face non-periodic
    rng = np.random.default_rng(7)
    for kind, edges in (("cavity", (57, 43, 61)), ("channel", (70, 35, 29)), ("sphere", (83, 47, 39))):
        c = solve_case(kind, edges, 0.6, rng)
        c.steps = 12
        out.append(c)
    return out


def run(case, precision, variant, rounding):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.rounding(rounding)
        lat.tune(variant)
        lat.step(case.steps)
        return lat.populations()


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("rounding", ["stochastic", "nearest"])
def test_span_pipeline_equals_pair_kernel(precision, variant, rounding):
    for case in cases():
        f_ref = run(case, precision, 4, rounding)
        f = run(case, precision, variant, rounding)
        assert np.isfinite(f).all()
        diff = np.argwhere(f != f_ref)
        assert diff.size == 0, f"{case.name}: {len(diff)} values differ, first (dir, z, y, x) {diff[:4]}"


def test_span_pipeline_serving_lattice_in_a_concurrent_batch():
    """A serving lattice stepped by the span pipeline alone equals the same lattice stepped inside a
    concurrent batch (variant 10: members' own kernels forked from one captured graph)."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    rng = np.random.default_rng(11)
    cs = [solve_case("sphere", (45, 38, 29), 0.7, rng), solve_case("cavity", (33, 27, 50), 0.9, rng)]
    alone = []
    for c in cs:
        with Lattice.from_case(c, "f16") as lat:
            lat.tune(9)
            lat.step(20)
            alone.append(lat.populations())
    lats = [Lattice.from_case(c, "f16").tune(9) for c in cs]
    try:
        with Batch("f16") as b:
            b.tune(10)
            for lat in lats:
                b.add(lat)
            b.step(20)
            got = [lat.populations() for lat in lats]
            for lat in lats:
                b.remove(lat)
        for f, ref in zip(got, alone):
            assert np.array_equal(f, ref)
    finally:
        for lat in lats:
            lat.close()
