"""Batches: one persistent-kernel launch per step over many lattices of different sizes, plans,
collisions and boundary operators gives each member the populations it gets when stepped alone
(same pipelined kernel): bit for bit in strict FP64, 1e-6 of the largest population in FP32."""
import numpy as np
import pytest

from hippolbm_b200.deck import Case, Op

pytestmark = pytest.mark.gpu


def member(i, nx, ny, nz, kind, collision, tau):
    per = (True, True, False) if kind != "cavity" else (False, False, False)
    c = Case(name=f"m{i}", cell_dims=(nx - 1, ny - 1, nz - 1), bmin=(0, 0, 0), bmax=(nx - 1, ny - 1, nz - 1),
             periodic=per, tau=tau, nuth=(tau - 0.5) / 3, collision=collision, steps=30)
    if kind == "couette":
        c.pre_stream_bcs = [Op("pre_bounce_back"), Op("cavity_z_l", {"U": [0.03 + 0.01 * i, 0.0, 0.0]})]
        c.post_stream_bcs = [Op("post_bounce_back")]
    elif kind == "poiseuille":
        c.Fext = (1e-5 * (1 + i), 0.0, 0.0)
        c.boundary_conditions = [Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_xy_0", "plan_xy_l"]})]
    else:
        c.pre_stream_bcs = [Op("pre_bounce_back"), Op("wall_bounce_back")]
        c.post_stream_bcs = [Op("post_bounce_back"),
                             Op("lid_driven_cavity", {"U": [0.05, 0.0, 0.0], "regions": ["plan_xy_l"]})]
        c.obstacles = [("ball", 0, ((nx / 2, ny / 2, nz / 3), min(nx, ny, nz) / 5))]
    return c


CASES = [member(0, 32, 40, 24, "couette", "bgk", 0.7), member(1, 48, 16, 32, "poiseuille", "mrt", 0.9),
         member(2, 40, 40, 40, "cavity", "bgk", 0.6), member(3, 64, 24, 16, "couette", "mrt", 1.1),
         member(4, 32, 32, 56, "cavity", "mrt", 0.8)]
RTOL = {"f64_strict": 0.0, "f32": 1e-6}


def alone(case, precision, steps):
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(case, precision) as lat:
        lat.tune(6)
        lat.step(steps)
        return lat.populations(), lat.flags()


def carried(case, flags):
    return flags != -2 if any(o.name == "wall_bounce_back" for o in case.pre_stream_bcs) else np.ones_like(flags, bool)


@pytest.mark.parametrize("precision", ["f64_strict", "f32"])
@pytest.mark.parametrize("variant", [8, 9, 6, 10])
def test_batch_members_equal_their_runs_alone(precision, variant):
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    lats = [Lattice.from_case(c, precision) for c in CASES]
    with Batch(precision) as b:
        b.tune(variant)
        for lat in lats:
            b.add(lat)
        b.step(7)   # fresh members take their first step inside the batch launch; odd count
        b.step(16)  # graph replays
        b.step(1)
        info = b.info()
        assert info["members"] == len(CASES) and info["graph_replays"] >= 8
        for case, lat in zip(CASES, lats):
            assert lat.info()["steps"] == 24
            f_ref, flags = alone(case, precision, 24)
            f = lat.populations()
            m = carried(case, flags)
            tol = RTOL[precision] * np.abs(f_ref).max()
            assert np.abs(f - f_ref)[:, m].max() <= tol, case.name
    for lat in lats:
        lat.close()


def test_batch_admits_and_releases_between_steps():
    """Continuous batching: a member joins after others have stepped and one leaves early; each
    ends with the populations of its own step count."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    a, b2, c = (Lattice.from_case(CASES[i], "f64_strict") for i in (0, 1, 2))
    with Batch("f64_strict") as b:
        b.add(a).add(b2)
        b.step(5)
        b.add(c)           # joins with 0 steps
        b.step(6)
        b.remove(b2)       # leaves with 11 steps
        b.step(3)
    for lat, case, n in ((a, CASES[0], 14), (b2, CASES[1], 11), (c, CASES[2], 9)):
        assert lat.info()["steps"] == n
        f_ref, flags = alone(case, "f64_strict", n)
        m = carried(case, flags)
        assert np.array_equal(lat.populations()[:, m], f_ref[:, m]), case.name
        lat.close()


def test_batch_any_row_length_and_pipelined_rejects_unaligned():
    """The tile-list kernel takes any nx; the pipelined one needs 16-byte rows."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200 import capi
    from hippolbm_b200.lattice import Lattice

    case = member(9, 30, 8, 8, "couette", "bgk", 0.7)  # 30 x 2 bytes is not a multiple of 16
    f_ref, _ = alone(case, "f64_strict", 9)
    with Batch("f64_strict") as b, Lattice.from_case(case, "f64_strict") as lat:
        b.add(lat)
        b.step(9)
        assert np.array_equal(lat.populations(), f_ref)
    with Batch("f16") as b, Lattice.from_case(case, "f16") as lat:
        b.tune(6)
        with pytest.raises(capi.HlbmError):
            b.add(lat)


@pytest.mark.parametrize("variant", [8, 6])
def test_f16_members_equal_their_batch_of_one(variant):
    """16-bit storage with stochastic rounding: the random bits hash each member's own node index
    and step count, so a member's populations in the mixed batch equal those of the same lattice in
    a batch of its own, bit for bit, whatever joins or leaves around it."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    lats = [Lattice.from_case(c, "f16") for c in CASES]
    with Batch("f16") as b:
        b.tune(variant)
        for lat in lats[:3]:
            b.add(lat)
        b.step(5)
        for lat in lats[3:]:
            b.add(lat)     # join with 0 steps while the others are at 5
        b.step(12)
        out = [(lat.info()["steps"], lat.populations()) for lat in lats]
        for lat in lats:
            b.remove(lat)
    for case, lat, (n, f) in zip(CASES, lats, out):
        lat.close()
        with Lattice.from_case(case, "f16") as one:
            with Batch("f16") as b1:
                b1.tune(variant)
                b1.add(one)
                b1.step(n)
                b1.remove(one)
            f1 = one.populations()
            m = carried(case, one.flags())
        assert np.array_equal(f[:, m], f1[:, m]), case.name


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_concurrent_members_equal_their_runs_alone(precision):
    """Variant 10 steps every member with its own single-lattice kernel, forked onto the members'
    streams inside one captured graph; graph-replayed launches read the stochastic-rounding step
    number from a device counter.  Each member ends bit for bit where it ends stepped alone, through
    joins, an odd step count and a rounding-mode change that forces a new capture."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    lats = [Lattice.from_case(c, precision) for c in CASES]
    with Batch(precision) as b:
        b.tune(10)
        for lat in lats[:3]:
            b.add(lat)
        b.step(5)
        for lat in lats[3:]:
            b.add(lat)
        b.step(12)
        lats[1].rounding("nearest")
        b.step(4)
        assert b.info()["graph_replays"] >= 8
        out = [(lat.info()["steps"], lat.populations()) for lat in lats]
        for lat in lats:
            b.remove(lat)
    for i, (case, lat, (n, f)) in enumerate(zip(CASES, lats, out)):
        lat.close()
        with Lattice.from_case(case, precision) as one:
            if i == 1:
                one.step(17)
                one.rounding("nearest")
                one.step(n - 17)
            else:
                one.step(n)
            f1 = one.populations()
            m = carried(case, one.flags())
        assert np.array_equal(f[:, m], f1[:, m]), case.name


@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_batch_autotune_leaves_every_member_unchanged(precision):
    """hlbm_batch_autotune times every batch kernel on the batch and keeps the fastest: no member's
    state moves (also for members that have not stepped yet), and the batch then steps like a batch
    tuned to that kernel by hand."""
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    lats = [Lattice.from_case(c, precision) for c in CASES]
    with Batch(precision) as b:
        for lat in lats:
            b.add(lat)
        b.step(3)
        before = [lat.populations() for lat in lats]
        fresh = Lattice.from_case(CASES[0], precision)  # joins now: it has not stepped yet
        b.add(fresh)
        fresh_before = fresh.populations()
        chosen, ms = b.autotune(reps=2)
        assert chosen in ms and set(ms) <= {6, 7, 8, 9, 10} and {8, 9, 10} <= set(ms)
        assert all(t > 0 for t in ms.values())
        for lat, f in zip(lats, before):
            assert np.array_equal(lat.populations(), f)
        assert np.array_equal(fresh.populations(), fresh_before)
        b.step(4)
        got = [lat.populations() for lat in lats + [fresh]]
    ref_lats = [Lattice.from_case(c, precision) for c in CASES]
    with Batch(precision) as r:  # the same calls with the chosen kernel set by hand
        for lat in ref_lats:
            r.add(lat)
        r.step(3)
        ref_fresh = Lattice.from_case(CASES[0], precision)
        r.add(ref_fresh)
        r.tune(chosen)
        r.step(4)
        want = [lat.populations() for lat in ref_lats + [ref_fresh]]
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    for lat in lats + [fresh] + ref_lats + [ref_fresh]:
        lat.close()
