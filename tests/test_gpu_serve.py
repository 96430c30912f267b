"""Solve server: requests that arrive while others run are admitted as memory frees up, share the
batched launches, and each result equals the same solve run alone in a batch of its own -- bit for
bit in every precision (the per-node arithmetic and the rounding salt do not depend on the other
members).  Against the single-lattice kernel the FP16 result agrees to a few storage quanta (the
two kernels may contract a product differently, which can flip one rounding)."""
import numpy as np
import pytest

from hippolbm_b200 import serve

pytestmark = pytest.mark.gpu

QUANTA = {"f64_strict": 0.0, "f16": 16.0}
L2 = {"f64_strict": 0.0, "f16": 1e-3}
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def small_stream():
    reqs = serve.make_stream(rate=2e4, count=7, seed=7, edge_range=(16, 40), budget_range=(150, 450),
                             tol=1e-3, tol_fraction=0.4)
    return reqs


@pytest.mark.parametrize("precision", ["f64_strict", "f16"])
def test_each_result_is_the_same_alone_and_in_the_mix(precision):
    from hippolbm_b200.batch import Batch
    from hippolbm_b200.lattice import Lattice

    reqs = small_stream()
    # a memory budget that holds only about three solves forces queueing and later admission
    fp = sorted(serve.footprint_bytes(r.case, precision) for r in reqs)
    stats = serve.serve_batched(reqs, precision, hbm_budget=sum(fp[-3:]), chunk=50, check_every=100,
                                keep_results=True)
    assert stats["requests"] == len(reqs)
    admitted_late = [r for r in reqs if r.admitted - r.arrival > 1e-3]
    assert admitted_late, "the budget should have made some requests wait"
    for r in reqs:
        assert r.finished >= r.admitted >= r.arrival - 1e-9
        walls = any(o.name == "wall_bounce_back" for o in r.case.pre_stream_bcs)
        with Lattice.from_case(r.case, precision) as lat:
            with Batch(precision) as b:
                b.add(lat)
                b.step(r.steps)
                b.remove(lat)
            f_own = lat.populations()
            flags = lat.flags()
        m = flags != -2 if walls else np.ones_like(flags, bool)
        assert np.array_equal(r.result[:, m], f_own[:, m]), r.rid
        with Lattice.from_case(r.case, precision) as lat:
            lat.step(r.steps)
            f = lat.populations()
        # against the single-lattice kernel: a handful of storage quanta at most, and a relative
        # L2 difference of the stored deviations far below the storage precision
        dev = (f - W[:, None, None, None])[:, m]
        quantum = 2.0 ** -10 * np.abs(dev).max()
        diff = (r.result - f)[:, m]
        assert np.abs(diff).max() <= QUANTA[precision] * quantum, r.rid
        assert np.sqrt((diff ** 2).sum() / max((dev ** 2).sum(), 1e-300)) <= L2[precision], r.rid


def test_plain_path_serves_the_same_stream():
    reqs = small_stream()
    stats = serve.serve_plain(reqs, "f64", chunk=50, check_every=100)
    assert stats["requests"] == len(reqs) and stats["p99_s"] >= stats["p50_s"] > 0
