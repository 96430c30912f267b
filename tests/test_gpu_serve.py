"""Solve server: requests that arrive while others run are admitted as memory frees up, share the
batched launches, and each result equals the same solve run alone -- exactly in strict FP64,
within 1e-4 of the largest population with FP16 storage (a few storage quanta: the batched and the
single-lattice kernels may round a product differently, which can flip one FP16 rounding)."""
import numpy as np
import pytest

from hippolbm_b200 import serve

pytestmark = pytest.mark.gpu

TOL = {"f64_strict": 0.0, "f16": 1e-4}


def small_stream():
    reqs = serve.make_stream(rate=200.0, count=7, seed=7, edge_range=(16, 40), budget_range=(150, 450),
                             tol=1e-3, tol_fraction=0.4)
    return reqs


@pytest.mark.parametrize("precision", ["f64_strict", "f16"])
def test_each_result_is_the_same_alone_and_in_the_mix(precision):
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
        with Lattice.from_case(r.case, precision) as lat:
            lat.step(r.steps)
            f = lat.populations()
        walls = any(o.name == "wall_bounce_back" for o in r.case.pre_stream_bcs)
        m = lat_flags = None
        with Lattice.from_case(r.case, precision) as l2:
            lat_flags = l2.flags()
        m = lat_flags != -2 if walls else np.ones_like(lat_flags, bool)
        err = np.abs(r.result - f)[:, m].max()
        assert err <= TOL[precision] * np.abs(f).max(), (r.rid, err)


def test_plain_path_serves_the_same_stream():
    reqs = small_stream()
    stats = serve.serve_plain(reqs, "f64", chunk=50, check_every=100)
    assert stats["requests"] == len(reqs) and stats["p99_s"] >= stats["p50_s"] > 0
