"""Admission policies of the solve server (host logic only, no GPU)."""
import numpy as np
import pytest

from hippolbm_b200 import serve


def req(rid, edges, budget, arrival=0.0):
    case = serve.solve_case("cavity", edges, 0.7, np.random.default_rng(rid))
    return serve.Request(rid, arrival, case, budget)


def test_fifo_blocks_behind_a_request_that_does_not_fit():
    a, b, c = req(0, (32, 32, 32), 100), req(1, (96, 96, 96), 100), req(2, (24, 24, 24), 100)
    budget = serve.footprint_bytes(a.case, "f16") + serve.footprint_bytes(c.case, "f16") + 1
    got = serve.admit([a, b, c], [], 0, "f16", budget, "fifo")
    assert [r.rid for r in got] == [0]


def test_sjf_takes_smallest_work_first_and_skips_what_does_not_fit():
    a, b, c = req(0, (32, 32, 32), 1000), req(1, (96, 96, 96), 100), req(2, (24, 24, 24), 100)
    budget = serve.footprint_bytes(a.case, "f16") + serve.footprint_bytes(c.case, "f16") + 1
    got = serve.admit([a, b, c], [], 0, "f16", budget, "sjf")
    assert [r.rid for r in got] == [2, 0]


def test_active_node_cap_and_lone_request():
    small = [req(i, (24, 24, 24), 100) for i in range(4)]
    big = req(9, (128, 128, 128), 100)
    cap = 2 * small[0].nodes
    got = serve.admit(small, [], 0, "f16", 1e12, "sjf", max_active_nodes=cap)
    assert len(got) == 2
    # a request larger than the cap is admitted when nothing else runs, and blocks nothing
    assert serve.admit([big], [], 0, "f16", 1e12, "sjf", max_active_nodes=cap) == [big]
    assert serve.admit([big], [small[0]], 0, "f16", 1e12, "sjf", max_active_nodes=small[0].nodes) == []
    # memory: a lone request is admitted even beyond the budget
    assert serve.admit([big], [], 0, "f16", 1.0, "fifo") == [big]


def test_unknown_policy_is_rejected():
    with pytest.raises(ValueError):
        serve.admit([], [], 0, "f16", 1e12, "lifo")
