"""The bounded waits of the pipelined kernel (variants 6 and 7) report a timeout instead of hanging.

hlbm_set_wait_limit bounds each barrier wait of the kernel to a number of polls.  With one poll the
consumer warps give up on their first stage before its bulk copies land (they take microseconds;
a poll takes nanoseconds): the kernel records the timeout in the context's device error word, its
producer waits (with the default bound) for the copies it has in flight, and every CTA returns.
No wait is made endless and nothing traps: the error reaches the host through the next read-out,
which fails with HLBM_ECUDA and clears the word, and the context then steps on normally.
"""
import numpy as np
import pytest

from hippolbm_b200 import capi
from hippolbm_b200.deck import couette_case

pytestmark = pytest.mark.gpu


def test_wait_timeout_reaches_the_host_and_the_context_recovers():
    from hippolbm_b200.lattice import Lattice

    case = couette_case(48, tau=0.8, u_wall=0.05, steps=6)
    with Lattice.from_case(case, "f32") as ref:
        ref.tune(6)
        ref.step(3)
        f0 = ref.populations()
        ref.step(3)
        f_expected = ref.populations()
    with Lattice.from_case(case, "f32") as lat:
        lat.tune(6)
        capi.check(lat.L.hlbm_set_wait_limit(lat.h, 1))
        lat.step(3)  # the prologue, then two fused launches of the pipelined kernel
        with pytest.raises(capi.HlbmError) as e:
            lat.populations()
        assert e.value.code == -3 and "timed out" in str(e.value)  # HLBM_ECUDA
        capi.check(lat.L.hlbm_set_wait_limit(lat.h, 0))  # the default bound again
        lat.put_populations(f0)
        lat.step(3)
        f = lat.populations()
    assert np.array_equal(f, f_expected)


def test_wait_limit_rejects_negative_bounds():
    from hippolbm_b200.lattice import Lattice

    with Lattice((8, 8, 8), (0, 0, 0), (8, 8, 8), (True, True, True), "f32") as lat:
        assert lat.L.hlbm_set_wait_limit(lat.h, -1) == -1
        assert lat.L.hlbm_set_wait_limit(lat.h, 0) == 0
