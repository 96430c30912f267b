"""hlbm_simulation_state_static: the statistics entry point that allocates nothing.

It exists for callers that cannot allocate device memory when they need the statistics -- an
analysis hook inside a host application that owns the whole device budget, or a loop that must
not pay cudaMalloc's device-wide synchronisation.  The caller hands it device pointers to the
populations, the flags and a 3-double output; its partial sums live in a static __device__
array.  This file is collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from hippolbm_b200 import capi
from hippolbm_b200.deck import Case, Op


def lid_case():
    return Case(name="noalloc", cell_dims=(23, 17, 13), bmin=(0, 0, 0), bmax=(23, 17, 13),
                periodic=(True, False, False), tau=0.7, nuth=0.2 / 3,
                obstacles=[("ball", 0, ((12.0, 8.0, 6.0), 3.0))],
                pre_stream_bcs=[Op("pre_bounce_back"), Op("wall_bounce_back")],
                post_stream_bcs=[Op("post_bounce_back"),
                                 Op("lid_driven_cavity", {"U": [0.08, 0.0, 0.0], "regions": ["plan_xy_l"]})],
                steps=10)


def static_stats(f_dev, flags_dev, n, out_dev, stream_ptr):
    L = capi.lib()
    rc = L.hlbm_simulation_state_static(C.cast(f_dev.data_ptr(), C.POINTER(C.c_double)), f_dev.numel() // 19,
                                        C.cast(flags_dev.data_ptr(), C.POINTER(C.c_int8)), capi.ivec(n),
                                        C.cast(out_dev.data_ptr(), C.POINTER(C.c_double)), stream_ptr)
    capi.check(rc)


@pytest.mark.gpu
def test_static_stats_match_the_allocating_entry_point_twice():
    import torch

    from hippolbm_b200.lattice import Lattice

    case = lid_case()
    n = [c + 1 for c in case.cell_dims]
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with Lattice.from_case(case, "f64") as lat:
        for steps in (10, 25):  # two calls in a row, on two different states
            lat.step(steps)
            expected = lat.simulation_state()  # existing entry point (allocated scratch)
            f_dev = torch.from_numpy(lat.populations().reshape(-1)).cuda()
            flags_dev = torch.from_numpy(lat.flags().reshape(-1)).cuda()
            out.fill_(-1.0)
            torch.cuda.synchronize()
            static_stats(f_dev, flags_dev, n, out, C.c_void_p(stream.cuda_stream))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert got[0] == pytest.approx(expected[0], rel=1e-13)  # summation order differs
            assert got[1] == expected[1] and got[2] == expected[2]   # same per-node arithmetic
            assert np.isfinite(got).all() and got[2] > 0.0


@pytest.mark.gpu
def test_static_stats_many_blocks_and_padded_stride():
    """41^3 = 68,921 nodes (5 partial slots, the last one partial, so the fixed-order fold runs over
    several blocks) with the planes 7 elements apart beyond the node count, twice in a row."""
    import torch

    from hippolbm_b200.lattice import Lattice

    case = Case(name="noalloc41", cell_dims=(40, 40, 40), bmin=(0, 0, 0), bmax=(40, 40, 40),
                periodic=(True, True, False), tau=0.8, nuth=0.1,
                obstacles=[("ball", 0, ((20.0, 20.0, 20.0), 6.0))],
                pre_stream_bcs=[Op("pre_bounce_back"), Op("cavity_z_l", {"U": [0.05, 0.0, 0.0]}),
                                Op("wall_bounce_back")],
                post_stream_bcs=[Op("post_bounce_back")], steps=10)
    n = [41, 41, 41]
    ncell = 41 ** 3
    stride = ncell + 7
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with Lattice.from_case(case, "f64") as lat:
        for steps in (10, 15):
            lat.step(steps)
            expected = lat.simulation_state()
            f = torch.from_numpy(lat.populations().reshape(19, ncell))
            f_dev = torch.full((19, stride), float("nan"), dtype=torch.float64, device="cuda")
            f_dev[:, :ncell] = f.cuda()
            flags_dev = torch.from_numpy(lat.flags().reshape(-1)).cuda()
            out.fill_(-1.0)
            torch.cuda.synchronize()
            L = capi.lib()
            capi.check(L.hlbm_simulation_state_static(C.cast(f_dev.data_ptr(), C.POINTER(C.c_double)), stride,
                                                      C.cast(flags_dev.data_ptr(), C.POINTER(C.c_int8)),
                                                      capi.ivec(n), C.cast(out.data_ptr(), C.POINTER(C.c_double)),
                                                      C.c_void_p(stream.cuda_stream)))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert got[0] == pytest.approx(expected[0], rel=1e-13)
            assert got[1] == expected[1] and got[2] == expected[2]


def test_static_stats_reject_lattices_beyond_the_scratch_limit():
    L = capi.lib()
    dummy = (C.c_double * 3)()
    flags = (C.c_int8 * 1)()
    rc = L.hlbm_simulation_state_static(dummy, 1 << 40, flags, capi.ivec([16384, 16384, 2]), dummy, None)
    assert rc == -1
    assert b"static scratch limit" in L.hlbm_last_error()
