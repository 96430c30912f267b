"""Python driver for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads either the C restatement (oracle/_build/libhlbm_oracle.so, kind "port") or the
reference functor harness (oracle/_ref/libhlbm_ref.so, kind "reference") and runs a
`hippolbm_b200.deck.Case` through the reference's compute-loop order
(config_compute_loop.msp:27-37):

    start_iteration -> macro_variables -> collision -> pre_stream_bcs -> streaming
    -> post_stream_bcs -> boundary_conditions

after the initialize sequence of config_initialize.msp:14-32.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "port": os.path.join(HERE, "_build", "libhlbm_oracle.so"),
    "reference": os.path.join(HERE, "_ref", "libhlbm_ref.so"),
}
Q = 19
_FACE_OF_PLANE = {"plan_yz_0": 0, "plan_yz_l": 1, "plan_xz_0": 2, "plan_xz_l": 3, "plan_xy_0": 4, "plan_xy_l": 5}


def build(kind: str = "port") -> None:
    target = {"port": "oracle", "reference": "ref"}[kind]
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind])


_loaded: dict = {}


def _lib(kind: str):
    if kind in _loaded:
        return _loaded[kind]
    path = LIBS[kind]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    lib = C.CDLL(path)
    d3, i3 = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    vp = C.c_void_p
    sig = {
        "orc_create": (vp, [i3, d3, d3, i3, i3]),
        "orc_destroy": (None, [vp]),
        "orc_lbm_parameters": (None, [vp, d3, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_double]),
        "orc_get_parameters": (None, [vp, d3]),
        "orc_set_distribution": (None, [vp, C.c_double, d3, C.c_int32]),
        "orc_init_obstacles": (None, [vp]),
        "orc_register_ball": (None, [vp, C.c_int32, d3, C.c_double]),
        "orc_register_wall": (None, [vp, C.c_int32, d3, d3]),
        "orc_register_quadric": (None, [vp, C.c_int32, d3]),
        "orc_update_obstacles": (None, [vp]),
        "orc_macro_variables": (None, [vp]),
        "orc_bgk": (None, [vp]),
        "orc_mrt": (None, [vp, d3]),
        "orc_pre_bounce_back": (None, [vp]),
        "orc_post_bounce_back": (None, [vp]),
        "orc_cavity": (None, [vp, C.c_int32, d3]),
        "orc_wall_bounce_back": (None, [vp]),
        "orc_streaming": (None, [vp]),
        "orc_update_ghost": (None, [vp]),
        "orc_neumann": (C.c_int32, [vp, C.c_int32, d3]),
        "orc_lid_driven_cavity": (C.c_int32, [vp, C.c_int32, d3]),
        "orc_simulation_state": (None, [vp, d3]),
        "orc_snapshot_streamed": (None, [vp]),
        "orc_zero_gradient": (C.c_int32, [vp, C.c_int32]),
        "orc_init_double_couette": (None, [vp, d3, C.c_int32]),
        "orc_plane_velocity_profile": (None, [vp, C.c_int32, d3, d3, d3, C.POINTER(C.c_int64)]),
        "orc_info": (None, [vp, C.POINTER(C.c_int64)]),
        "orc_f": (d3, [vp]),
        "orc_m0": (d3, [vp]),
        "orc_m1": (d3, [vp]),
        "orc_obst": (i3, [vp]),
        "orc_level": (i3, [vp]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(lib, name):  # operators the reference does not have
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _loaded[kind] = lib
    return lib


def _d(v):
    a = (C.c_double * len(v))(*[float(x) for x in v])
    return a


class OracleLattice:
    """One lattice on the CPU oracle, in the reference's ghosted layout."""

    def __init__(self, case, kind: str = "port"):
        self.kind = kind
        self.lib = _lib(kind)
        self.case = case
        err = C.c_int32(0)
        dims = (C.c_int32 * 3)(*case.cell_dims)
        per = (C.c_int32 * 3)(*[1 if p else 0 for p in case.periodic])
        h = self.lib.orc_create(dims, _d(case.bmin), _d(case.bmax), per, C.byref(err))
        if not h:
            raise ValueError(f"orc_create failed ({err.value})")
        self.h = C.c_void_p(h)
        info = (C.c_int64 * 13)()
        self.lib.orc_info(self.h, info)
        self.L = tuple(info[0:3])
        self.n = tuple(info[3:6])
        self.ncell = int(info[6])

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- views
    def f(self) -> np.ndarray:
        """(19, Lz, Ly, Lx) view of the populations (ghost layers included)."""
        p = self.lib.orc_f(self.h)
        a = np.ctypeslib.as_array(p, shape=(Q * self.ncell,))
        return a.reshape(Q, self.L[2], self.L[1], self.L[0])

    def obst(self) -> np.ndarray:
        p = self.lib.orc_obst(self.h)
        return np.ctypeslib.as_array(p, shape=(self.ncell,)).reshape(self.L[2], self.L[1], self.L[0])

    def m0(self) -> np.ndarray:
        p = self.lib.orc_m0(self.h)
        return np.ctypeslib.as_array(p, shape=(self.ncell,)).reshape(self.L[2], self.L[1], self.L[0])

    def m1(self) -> np.ndarray:
        p = self.lib.orc_m1(self.h)
        return np.ctypeslib.as_array(p, shape=(3 * self.ncell,)).reshape(3, self.L[2], self.L[1], self.L[0])

    def real(self, a: np.ndarray) -> np.ndarray:
        """Real-box slice (ghost layers dropped) of a (..., Lz, Ly, Lx) array: (..., nz, ny, nx)."""
        return a[..., 2:self.L[2] - 2, 2:self.L[1] - 2, 2:self.L[0] - 2]

    def parameters(self) -> dict:
        out = (C.c_double * 9)()
        self.lib.orc_get_parameters(self.h, out)
        o = list(out)
        return {"Fext": tuple(o[0:3]), "celerity": o[3], "dtLB": o[4], "nuth": o[5], "nu": o[6], "tau": o[7],
                "avg_rho": o[8]}

    def simulation_state(self) -> tuple:
        out = (C.c_double * 3)()
        self.lib.orc_simulation_state(self.h, out)
        return tuple(out)

    def plane_velocity_profile(self, dimension: str = "Z"):
        """(mean, min, max, count) per plane of the current state (macro_variables refreshed)."""
        if not hasattr(self.lib, "orc_plane_velocity_profile"):
            raise ValueError("plane_velocity_profile is restated by the C oracle only")
        dim = {"X": 0, "Y": 1, "Z": 2}[dimension.upper()]
        n = self.n[dim]
        avg, vmin, vmax = np.empty(n), np.empty(n), np.empty(n)
        cnt = np.empty(n, dtype=np.int64)
        self.lib.orc_macro_variables(self.h)
        dp = C.POINTER(C.c_double)
        self.lib.orc_plane_velocity_profile(self.h, dim, avg.ctypes.data_as(dp), vmin.ctypes.data_as(dp),
                                            vmax.ctypes.data_as(dp), cnt.ctypes.data_as(C.POINTER(C.c_int64)))
        return avg, vmin, vmax, cnt

    # ----------------------------------------------------------- initialise
    def initialize(self):
        """config_initialize.msp:14-32 after domain/build_traversal/define_grid/init_obst."""
        c = self.case
        lib = self.lib
        lib.orc_lbm_parameters(self.h, _d(c.Fext), c.celerity, c.nuth, c.avg_rho, 1 if c.tau is not None else 0,
                               c.tau if c.tau is not None else 0.0, c.dt)
        for value, bounds6 in c.init_distributions:
            lib.orc_set_distribution(self.h, value, _d(bounds6) if bounds6 else None, 0)
        if getattr(c, "double_couette", None):
            lib.orc_init_double_couette(self.h, _d(c.double_couette["U"]), "XYZ".index(c.double_couette["dimension"]))
        lib.orc_init_obstacles(self.h)
        for kind, oid, prm in c.obstacles:
            if kind == "ball":
                lib.orc_register_ball(self.h, oid, _d(prm[0]), prm[1])
            elif kind == "wall":
                lib.orc_register_wall(self.h, oid, _d(prm[0]), _d(prm[1]))
            else:
                lib.orc_register_quadric(self.h, oid, _d(prm))
        lib.orc_update_obstacles(self.h)
        lib.orc_macro_variables(self.h)
        return self

    # ------------------------------------------------------------------ ops
    def _op(self, op):
        lib, h, s = self.lib, self.h, op.slots
        if op.name == "pre_bounce_back":
            lib.orc_pre_bounce_back(h)
        elif op.name == "post_bounce_back":
            lib.orc_post_bounce_back(h)
        elif op.name in ("cavity_z_0", "cavity_z_l"):
            lib.orc_cavity(h, 1 if op.name.endswith("_l") else 0, _d(s["U"]))
        elif op.name == "wall_bounce_back":
            lib.orc_wall_bounce_back(h)
        elif op.name == "neumann":
            for r in s["regions"]:
                lib.orc_neumann(h, _FACE_OF_PLANE[r], _d(s["U"]))
        elif op.name == "lid_driven_cavity":
            for r in s["regions"]:
                lib.orc_lid_driven_cavity(h, _FACE_OF_PLANE[r], _d(s["U"]))
        elif op.name == "zero_gradient":
            if not hasattr(lib, "orc_zero_gradient"):
                raise ValueError("zero_gradient has no reference counterpart")
            for r in s["regions"]:
                lib.orc_zero_gradient(h, _FACE_OF_PLANE[r])
        elif op.name == "set_distribution":
            b = s.get("bounds")
            b6 = None
            if b is not None:
                b6 = tuple(b[0]) + tuple(b[1]) if len(b) == 2 else tuple(b)
            lib.orc_set_distribution(h, float(s.get("value", 1.0)), _d(b6) if b6 else None,
                                     1 if s.get("do_update") else 0)
        else:
            raise ValueError(f"oracle: unknown operator {op.name}")

    def step(self, nsteps: int = 1):
        c = self.case
        rates = _d(c.mrt_rates) if (c.collision == "mrt" and c.mrt_rates is not None) else None
        for _ in range(nsteps):
            for op in c.start_iteration:
                self._op(op)
            self.lib.orc_macro_variables(self.h)
            if c.collision == "bgk":
                self.lib.orc_bgk(self.h)
            else:
                self.lib.orc_mrt(self.h, rates)
            for op in c.pre_stream_bcs:
                self._op(op)
            self.lib.orc_streaming(self.h)
            if any(op.name == "zero_gradient" for op in c.post_stream_bcs + c.boundary_conditions):
                self.lib.orc_snapshot_streamed(self.h)
            for op in c.post_stream_bcs:
                self._op(op)
            for op in c.boundary_conditions:
                self._op(op)
        return self


def run_case(case, steps: int | None = None, kind: str = "port") -> OracleLattice:
    lat = OracleLattice(case, kind).initialize()
    lat.step(case.steps if steps is None else steps)
    return lat
