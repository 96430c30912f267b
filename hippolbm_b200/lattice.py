"""One lattice on one GPU, driven through the C-ABI in the reference's operator order.

`Lattice.from_case(case)` runs the `initialize` list of config_initialize.msp:14-32 (domain,
lbm_parameters, default and user set_distribution, obstacles, update_obstacles) and records
the compute-loop hook operators; `step(n)` then runs n iterations of compute_loop
(config_compute_loop.msp:27-37) as fused kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .deck import PLANE_INDEX, Case, lbm_parameters

Q = 19


class Lattice:
    def __init__(self, cell_dims, bmin, bmax, periodic, precision: str = "f64", device: int = 0):
        L = capi.lib()
        h = C.c_void_p()
        capi.check(L.hlbm_domain(capi.ivec(cell_dims), capi.dvec(bmin), capi.dvec(bmax),
                                 capi.ivec([1 if p else 0 for p in periodic]), capi.PRECISIONS[precision], device,
                                 C.byref(h)))
        self.h = h
        self.L = L
        self.precision = precision
        self.n = tuple(int(c) + 1 for c in cell_dims)
        self.ncell = self.n[0] * self.n[1] * self.n[2]

    # ----------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.hlbm_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ initialise
    @classmethod
    def from_case(cls, case: Case, precision: str = "f64", device: int = 0) -> "Lattice":
        case.validate()
        lat = cls(case.cell_dims, case.bmin, case.bmax, case.periodic, precision, device)
        lat.apply_case(case)
        return lat

    def apply_case(self, case: Case):
        L, h = self.L, self.h
        lbm_parameters(case)  # validates tau > 0.5 in the reference's arithmetic
        capi.check(L.hlbm_lbm_parameters(h, capi.dvec(case.Fext), case.celerity, case.nuth, case.avg_rho,
                                         1 if case.tau is not None else 0,
                                         case.tau if case.tau is not None else 0.0, case.dt))
        rates = capi.dvec(case.mrt_rates) if case.mrt_rates is not None else None
        capi.check(L.hlbm_collision(h, 0 if case.collision == "bgk" else 1, rates))
        for value, bounds6 in case.init_distributions:
            capi.check(L.hlbm_set_distribution(h, value, capi.dvec(bounds6) if bounds6 else None, 0))
        if case.double_couette:
            dc = case.double_couette
            capi.check(L.hlbm_init_double_couette(h, capi.dvec(dc["U"]), "XYZ".index(dc["dimension"])))
        capi.check(L.hlbm_init_obstacles(h))
        for kind, oid, prm in case.obstacles:
            if kind == "ball":
                capi.check(L.hlbm_register_solid_ball(h, oid, capi.dvec(prm[0]), prm[1]))
            elif kind == "wall":
                capi.check(L.hlbm_register_solid_wall(h, oid, capi.dvec(prm[0]), capi.dvec(prm[1])))
            else:
                capi.check(L.hlbm_register_quadric(h, oid, capi.dvec(prm)))
        capi.check(L.hlbm_update_obstacles(h))
        self.record_hooks(case)

    def record_hooks(self, case: Case):
        L, h = self.L, self.h
        capi.check(L.hlbm_clear_hooks(h))
        for hook_name in ("start_iteration", "pre_stream_bcs", "post_stream_bcs", "boundary_conditions"):
            hook = capi.HOOKS[hook_name]
            for op in getattr(case, hook_name):
                s = op.slots
                if op.name == "pre_bounce_back":
                    capi.check(L.hlbm_pre_bounce_back(h))
                elif op.name in ("cavity_z_0", "cavity_z_l"):
                    capi.check(L.hlbm_cavity(h, 1 if op.name.endswith("_l") else 0, capi.dvec(s["U"])))
                elif op.name == "wall_bounce_back":
                    capi.check(L.hlbm_wall_bounce_back(h))
                elif op.name == "post_bounce_back":
                    capi.check(L.hlbm_post_bounce_back(h, hook))
                elif op.name in ("neumann", "lid_driven_cavity"):
                    regions = [PLANE_INDEX[r] for r in s["regions"]]
                    fn = L.hlbm_neumann if op.name == "neumann" else L.hlbm_lid_driven_cavity
                    capi.check(fn(h, hook, capi.dvec(s["U"]), capi.ivec(regions), len(regions)))
                elif op.name == "zero_gradient":
                    regions = [PLANE_INDEX[r] for r in s["regions"]]
                    capi.check(L.hlbm_zero_gradient(h, hook, capi.ivec(regions), len(regions)))
                elif op.name == "set_distribution":
                    b = s.get("bounds")
                    if b is None:
                        raise capi.HlbmError(-5, "start_iteration set_distribution needs bounds")
                    b6 = tuple(b[0]) + tuple(b[1])
                    capi.check(L.hlbm_start_set_distribution(h, float(s.get("value", 1.0)), capi.dvec(b6)))
                else:
                    raise capi.HlbmError(-5, f"operator {op.name} is not on the step path")

    # ------------------------------------------------------------------- run
    def step(self, n: int = 1):
        capi.check(self.L.hlbm_step(self.h, int(n)))
        return self

    def sync(self):
        capi.check(self.L.hlbm_sync(self.h))

    # ---------------------------------------------------------------- output
    def populations(self) -> np.ndarray:
        """(19, nz, ny, nx) FP64 populations of the current state S_k."""
        out = np.empty(Q * self.ncell, dtype=np.float64)
        capi.check(self.L.hlbm_get_populations(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out.reshape(Q, self.n[2], self.n[1], self.n[0])

    def put_populations(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        assert a.size == Q * self.ncell
        capi.check(self.L.hlbm_put_populations(self.h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def checkpoint(self) -> np.ndarray:
        """The carried state as one byte image (header, flags, populations as stored)."""
        n = C.c_int64()
        capi.check(self.L.hlbm_checkpoint_bytes(self.h, C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        capi.check(self.L.hlbm_checkpoint_save(self.h, buf.ctypes.data_as(C.c_void_p), n.value))
        return buf

    def restore(self, image: np.ndarray):
        """Load an image from `checkpoint()` of a lattice built from the same deck."""
        a = np.ascontiguousarray(image, dtype=np.uint8)
        capi.check(self.L.hlbm_checkpoint_load(self.h, a.ctypes.data_as(C.c_void_p), a.size))
        return self

    def save_checkpoint(self, path: str):
        self.checkpoint().tofile(path)

    def load_checkpoint(self, path: str):
        return self.restore(np.fromfile(path, dtype=np.uint8))

    def flags(self) -> np.ndarray:
        out = np.empty(self.ncell, dtype=np.int8)
        capi.check(self.L.hlbm_get_flags(self.h, out.ctypes.data_as(C.POINTER(C.c_int8))))
        return out.reshape(self.n[2], self.n[1], self.n[0])

    def put_flags(self, flags: np.ndarray):
        a = np.ascontiguousarray(flags, dtype=np.int8).reshape(-1)
        capi.check(self.L.hlbm_put_flags(self.h, a.ctypes.data_as(C.POINTER(C.c_int8))))

    def macro(self):
        rho = np.empty(self.ncell)
        u = np.empty(3 * self.ncell)
        capi.check(self.L.hlbm_macro_variables(self.h, rho.ctypes.data_as(C.POINTER(C.c_double)),
                                               u.ctypes.data_as(C.POINTER(C.c_double))))
        s = (self.n[2], self.n[1], self.n[0])
        return rho.reshape(s), u.reshape((3,) + s)

    def simulation_state(self) -> tuple:
        out = (C.c_double * 3)()
        capi.check(self.L.hlbm_simulation_state(self.h, out))
        return tuple(out)

    def plane_velocity_profile(self, dimension: str = "Z"):
        """plane_velocity_profile (plane_velocity_profile.cu:179-260): per plane normal to
        `dimension`, (mean, min, max) of the velocity norm over fluid nodes and the fluid count."""
        dim = {"X": 0, "Y": 1, "Z": 2}[dimension.upper()]
        n = self.n[dim]
        avg, vmin, vmax = np.empty(n), np.empty(n), np.empty(n)
        cnt = np.empty(n, dtype=np.int64)
        dp = C.POINTER(C.c_double)
        capi.check(self.L.hlbm_plane_velocity_profile(self.h, dim, avg.ctypes.data_as(dp), vmin.ctypes.data_as(dp),
                                                      vmax.ctypes.data_as(dp),
                                                      cnt.ctypes.data_as(C.POINTER(C.c_int64))))
        return avg, vmin, vmax, cnt

    def residual(self) -> float:
        out = C.c_double()
        capi.check(self.L.hlbm_residual(self.h, C.byref(out)))
        return out.value

    def moments(self) -> tuple:
        out = (C.c_double * 4)()
        capi.check(self.L.hlbm_moments(self.h, out))
        return tuple(out)

    def wall_force(self) -> tuple:
        out = (C.c_double * 3)()
        capi.check(self.L.hlbm_wall_force(self.h, out))
        return tuple(out)

    def parameters(self) -> dict:
        out = (C.c_double * 9)()
        capi.check(self.L.hlbm_get_parameters(self.h, out))
        o = list(out)
        return {"Fext": tuple(o[0:3]), "celerity": o[3], "dtLB": o[4], "nuth": o[5], "nu": o[6], "tau": o[7],
                "avg_rho": o[8]}

    def info(self) -> dict:
        out = (C.c_int64 * 8)()
        capi.check(self.L.hlbm_info(self.h, out))
        keys = ["nx", "ny", "nz", "precision", "steps", "launches", "bytes_per_population", "device"]
        return dict(zip(keys, list(out)))

    def rounding(self, mode: str):
        """16-bit storage rounding of the carried state: "stochastic" (default) or "nearest"."""
        capi.check(self.L.hlbm_storage_rounding(self.h, {"nearest": 0, "stochastic": 1}[mode]))
        return self

    def tune(self, variant: int):
        capi.check(self.L.hlbm_tune(self.h, int(variant)))
        return self

    def autotune(self, reps: int = 5):
        """Time every step-kernel variant on this lattice (state unchanged) and keep the fastest;
        returns (chosen variant, {variant: ms per step})."""
        chosen = C.c_int32(0)
        ms = (C.c_double * capi.NUM_VARIANTS)()
        capi.check(self.L.hlbm_autotune(self.h, int(reps), C.byref(chosen), ms))
        return chosen.value, {v: ms[v] for v in range(capi.NUM_VARIANTS) if ms[v] >= 0}

    def stream_handle(self) -> int:
        return self.L.hlbm_stream(self.h) or 0
