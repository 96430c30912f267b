"""ctypes binding of include/hippolbm.h (libhippolbm.so, built in-tree for sm_100a).

The library is loaded from the package directory; a missing or unloadable library is an
error (there is no fallback path).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhippolbm.so")

HLBM_F64, HLBM_F64_STRICT, HLBM_F32, HLBM_F16, HLBM_BF16 = 0, 1, 2, 3, 4
PRECISIONS = {"f64": HLBM_F64, "f64_strict": HLBM_F64_STRICT, "f32": HLBM_F32, "f16": HLBM_F16, "bf16": HLBM_BF16}
HOOK_START, HOOK_PRE, HOOK_POST, HOOK_BC = 0, 1, 2, 3
HOOKS = {"start_iteration": HOOK_START, "pre_stream_bcs": HOOK_PRE, "post_stream_bcs": HOOK_POST,
         "boundary_conditions": HOOK_BC}
ERRORS = {-1: "EINVAL", -2: "EDOMAIN", -3: "ECUDA", -4: "ENOMEM", -5: "EPLAN", -6: "ESTATE"}

_d3 = C.POINTER(C.c_double)
_i3 = C.POINTER(C.c_int32)
_vp = C.c_void_p
# name -> (restype, argtypes); every symbol include/hippolbm.h declares
NUM_VARIANTS = 10  # HLBM_NUM_VARIANTS of include/hippolbm.h
BATCH_VARIANTS = 5  # HLBM_BATCH_VARIANTS: batch variants 6 .. 10

SIGNATURES = {
    "hlbm_last_error": (C.c_char_p, []),
    "hlbm_version": (C.c_char_p, []),
    "hlbm_domain": (C.c_int, [_i3, _d3, _d3, _i3, C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "hlbm_destroy": (C.c_int, [_vp]),
    "hlbm_trim_memory": (C.c_int, [C.c_int32]),
    "hlbm_lbm_parameters": (C.c_int, [_vp, _d3, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_double,
                                      C.c_double]),
    "hlbm_get_parameters": (C.c_int, [_vp, _d3]),
    "hlbm_collision": (C.c_int, [_vp, C.c_int32, _d3]),
    "hlbm_storage_scale": (C.c_int, [_vp, C.c_double, C.c_double]),
    "hlbm_storage_rounding": (C.c_int, [_vp, C.c_int32]),
    "hlbm_set_distribution": (C.c_int, [_vp, C.c_double, _d3, C.c_int32]),
    "hlbm_init_double_couette": (C.c_int, [_vp, _d3, C.c_int32]),
    "hlbm_init_obstacles": (C.c_int, [_vp]),
    "hlbm_register_solid_ball": (C.c_int, [_vp, C.c_int32, _d3, C.c_double]),
    "hlbm_register_solid_wall": (C.c_int, [_vp, C.c_int32, _d3, _d3]),
    "hlbm_register_quadric": (C.c_int, [_vp, C.c_int32, _d3]),
    "hlbm_update_obstacles": (C.c_int, [_vp]),
    "hlbm_clear_hooks": (C.c_int, [_vp]),
    "hlbm_pre_bounce_back": (C.c_int, [_vp]),
    "hlbm_cavity": (C.c_int, [_vp, C.c_int32, _d3]),
    "hlbm_wall_bounce_back": (C.c_int, [_vp]),
    "hlbm_post_bounce_back": (C.c_int, [_vp, C.c_int32]),
    "hlbm_neumann": (C.c_int, [_vp, C.c_int32, _d3, _i3, C.c_int32]),
    "hlbm_lid_driven_cavity": (C.c_int, [_vp, C.c_int32, _d3, _i3, C.c_int32]),
    "hlbm_start_set_distribution": (C.c_int, [_vp, C.c_double, _d3]),
    "hlbm_zero_gradient": (C.c_int, [_vp, C.c_int32, _i3, C.c_int32]),
    "hlbm_step": (C.c_int, [_vp, C.c_int64]),
    "hlbm_sync": (C.c_int, [_vp]),
    "hlbm_macro_variables": (C.c_int, [_vp, _d3, _d3]),
    "hlbm_simulation_state": (C.c_int, [_vp, _d3]),
    "hlbm_plane_velocity_profile": (C.c_int, [_vp, C.c_int32, _d3, _d3, _d3, C.POINTER(C.c_int64)]),
    "hlbm_residual": (C.c_int, [_vp, _d3]),
    "hlbm_moments": (C.c_int, [_vp, _d3]),
    "hlbm_wall_force": (C.c_int, [_vp, _d3]),
    "hlbm_get_populations": (C.c_int, [_vp, _d3]),
    "hlbm_put_populations": (C.c_int, [_vp, _d3]),
    "hlbm_checkpoint_bytes": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "hlbm_checkpoint_save": (C.c_int, [_vp, _vp, C.c_int64]),
    "hlbm_checkpoint_load": (C.c_int, [_vp, _vp, C.c_int64]),
    "hlbm_get_flags": (C.c_int, [_vp, C.POINTER(C.c_int8)]),
    "hlbm_put_flags": (C.c_int, [_vp, C.POINTER(C.c_int8)]),
    "hlbm_info": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "hlbm_tune": (C.c_int, [_vp, C.c_int32]),
    "hlbm_autotune": (C.c_int, [_vp, C.c_int32, _i3, _d3]),
    "hlbm_stream": (_vp, [_vp]),
    "hlbm_set_wait_limit": (C.c_int, [_vp, C.c_int64]),
    "hlbm_batch_create": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "hlbm_batch_add": (C.c_int, [_vp, _vp]),
    "hlbm_batch_remove": (C.c_int, [_vp, _vp]),
    "hlbm_batch_step": (C.c_int, [_vp, C.c_int64]),
    "hlbm_batch_tune": (C.c_int, [_vp, C.c_int32]),
    "hlbm_batch_autotune": (C.c_int, [_vp, C.c_int32, _i3, _d3]),
    "hlbm_batch_info": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "hlbm_batch_stream": (_vp, [_vp]),
    "hlbm_batch_destroy": (C.c_int, [_vp]),
    "hlbm_simulation_state_static": (C.c_int, [_d3, C.c_int64, C.POINTER(C.c_int8), _i3, _d3, _vp]),
}

_lib = None


class HlbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load libhippolbm.so (raises if it is missing: the CUDA path has no substitute)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run `python __graft_entry__.py build` or "
                                f"`make -C hippolbm_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != 0:
        raise HlbmError(rc, lib().hlbm_last_error().decode())


def dvec(v):
    return (C.c_double * len(v))(*[float(x) for x in v])


def ivec(v):
    return (C.c_int32 * len(v))(*[int(x) for x in v])
