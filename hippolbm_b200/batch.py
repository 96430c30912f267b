"""Many independent lattices advanced together: one persistent-kernel launch per time step over
the tiles of every member (hlbm_batch_* in include/hippolbm.h)."""
from __future__ import annotations

import ctypes as C

from . import capi
from .lattice import Lattice


class Batch:
    def __init__(self, precision: str = "f32", device: int = 0):
        self.L = capi.lib()
        self.h = C.c_void_p()
        capi.check(self.L.hlbm_batch_create(capi.PRECISIONS[precision], device, C.byref(self.h)))
        self.members: list[Lattice] = []

    def add(self, lat: Lattice):
        capi.check(self.L.hlbm_batch_add(self.h, lat.h))
        self.members.append(lat)
        return self

    def remove(self, lat: Lattice):
        capi.check(self.L.hlbm_batch_remove(self.h, lat.h))
        self.members.remove(lat)
        return self

    def step(self, n: int = 1):
        capi.check(self.L.hlbm_batch_step(self.h, int(n)))
        return self

    def tune(self, variant: int):
        """8: one CTA per tile (default); 9: persistent tile walk; 6 / 7: pipelined kernel;
        10: every member's own single-lattice kernel, run concurrently from one captured graph."""
        capi.check(self.L.hlbm_batch_tune(self.h, int(variant)))
        return self

    def autotune(self, reps: int = 3):
        """Time one step of every batch variant on these members (no member's state advances) and
        keep the fastest; returns (chosen variant, {variant: ms per step})."""
        chosen = C.c_int32(0)
        ms = (C.c_double * capi.BATCH_VARIANTS)()
        capi.check(self.L.hlbm_batch_autotune(self.h, int(reps), C.byref(chosen), ms))
        return chosen.value, {6 + k: ms[k] for k in range(capi.BATCH_VARIANTS) if ms[k] >= 0}

    def info(self) -> dict:
        out = (C.c_int64 * 6)()
        capi.check(self.L.hlbm_batch_info(self.h, out))
        return dict(zip(["members", "tiles", "tile_elems", "stages", "graph_replays", "launches"], list(out)))

    def stream_handle(self) -> int:
        return self.L.hlbm_batch_stream(self.h) or 0

    def close(self):
        if self.h and self.h.value:
            self.L.hlbm_batch_destroy(self.h)
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
