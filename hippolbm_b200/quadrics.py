"""Quadric obstacles: named unit quadrics and affine transforms.

register_quadrics (register_quadrics.cpp:72-79) takes an Onika `Mat4d` (a named quadric)
and an optional transform M, and registers Q' = M^-T Q M^-1, so that a point p is solid
when (M^-1 p) is inside the unit quadric: p_h^T Q' p_h <= 0 with p_h = (x, y, z, 1)
(obstacle.hpp:134-136).  Onika's named-quadric table and its YAML transform reader are not
part of the reference tree; this module restates them from their geometric meaning, so the
quadric path has no reference pin (flags of ball and wall obstacles are pinned bit for bit).
"""
from __future__ import annotations

import numpy as np

# unit quadrics: x^T A x + ... <= 0 inside
_NAMED = {
    "sphere": np.diag([1.0, 1.0, 1.0, -1.0]),
    "cylx": np.diag([0.0, 1.0, 1.0, -1.0]),
    "cyly": np.diag([1.0, 0.0, 1.0, -1.0]),
    "cylz": np.diag([1.0, 1.0, 0.0, -1.0]),
    "conex": np.diag([-1.0, 1.0, 1.0, 0.0]),
    "coney": np.diag([1.0, -1.0, 1.0, 0.0]),
    "conez": np.diag([1.0, 1.0, -1.0, 0.0]),
}


def named_quadric(name: str) -> np.ndarray:
    try:
        return _NAMED[name].copy()
    except KeyError:
        raise ValueError(f"unknown quadric {name!r}; known: {sorted(_NAMED)}") from None


def transform_matrix(ops) -> np.ndarray:
    """Compose a list of {scale|translate|rotate_x|rotate_y|rotate_z: value} in order."""
    M = np.eye(4)
    for op in ops or []:
        (kind, v), = op.items()
        T = np.eye(4)
        if kind == "scale":
            T[0, 0], T[1, 1], T[2, 2] = (float(e) for e in v)
        elif kind == "translate":
            T[0, 3], T[1, 3], T[2, 3] = (float(e) for e in v)
        elif kind in ("rotate_x", "rotate_y", "rotate_z"):
            a = float(v)
            c, s = np.cos(a), np.sin(a)
            i, j = {"rotate_x": (1, 2), "rotate_y": (2, 0), "rotate_z": (0, 1)}[kind]
            T[i, i], T[i, j], T[j, i], T[j, j] = c, -s, s, c
        else:
            raise ValueError(f"unknown transform {kind!r}")
        M = T @ M
    return M


def apply_transform(Q: np.ndarray, M: np.ndarray) -> np.ndarray:
    Minv = np.linalg.inv(M)
    return Minv.T @ Q @ Minv


def quadric_from_slots(slots: dict) -> tuple:
    """(16 row-major doubles) from register_quadrics slots {quadrics, transform}."""
    q = slots["quadrics"]
    Q = named_quadric(q) if isinstance(q, str) else np.asarray(q, dtype=np.float64).reshape(4, 4)
    if slots.get("transform"):
        Q = apply_transform(Q, transform_matrix(slots["transform"]))
    return tuple(float(v) for v in Q.reshape(16))
