"""Case model and `.msp` deck reader for the D3Q19 step.

A `Case` is what one hippoLBM deck configures for the time step: the `domain`
(domain_lbm.cpp:41-49), `lbm_parameters` (lbm_parameters.cpp:50-66), the initial
`set_distribution` boxes (set_distribution.cu:52-58), the obstacle list
(register_solid_ball / register_solid_wall / register_quadrics), the collision model
(`collision: bgk|mrt`, config_compute_loop.msp:21) and the ordered operator lists of the
compute-loop hooks `start_iteration`, `pre_stream_bcs`, `post_stream_bcs` and
`boundary_conditions` (config_compute_loop.msp:7-38).  The reader accepts the subset
of Onika's YAML dialect the reference decks use: `includes:`, unit suffixes such as
`0.1 m`, `1e-4`-style numbers that YAML 1.1 leaves as strings, operator entries given
as a bare name or as `{name: {slot: value}}`.
"""
from __future__ import annotations

import copy
import dataclasses
import math
import os
import re
from typing import Any

import yaml

# Operators accepted in each compute-loop hook (the names the reference registers).
HOOK_OPERATORS = {
    "start_iteration": {"set_distribution"},
    "pre_stream_bcs": {"pre_bounce_back", "cavity_z_0", "cavity_z_l", "wall_bounce_back"},
    "post_stream_bcs": {"post_bounce_back", "lid_driven_cavity", "neumann", "zero_gradient"},
    "boundary_conditions": {"neumann", "lid_driven_cavity", "post_bounce_back", "zero_gradient"},
}
PLANES = ["plan_yz_0", "plan_yz_l", "plan_xz_0", "plan_xz_l", "plan_xy_0", "plan_xy_l"]
# traversal names accepted by neumann / lid_driven_cavity (neuman.cu:80-81)
PLANE_INDEX = {name: i for i, name in enumerate(PLANES)}


class DeckError(ValueError):
    """A deck the reference would reject (or that this path does not support)."""


@dataclasses.dataclass
class Op:
    name: str
    slots: dict = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class Case:
    cell_dims: tuple = (30, 30, 30)
    bmin: tuple = (0.0, 0.0, 0.0)
    bmax: tuple = (1.0, 1.0, 1.0)
    periodic: tuple = (False, False, False)
    # lbm_parameters slots and defaults (lbm_parameters.cpp:57-64)
    Fext: tuple = (0.0, 0.0, 0.0)
    celerity: float = 1.0
    nuth: float = 1e-4
    avg_rho: float = 1000.0
    tau: float | None = None
    dt: float = 0.0
    collision: str = "bgk"
    mrt_rates: tuple | None = None  # (s_e, s_eps, s_q, s_pi, s_m, w_eps, w_epsj, w_xx); None = reference
    init_distributions: list = dataclasses.field(default_factory=list)  # [(value, bounds6|None)]
    obstacles: list = dataclasses.field(default_factory=list)  # [(kind, id, params)]
    start_iteration: list = dataclasses.field(default_factory=list)
    pre_stream_bcs: list = dataclasses.field(default_factory=list)
    post_stream_bcs: list = dataclasses.field(default_factory=list)
    boundary_conditions: list = dataclasses.field(default_factory=list)
    steps: int = 100
    checks: list = dataclasses.field(default_factory=list)  # check_macro_quantities slots
    name: str = "case"
    # init_double_couette slots (init_double_couette.cu:51-58): {"U": [...], "dimension": "Z"}
    double_couette: dict | None = None
    # the deck's `analysis` operators (config_analysis.msp) and run controls (`global:`)
    analysis: list = dataclasses.field(default_factory=list)
    run: dict = dataclasses.field(default_factory=dict)

    @property
    def nodes(self) -> tuple:
        return tuple(int(c) + 1 for c in self.cell_dims)

    @property
    def dx(self) -> float:
        return (self.bmax[0] - self.bmin[0]) / float(self.nodes[0] - 1)

    def copy(self, **kw) -> "Case":
        c = copy.deepcopy(self)
        for k, v in kw.items():
            setattr(c, k, v)
        return c

    def to_dict(self) -> dict:
        d = dataclasses.asdict(self)
        for hook in HOOK_OPERATORS:
            d[hook] = [[op.name, op.slots] for op in getattr(self, hook)]
        return d

    @classmethod
    def from_dict(cls, d: dict) -> "Case":
        d = dict(d)
        for hook in HOOK_OPERATORS:
            d[hook] = [Op(name, dict(slots)) for name, slots in d.get(hook, [])]
        d["analysis"] = [Op(a["name"], dict(a["slots"])) if isinstance(a, dict) else a for a in d.get("analysis", [])]
        for k in ("cell_dims", "bmin", "bmax", "periodic", "Fext"):
            d[k] = tuple(d[k])
        if d.get("mrt_rates") is not None:
            d["mrt_rates"] = tuple(d["mrt_rates"])
        d["init_distributions"] = [(v, tuple(b) if b else None) for v, b in d.get("init_distributions", [])]
        obs = []
        for kind, oid, prm in d.get("obstacles", []):
            if kind == "ball":
                prm = (tuple(prm[0]), float(prm[1]))
            elif kind == "wall":
                prm = (tuple(prm[0]), tuple(prm[1]))
            else:
                prm = tuple(prm)
            obs.append((kind, int(oid), prm))
        d["obstacles"] = obs
        return cls(**d)

    def validate(self) -> None:
        """Reject decks the reference rejects (domain_lbm.cpp:81-106) or the plan cannot hold."""
        n = self.nodes
        if any(v < 2 for v in n):
            raise DeckError("domain: every cell_dims entry must be >= 1")
        reso = [(self.bmax[d] - self.bmin[d]) / float(n[d] - 1) for d in range(3)]
        if reso[0] != reso[1] or reso[0] != reso[2]:
            raise DeckError(f"[Error, domain], Dx is not the same for all dimension: {reso}")
        for d in range(3):
            if self.bmin[d] + (n[d] - 1) * reso[0] != self.bmax[d]:
                raise DeckError("[Error, domain], The resolution slot and bounds slot mismatch.")
        if self.collision not in ("bgk", "mrt"):
            raise DeckError(f"unknown collision model {self.collision!r}")
        for hook in HOOK_OPERATORS:
            for op in getattr(self, hook):
                if op.name not in HOOK_OPERATORS[hook]:
                    raise DeckError(f"operator {op.name!r} is not supported in hook {hook!r}")
                for r in op.slots.get("regions", []):
                    if r not in PLANE_INDEX:
                        raise DeckError(f"Traversal name not allowed: {r}")


# --------------------------------------------------------------------- parsing
_NUM_UNIT = re.compile(r"^\s*([-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)\s*([A-Za-z/%\.\-\^0-9]*)\s*$")
# Onika unit suffixes map to SI; the decks only use metres and seconds.
_UNIT_SCALE = {"": 1.0, "m": 1.0, "s": 1.0, "m/s": 1.0, "mm": 1e-3, "cm": 1e-2, "um": 1e-6, "ms": 1e-3}


def _num(v: Any) -> Any:
    if isinstance(v, bool):
        return v
    if isinstance(v, (int, float)):
        return v
    if isinstance(v, str):
        m = _NUM_UNIT.match(v)
        if m:
            unit = m.group(2)
            if unit not in _UNIT_SCALE:
                raise DeckError(f"unsupported unit {unit!r} in {v!r}")
            x = float(m.group(1)) * _UNIT_SCALE[unit]
            return x
    if isinstance(v, list):
        return [_num(e) for e in v]
    if isinstance(v, dict):
        return {k: _num(e) for k, e in v.items()}
    return v


def _vec3(v, what) -> tuple:
    v = _num(v)
    if not isinstance(v, list) or len(v) != 3:
        raise DeckError(f"{what}: expected a 3-vector, got {v!r}")
    return tuple(float(e) for e in v)


def _bounds(v, what) -> tuple:
    v = _num(v)
    if isinstance(v, dict):
        return _vec3(v["bmin"], what), _vec3(v["bmax"], what)
    if not isinstance(v, list) or len(v) != 2:
        raise DeckError(f"{what}: expected [[min],[max]], got {v!r}")
    return _vec3(v[0], what), _vec3(v[1], what)


def _ops(entries) -> list:
    """Operator list of a hook: bare names or {name: slots} (Onika batch syntax)."""
    if entries is None or entries == "nop":
        return []
    if isinstance(entries, str):
        entries = [entries]
    if isinstance(entries, dict):
        entries = [entries]
    out = []
    for e in entries:
        if isinstance(e, str):
            out.append(Op(e, {}))
        elif isinstance(e, dict) and len(e) == 1:
            (name, slots), = e.items()
            out.append(Op(name, _num(slots) if isinstance(slots, dict) else {}))
        else:
            raise DeckError(f"cannot read operator entry {e!r}")
    return out


def _load_yaml_tree(path: str, seen=None) -> dict:
    seen = seen or set()
    path = os.path.abspath(path)
    if path in seen:
        return {}
    seen.add(path)
    with open(path) as fh:
        doc = yaml.safe_load(fh) or {}
    merged: dict = {}
    for inc in doc.get("includes", []) or []:
        inc_path = inc if os.path.isabs(inc) else os.path.join(os.path.dirname(path), inc)
        if os.path.exists(inc_path):
            merged.update(_load_yaml_tree(inc_path, seen))
    for k, v in doc.items():
        if k == "includes":
            continue
        if k == "global" and isinstance(v, dict):
            merged.setdefault("global", {}).update(v)
        else:
            merged[k] = v
    return merged


def case_from_tree(tree: dict, name: str = "deck") -> Case:
    """Build a Case from a parsed deck (the keys a user's .msp overrides)."""
    c = Case(name=name)
    dom_ops = _ops(tree.get("do_domain"))
    for op in dom_ops:
        if op.name != "domain":
            continue
        s = op.slots
        if "cell_dims" not in s:
            raise DeckError("domain: slot cell_dims is REQUIRED (domain_lbm.cpp:47)")
        c.cell_dims = tuple(int(v) for v in _num(s["cell_dims"]))
        c.bmin, c.bmax = _bounds(s["bounds"], "domain.bounds")
        c.periodic = tuple(bool(v) for v in s.get("periodic", [False] * 3))
    for op in _ops(tree.get("set_lbm_parameters")):
        if op.name != "lbm_parameters":
            continue
        s = op.slots
        if "Fext" in s:
            c.Fext = _vec3(s["Fext"], "Fext")
        c.celerity = float(s.get("celerity", c.celerity))
        c.nuth = float(s.get("nuth", c.nuth))
        c.avg_rho = float(s.get("avg_rho", c.avg_rho))
        if "tau" in s:
            c.tau = float(s["tau"])
        c.dt = float(s.get("dt", c.dt))
    # initial distributions: the `set_distributions` hook (config_initialize.msp:4,24).
    for op in _ops(tree.get("set_distributions")):
        if op.name == "init_double_couette":
            dim = str(op.slots.get("dimension", ""))
            if dim not in ("X", "Y", "Z"):
                raise DeckError('[init_double_couette] Please, select a valid dimension "X", "Y", or "Z".')
            c.double_couette = {"U": list(_vec3(op.slots["U"], "init_double_couette.U")), "dimension": dim}
            continue
        if op.name != "set_distribution":
            continue
        b = op.slots.get("bounds")
        bounds6 = None
        if b is not None:
            lo, hi = _bounds(b, "set_distribution.bounds")
            bounds6 = lo + hi
        c.init_distributions.append((float(op.slots.get("value", 1.0)), bounds6))
    for op in _ops(tree.get("set_obstacles")):
        s = op.slots
        if op.name == "register_solid_ball":
            c.obstacles.append(("ball", int(s["id"]), (_vec3(s["center"], "center"), float(s["radius"]))))
        elif op.name == "register_solid_wall":
            c.obstacles.append(("wall", int(s["id"]), _bounds(s["bounds"], "wall.bounds")))
        elif op.name == "register_quadrics":
            from .quadrics import quadric_from_slots

            c.obstacles.append(("quadric", int(s["id"]), quadric_from_slots(s)))
        elif op.name == "init_obstacles":
            c.obstacles.clear()
        else:
            raise DeckError(f"unknown obstacle operator {op.name!r}")
    col = tree.get("collision", "bgk")
    c.collision = col if isinstance(col, str) else "bgk"
    c.start_iteration = _ops(tree.get("start_iteration"))
    c.pre_stream_bcs = _ops(tree.get("pre_stream_bcs"))
    c.post_stream_bcs = _ops(tree.get("post_stream_bcs"))
    c.boundary_conditions = _ops(tree.get("boundary_conditions"))
    g = tree.get("global", {}) or {}
    c.steps = int(_num(g.get("simulation_end_iteration", 100)))
    # run controls, defaults of config_initialize.msp:36-43 and write_paraview.cpp:51-53
    c.run = {"paraview_freq": int(_num(g.get("simulation_paraview_freq", -1))),
             "analysis_freq": int(_num(g.get("simulation_analysis_freq", -1))),
             "print_log_freq": int(_num(g.get("simulation_print_log_freq", 1))),
             "display_paraview_first_timestep": bool(g.get("display_paraview_first_timestep", True)),
             "output_directory": str(g.get("output_directory", "hippoLBMOutputDir"))}
    ana = tree.get("analysis")
    c.analysis = _ops(ana) if isinstance(ana, list) else []
    for op in _ops(tree.get("checker_op")):
        if op.name == "check_macro_quantities":
            c.checks.append(dict(op.slots))
    return c


def load_msp(path: str) -> Case:
    """Read a user deck (and its `includes:`) into a Case."""
    tree = _load_yaml_tree(path)
    c = case_from_tree(tree, name=os.path.splitext(os.path.basename(path))[0])
    c.validate()
    return c


def loads_msp(text: str, name: str = "deck") -> Case:
    tree = yaml.safe_load(text) or {}
    c = case_from_tree(tree, name=name)
    c.validate()
    return c


# ----------------------------------------------------------------- parameters
def lbm_parameters(case: Case) -> dict:
    """LBMParametersOp::execute (lbm_parameters.cpp:73-99) in the reference's arithmetic."""
    dx = case.dx
    p = {"nuth": case.nuth, "avg_rho": case.avg_rho}
    if case.dt > 0.0:  # define_by_dt, lbm_parameters.hpp:60-66
        p["dtLB"] = case.dt
        p["tau"] = 3 * p["nuth"] * p["dtLB"] / (dx * dx) + 0.5
        p["nu"] = (p["tau"] - 0.5) / 3.0
        p["celerity"] = dx / p["dtLB"]
    elif case.tau is not None:  # define_by_tau, lbm_parameters.hpp:68-74
        p["tau"] = case.tau
        p["dtLB"] = dx * dx * (p["tau"] - 0.5) / (3.0 * p["nuth"])
        p["nu"] = p["nuth"] * p["dtLB"] / (dx * dx)
        p["celerity"] = dx / p["dtLB"]
    else:  # define_by_c, lbm_parameters.hpp:76-81
        p["celerity"] = case.celerity
        p["dtLB"] = dx / p["celerity"]
        p["nu"] = p["nuth"] * p["dtLB"] / (dx * dx)
        p["tau"] = 3.0 * p["nu"] + 0.5
    ddx = p["celerity"] * p["dtLB"]  # convert_force<LBM_UNITS>, lbm_parameters.hpp:124-128
    p["Fext"] = tuple(f * p["dtLB"] * p["dtLB"] / ddx for f in case.Fext)
    if not (p["tau"] > 0.5) or not math.isfinite(p["tau"]):
        raise DeckError(f"lbm_parameters: tau = {p['tau']} must be > 0.5")
    return p


# ----------------------------------------------------------- built-in cases
def couette_case(n: int, tau: float, u_wall: float, steps: int, collision: str = "bgk",
                 periodic=(True, True, False)) -> Case:
    """Couette flow in lattice units: n^3 nodes, dx = 1, bounce-back at z = 0 and a wall moving
    along x at z = n - 1 (pre_bounce_back + cavity_z_l + post_bounce_back)."""
    return Case(
        name=f"couette{n}_{collision}", cell_dims=(n - 1,) * 3, bmin=(0.0,) * 3, bmax=(float(n - 1),) * 3,
        periodic=tuple(periodic), tau=tau, nuth=(tau - 0.5) / 3.0, collision=collision,
        pre_stream_bcs=[Op("pre_bounce_back"), Op("cavity_z_l", {"U": [u_wall, 0.0, 0.0]})],
        post_stream_bcs=[Op("post_bounce_back")], steps=steps)


# MRT rates with the stress-independent rates given explicitly and every other rate 1.0
# (s_e = 1.19, s_eps = 1.4, s_q = 1.2, s_pi = s_m = 1.0; the equilibrium weights stay those of
# mrt.hpp:43-47: w_eps = 0, w_epsj = -475/63, w_xx = 0).  The reference's own set keeps s_m = 1.98,
# which drives the closed sphere channel unstable at tau = 0.56 within a hundred steps.
MRT_RATES_REST_ONE = (1.19, 1.4, 1.2, 1.0, 1.0, 0.0, -475.0 / 63.0, 0.0)


def sphere_channel_case(nodes=(1024, 256, 256), center=(256.0, 128.0, 128.0), radius: float = 24.0,
                        tau: float = 0.56, u_in: float = 0.04, steps: int = 20000, collision: str = "mrt",
                        mrt_rates=MRT_RATES_REST_ONE) -> Case:
    """Flow past a sphere in a closed channel, lattice units (dx = dt = 1): bounce-back on the
    sphere (wall_bounce_back) and on the y / z walls (plane bounce-back), a Zou/He velocity inlet
    u_x = u_in on plan_yz_0 and a zero-gradient outlet on plan_yz_l.  Starts from rest (f = w)."""
    nx, ny, nz = (int(v) for v in nodes)
    return Case(
        name=f"sphere_channel{nx}x{ny}x{nz}_{collision}", cell_dims=(nx - 1, ny - 1, nz - 1), bmin=(0.0,) * 3,
        bmax=(float(nx - 1), float(ny - 1), float(nz - 1)), periodic=(False, False, False), tau=tau,
        nuth=(tau - 0.5) / 3.0, collision=collision, mrt_rates=mrt_rates,
        obstacles=[("ball", 0, (tuple(float(c) for c in center), float(radius)))],
        pre_stream_bcs=[Op("pre_bounce_back"), Op("wall_bounce_back")],
        post_stream_bcs=[Op("post_bounce_back")],
        boundary_conditions=[Op("neumann", {"U": [float(u_in), 0.0, 0.0], "regions": ["plan_yz_0"]}),
                             Op("zero_gradient", {"regions": ["plan_yz_l"]})],
        steps=steps)


def poiseuille_case(nodes, tau: float, force: float, steps: int, collision: str = "bgk") -> Case:
    """Body-force driven channel: periodic in x and y, Zou/He zero-velocity walls (neumann U = 0)
    on the z planes, force along x in lattice units."""
    nx, ny, nz = (int(v) for v in nodes)
    return Case(name=f"poiseuille{nx}x{ny}x{nz}_{collision}", cell_dims=(nx - 1, ny - 1, nz - 1), bmin=(0.0,) * 3,
                bmax=(float(nx - 1), float(ny - 1), float(nz - 1)), periodic=(True, True, False), tau=tau,
                nuth=(tau - 0.5) / 3.0, collision=collision, Fext=(float(force), 0.0, 0.0),
                boundary_conditions=[Op("neumann", {"U": [0.0, 0.0, 0.0], "regions": ["plan_xy_0", "plan_xy_l"]})],
                steps=steps)


def lid_cavity_case(nodes, tau: float, u_lid: float, steps: int, collision: str = "bgk") -> Case:
    """Closed box, plane bounce-back on every face and a lid moving along x on plan_xy_l."""
    nx, ny, nz = (int(v) for v in nodes)
    return Case(name=f"cavity{nx}x{ny}x{nz}_{collision}", cell_dims=(nx - 1, ny - 1, nz - 1), bmin=(0.0,) * 3,
                bmax=(float(nx - 1), float(ny - 1), float(nz - 1)), periodic=(False, False, False), tau=tau,
                nuth=(tau - 0.5) / 3.0, collision=collision,
                pre_stream_bcs=[Op("pre_bounce_back")],
                post_stream_bcs=[Op("post_bounce_back"),
                                 Op("lid_driven_cavity", {"U": [float(u_lid), 0.0, 0.0], "regions": ["plan_xy_l"]})],
                steps=steps)


def mixed_batch_cases(count: int = 256, seed: int = 20261203, steps: int = 2000) -> list[Case]:
    """Independent lattices drawn from `seed`: each axis length uniform on {32, 40, ..., 128}; the
    case uniform among Couette (wall speed U[0.01, 0.08]), Poiseuille (body force U[1e-6, 1e-5]) and
    lid-driven cavity (lid speed U[0.02, 0.1]); BGK or MRT; tau uniform in [0.55, 1.2]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    edges = np.arange(32, 129, 8)
    out = []
    for i in range(count):
        nodes = tuple(int(v) for v in rng.choice(edges, size=3))
        kind = str(rng.choice(["couette", "poiseuille", "cavity"]))
        collision = str(rng.choice(["bgk", "mrt"]))
        tau = float(rng.uniform(0.55, 1.2))
        if kind == "couette":
            c = couette_case(nodes[0], tau, float(rng.uniform(0.01, 0.08)), steps, collision)
            nx, ny, nz = nodes
            c.cell_dims = (nx - 1, ny - 1, nz - 1)
            c.bmax = (float(nx - 1), float(ny - 1), float(nz - 1))
        elif kind == "poiseuille":
            c = poiseuille_case(nodes, tau, float(rng.uniform(1e-6, 1e-5)), steps, collision)
        else:
            c = lid_cavity_case(nodes, tau, float(rng.uniform(0.02, 0.1)), steps, collision)
        c.name = f"m{i}_{kind}_{nodes[0]}x{nodes[1]}x{nodes[2]}_{collision}"
        out.append(c)
    return out
