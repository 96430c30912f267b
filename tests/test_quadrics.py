"""Quadric obstacles (register_quadrics, register_quadrics.cpp:72-84; Quadric::solid,
obstacle.hpp:134-136): a node at p is solid when p_h^T Q p_h <= 0, p_h = (x, y, z, 1).

Onika's quadric_eval and its named-quadric table are not in the reference tree, so quadric flags
have no reference pin.  They are checked here against the oracle's restatement (bit-exact flags on
the GPU), against geometry (named quadrics under transforms), and against the reference-pinned
ball: a quadric sphere and register_solid_ball rasterise to the same flags where no node lies on
the surface.
"""
import numpy as np
import pytest

from hippolbm_b200 import quadrics
from hippolbm_b200.deck import Case, Op, loads_msp


def qval(q16, p):
    Q = np.asarray(q16, dtype=np.float64).reshape(4, 4)
    ph = np.array([p[0], p[1], p[2], 1.0])
    return float(ph @ Q @ ph)


def test_named_quadrics_and_transform_geometry():
    sph = quadrics.quadric_from_slots({"id": 0, "quadrics": "sphere",
                                       "transform": [{"scale": [3, 3, 3]}, {"translate": [10, 4, 5]}]})
    assert qval(sph, (10, 4, 5)) < 0 and qval(sph, (13.1, 4, 5)) > 0 and qval(sph, (12.9, 4, 5)) < 0
    cyl = quadrics.quadric_from_slots({"id": 1, "quadrics": "cylz",
                                       "transform": [{"scale": [2, 2, 1]}, {"translate": [5, 5, 0]}]})
    assert qval(cyl, (5, 5, -100)) < 0 and qval(cyl, (5, 6.9, 40)) < 0 and qval(cyl, (5, 7.1, 0)) > 0
    # a cylinder along x rotated by +90 degrees about z runs along y
    rot = quadrics.quadric_from_slots({"id": 2, "quadrics": "cylx", "transform": [{"rotate_z": np.pi / 2}]})
    assert qval(rot, (0.0, 50.0, 0.0)) < 0 and qval(rot, (50.0, 0.0, 0.0)) > 0
    with pytest.raises(ValueError):
        quadrics.named_quadric("torus")
    with pytest.raises(ValueError):
        quadrics.transform_matrix([{"shear": 1}])


def test_deck_register_quadrics_slots():
    case = loads_msp("""
domain:
  cell_dims: [15, 15, 15]
  bounds: [[0, 0, 0], [15, 15, 15]]
  periodic: [false, false, false]
lbm_parameters:
  tau: 0.8
  nuth: 0.1
set_obstacles:
  - register_quadrics:
      id: 0
      quadrics: sphere
      transform:
        - scale: [3, 3, 3]
        - translate: [7.5, 7.5, 7.5]
""")
    (kind, oid, q), = case.obstacles
    assert kind == "quadric" and oid == 0 and len(q) == 16
    assert qval(q, (7.5, 7.5, 7.5)) == pytest.approx(-1.0)


def quadric_case():
    sphere = quadrics.quadric_from_slots({"id": 0, "quadrics": "sphere",
                                          "transform": [{"scale": [4.2, 3.1, 2.7]}, {"rotate_y": 0.4},
                                                        {"translate": [9.3, 8.0, 7.6]}]})
    cylinder = quadrics.quadric_from_slots({"id": 1, "quadrics": "cylz",
                                            "transform": [{"scale": [1.8, 1.8, 1.0]}, {"rotate_x": 0.3},
                                                          {"translate": [20.4, 6.6, 0.0]}]})
    # half-space x >= 27.5 as a plane quadric: 2 * (-0.5) * x + 27.5 <= 0
    plane = (0, 0, 0, -0.5, 0, 0, 0, 0, 0, 0, 0, 0, -0.5, 0, 0, 27.5)
    cone = quadrics.quadric_from_slots({"id": 3, "quadrics": "conex",
                                        "transform": [{"scale": [1.0, 0.5, 0.5]}, {"translate": [12.0, 13.0, 12.0]}]})
    # no periodic axis: the reference rasterises walls on its ghost layers from their own positions
    # rather than as periodic images, so walls that touch a periodic face differ by design
    return Case(name="quadrics", cell_dims=(31, 17, 15), bmin=(0, 0, 0), bmax=(31, 17, 15),
                periodic=(False, False, False), tau=0.8, nuth=0.1,
                obstacles=[("quadric", 0, sphere), ("quadric", 1, cylinder), ("quadric", 2, plane),
                           ("quadric", 3, cone)],
                pre_stream_bcs=[Op("pre_bounce_back"), Op("wall_bounce_back")],
                post_stream_bcs=[Op("post_bounce_back")], steps=10)


def test_oracle_rasterises_every_quadric(oracle_mod):
    lat = oracle_mod.OracleLattice(quadric_case(), "port").initialize()
    walls = lat.real(lat.obst()) == -2
    lat.close()
    # [z, y, x]: the half-space x >= 28, the sphere's centre, the cylinder's axis, the cone's axis on
    # both sides of its apex (12, 13, 12), and off-axis points near the apex; the cylinder, tilted about
    # x, moves to smaller y as z grows
    assert walls[:, :, 28:].all() and not walls[:, :, 27].all()
    assert walls[8, 8, 9] and walls[0, 7, 20] and walls[14, 2, 20] and not walls[14, 7, 20]
    assert walls[12, 13, 5] and walls[12, 13, 19] and not walls[12, 16, 12] and not walls[12, 13 - 3, 13]


@pytest.mark.gpu
def test_gpu_quadric_flags_equal_oracle(oracle_mod):
    from hippolbm_b200.lattice import Lattice

    case = quadric_case()
    ref = oracle_mod.OracleLattice(case, "port").initialize()
    obst = ref.real(ref.obst()).copy()
    ref.step(case.steps)
    f_ref = ref.real(ref.f()).copy()
    ref.close()
    with Lattice.from_case(case, "f64_strict") as lat:
        flags = lat.flags()
        lat.step(case.steps)
        f = lat.populations()
    assert np.count_nonzero(obst == -2) > 500
    assert np.array_equal(flags.astype(np.int32), obst)
    fluid = obst != -2
    assert np.array_equal(f[:, fluid], f_ref[:, fluid])


@pytest.mark.gpu
def test_gpu_quadric_sphere_equals_ball():
    """No node lies on the sphere (centre at half-integers, radius 3: |p - c|^2 = k + 0.75), so the
    two tests decide every node the same way."""
    from hippolbm_b200.lattice import Lattice

    centre, r = (8.5, 7.5, 6.5), 3.0
    q = quadrics.quadric_from_slots({"id": 0, "quadrics": "sphere",
                                     "transform": [{"scale": [r, r, r]}, {"translate": list(centre)}]})
    base = dict(cell_dims=(17, 15, 13), bmin=(0, 0, 0), bmax=(17, 15, 13), periodic=(True, True, True), tau=0.8,
                nuth=0.1, steps=1)
    with Lattice.from_case(Case(name="qs", obstacles=[("quadric", 0, q)], **base), "f64") as a:
        fa = a.flags()
    with Lattice.from_case(Case(name="ball", obstacles=[("ball", 0, (centre, r))], **base), "f64") as b:
        fb = b.flags()
    assert np.count_nonzero(fa == -2) > 50
    assert np.array_equal(fa, fb)
