"""The reduced-precision tiers against FP64 on a reduced flow past a sphere.

MRT (stress-independent rates 1.0, deck.MRT_RATES_REST_ONE), tau = 0.56, a 256 x 64 x 64 closed
channel with a sphere of radius 6 at (64, 32, 32), Zou/He velocity inlet u_x = 0.04 at x = 0,
zero-gradient outlet at x = 255, bounce-back on the sphere and the y / z walls, 4000 steps from
rest.  Each tier runs the same deck; against the FP64 run of it:

  tier                               rel. L2 of u   |mass drift - FP64's|   |drag rel. diff|
  FP32                                   1e-5              1e-7                  1e-4
  FP16 deviations, stochastic rounding   1e-3              1e-5                  3e-3
  BF16 deviations, stochastic rounding   5e-3              1e-4                  2e-2

The L2 bound of FP16 storage is the target the tier is built for; the others bound what an error
in the shared deviation-form collision (bgk_v / mrt_fast with DEVF, the rest-state reference
dref, the stochastic rounding) would break.
"""
import pytest

from hippolbm_b200.deck import sphere_channel_case

pytestmark = pytest.mark.gpu

BOUNDS = {"f32": (1e-5, 1e-7, 1e-4), "f16": (1e-3, 1e-5, 3e-3), "bf16": (5e-3, 1e-4, 2e-2)}


@pytest.fixture(scope="module")
def study():
    from hippolbm_b200.precision import precision_study

    case = sphere_channel_case((256, 64, 64), (64.0, 32.0, 32.0), 6.0, tau=0.56, u_in=0.04, steps=4000)
    recs = precision_study(case, ("f64", "f32", "f16", "bf16"), case.steps, chunk=1000)
    for r in recs:
        print({k: r[k] for k in ("precision", "l2_u", "mass_drift", "mass_drift_diff", "drag", "drag_rel_diff")})
    return {r["precision"]: r for r in recs}


def test_fp64_reference_run_is_physical(study):
    r = study["f64"]
    assert r["drag"] > 0.0  # the flow pushes the sphere downstream
    assert abs(r["mass_drift"]) < 0.1


@pytest.mark.parametrize("tier", ["f32", "f16", "bf16"])
def test_tier_against_fp64(study, tier):
    l2_max, drift_max, drag_max = BOUNDS[tier]
    r = study[tier]
    assert r["l2_u"] <= l2_max, r
    assert abs(r["mass_drift_diff"]) <= drift_max, r
    assert abs(r["drag_rel_diff"]) <= drag_max, r
