"""The landmark term on the GPU (b200bsp_set_landmarks,
b200bsp_landmarks_score) and inside bspline_score and the optimiser.

Bars:
  landmark term alone   bit-exact against the reference (golden fixtures):
                        the device rounds every product and sum to float in
                        the reference's order
  added in place        bit-exact against the oracle adding the same term
                        into the same starting gradient
  whole bspline_score   the MSE bars (score 1e-5, gradient 1e-3) against the
                        reference, and bit-exact against the device's own
                        score without landmarks plus the landmark term
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import load_golden, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

CASES = ["landmarks_small", "landmarks_dcos"]


@pytest.mark.parametrize("name", CASES)
def test_landmark_term_matches_reference(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_landmarks(rec["fixed_pts"], rec["moving_pts"],
                          float(rec["stiffness"]))
        for _ in range(2):
            lm, g = ctx.landmarks_score(coeff)
            assert np.float32(lm) == rec["lm_score"]
            np.testing.assert_array_equal(g, rec["lm_grad"])


@pytest.mark.parametrize("name", CASES)
def test_landmark_gradient_adds_in_place(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    base = np.linspace(-2, 3, grid.num_coeff).astype(np.float32)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_landmarks(rec["fixed_pts"], rec["moving_pts"], 1.7)
        lm, g = ctx.landmarks_score(coeff, grad=base.copy())
    r = O.port_landmarks(grid, fixed, coeff, rec["fixed_pts"],
                         rec["moving_pts"], 1.7, grad=base)
    assert lm == r.score
    np.testing.assert_array_equal(g, r.grad)


@pytest.mark.parametrize("form", ["tc", "fp32"])
@pytest.mark.parametrize("name", CASES)
def test_bspline_score_with_landmarks(form, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    reg = P.reg_parms(curvature=0.005)
    k = float(rec["stiffness"])
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()           # moving gradient computed on the device
        t0, g0, s0, _ = ctx.score(coeff, "mse", 1.0, reg)
        ctx.set_landmarks(rec["fixed_pts"], rec["moving_pts"], k)
        t1, g1, s1, _ = ctx.score(coeff, "mse", 1.0, reg)
        ctx.set_landmarks([], [])                  # removed again
        t2, g2, _, _ = ctx.score(coeff, "mse", 1.0, reg)
    assert s1 == s0 and t2 == t0
    np.testing.assert_array_equal(g2, g0)
    # the landmark step on top of the device's own metric + regulariser
    r = O.port_landmarks(grid, fixed, coeff, rec["fixed_pts"],
                         rec["moving_pts"], k, grad=g0)
    np.testing.assert_array_equal(g1, r.grad)
    assert np.float32(t1) == np.float32(np.float32(t0)
                                        + np.float32(k) * np.float32(r.score))
    # and against the reference's whole bspline_score
    ref = rec["total_lm_score"]
    assert abs(t1 - ref) <= 1e-5 * abs(ref)
    assert rel_err(g1, rec["total_lm_grad"]) < 1e-3


def test_optimiser_sees_landmarks():
    """With the image metric weighted 0, L-BFGS over the landmark term
    alone pulls the fixed landmarks onto the moving ones."""
    fixed = synth.gaussian_blobs((40, 36, 30), spacing=(1.0, 1.0, 1.5), seed=9)
    grid = BsplineGrid.for_volume(fixed, (8, 8, 6))
    rng = np.random.default_rng(10)
    ijk = rng.uniform(4, 26, (12, 3))
    f = (np.array(fixed.origin) + ijk * np.array(fixed.spacing)).astype(np.float32)
    m = (f + np.array([1.5, -1.0, 0.8], np.float32)).astype(np.float32)
    x0 = np.zeros(grid.num_coeff, np.float32)
    with P.Context(fixed, fixed, grid) as ctx:
        ctx.set_images()
        ctx.set_landmarks(f, m, 1.0)
        lm0, _ = ctx.landmarks_score(x0)
        x, res = ctx.optimize_lbfgs(x0, metric="mse", lam=0.0, max_its=30,
                                    max_feval=60)
        lm1, _ = ctx.landmarks_score(x)
    assert lm0 == pytest.approx(1.5 ** 2 + 1.0 + 0.8 ** 2, rel=1e-5)
    assert lm1 < 0.01 * lm0
    assert res["score"] == pytest.approx(lm1, abs=1e-3 * lm0)


def test_landmark_errors():
    fixed = synth.gaussian_blobs((20, 18, 16), spacing=(1.0, 1.0, 1.0), seed=4)
    grid = BsplineGrid.for_volume(fixed, 5)
    coeff = np.zeros(grid.num_coeff, np.float32)
    o = np.array(fixed.origin, np.float32)
    with P.Context(fixed, fixed, grid) as ctx:
        with pytest.raises(P.B200Error):
            ctx.landmarks_score(coeff)             # none set
        with pytest.raises(P.B200Error):
            ctx.set_landmarks([o + (-3.0, 1.0, 1.0)], [o])
        with pytest.raises(P.B200Error):
            ctx.set_landmarks([o + (1.0, 1.0, 16.5)], [o])
        ctx.set_landmarks([o + (1.0, 2.0, 3.0)], [o + (1.0, 2.0, 3.0)])
        lm, g = ctx.landmarks_score(coeff)
        assert lm == 0.0 and not g.any()
