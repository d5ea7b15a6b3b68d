"""The device L-BFGS against the reference's optimiser.

  Rosenbrock (n = 100): b200bsp_lbfgs_minimize and liblbfgs (vendored in the
    reference, default parameters) see the same function values, so they
    take the same decisions: equal iteration and evaluation counts, final x
    within 1e-9 (only dot-product rounding differs).
  Registration: b200bsp_optimize_lbfgs and Plastimatch's bspline_optimize
    (implementation liblbfgs) from the same coefficients, 10 iterations: the
    GPU score differs from the CPU one in the last float bits, which the
    trajectory amplifies; the bar is the same evaluation count and a final
    (last evaluated) score within 1e-3 relative.
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import load_golden

pytestmark = pytest.mark.gpu


def rosenbrock(x):
    f = 0.0
    g = np.zeros_like(x)
    for i in range(0, len(x), 2):
        t1 = 1.0 - x[i]
        t2 = 10.0 * (x[i + 1] - x[i] * x[i])
        g[i + 1] = 20.0 * t2
        g[i] = -2.0 * (x[i] * g[i + 1] + t1)
        f += t1 * t1 + t2 * t2
    return f, g


@pytest.mark.parametrize("max_its", [10, 1000])
def test_rosenbrock_matches_liblbfgs(max_its):
    x0 = np.tile([-1.2, 1.0], 50)
    xr, fr, rc, kr, fer = O.ref_lbfgs(rosenbrock, x0, max_its=max_its)
    x, res = P.lbfgs_minimize(rosenbrock, x0, max_its=max_its,
                              max_feval=10 ** 6)
    assert res["fevals"] == fer
    assert res["iterations"] == kr
    np.testing.assert_allclose(x, xr, rtol=0, atol=1e-9)
    if max_its == 1000:
        assert res["status"] == 0 and res["score"] < 1e-10
    else:
        # stopped at the first evaluation of iteration 11: back at the
        # point of iteration 10
        assert res["status"] == 1 and res["iterations"] == 10


def test_quadratic_converges_and_start_at_minimum():
    a = np.linspace(1.0, 5.0, 40)

    def quad(x):
        return 0.5 * float(np.sum(a * x * x)), a * x

    x, res = P.lbfgs_minimize(quad, np.ones(40), max_its=100, max_feval=1000)
    assert res["status"] == 0 and np.abs(x).max() < 1e-4
    x, res = P.lbfgs_minimize(quad, np.zeros(40))
    assert res["status"] == 2 and res["fevals"] == 1


@pytest.mark.parametrize("form", ["fp32", "tc"])
def test_registration_matches_plastimatch_liblbfgs(form):
    fixed, moving, grid, coeff, rec = load_golden("mse_small")
    c_ref, s_ref, it_ref, fe_ref = O.ref_optimize(grid, fixed, moving, coeff,
                                                  max_its=10, max_feval=30)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        c, res = ctx.optimize_lbfgs(coeff, max_its=10, max_feval=30)
    assert res["fevals"] == fe_ref
    assert abs(res["score"] - s_ref) <= 1e-3 * abs(s_ref), (res["score"], s_ref)
    assert res["score"] < 0.05 * float(rec["g_score"])
    assert np.linalg.norm(c - c_ref) <= 1e-2 * np.linalg.norm(c_ref - coeff)
