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
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

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


def _blobs_case(seed=20261208):
    fixed = synth.gaussian_blobs((64, 56, 48), spacing=(1.0, 1.1, 1.3),
                                 seed=seed)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, seed + 1))
    return fixed, moving


@pytest.mark.parametrize("form", ["fp32", "tc"])
@pytest.mark.parametrize("vpr, with_reg", [(8, True), (8, False), (4, True)])
def test_graph_run_matches_host_driven_run(form, vpr, with_reg):
    """The graph-resident iterations (one launch) against the host-driven
    loop on the same registration: MSE, optionally with the curvature
    regulariser.  The controller rounds as the host does; the two differ
    only in the summation order of their dot products (the graph sums each
    one's block partials with one warp, and small grids' new-line-search
    branch runs in one block), so the bar is the same trials and scores to
    1e-5."""
    _compare_graph_and_host(_blobs_case(), form, vpr, with_reg)


@pytest.mark.parametrize("with_reg", [False, True])
def test_graph_run_matches_host_driven_run_large_grid(with_reg):
    """As above on a grid of more than 2^17 coefficients, whose
    new-line-search branch is the multi-block chain (correction pair and
    first loop step, each loop step fused with the next dot product's
    partials, gp.d after the last step)."""
    fixed = synth.gaussian_blobs((160, 160, 96), spacing=(1.0, 1.0, 1.5),
                                 seed=20261209)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, 20261210))
    assert BsplineGrid.for_volume(fixed, 4).num_coeff > 1 << 17
    _compare_graph_and_host((fixed, moving), "tc", 4, with_reg)


@pytest.mark.parametrize("form", ["fp32", "tc"])
@pytest.mark.parametrize("with_reg", [False, True])
def test_graph_run_matches_host_driven_run_mattes_mi(form, with_reg):
    """As above with Mattes MI (PVI-8, 32 bins) as the metric: its
    evaluation in the graph is both passes, the regulariser and the combine
    kernel, the same kernels the host-driven loop launches."""
    _compare_graph_and_host(_blobs_case(), form, 8, with_reg, metric="mi")


def _compare_graph_and_host(case, form, vpr, with_reg, metric="mse"):
    fixed, moving = case
    grid = BsplineGrid.for_volume(fixed, vpr)
    reg = P.reg_parms(curvature=0.005) if with_reg else None
    x0 = np.zeros(grid.num_coeff, np.float32)
    out = []
    for host in (1, 0):
        P.lib().b200bsp_debug_host_lbfgs(host)
        try:
            with P.Context(fixed, moving, grid, form=form) as ctx:
                ctx.set_images()
                out.append(ctx.optimize_lbfgs(x0, metric=metric, reg=reg,
                                              max_its=15, max_feval=40))
        finally:
            P.lib().b200bsp_debug_host_lbfgs(0)
    (c_h, r_h), (c_g, r_g) = out
    assert r_g["fevals"] == r_h["fevals"], (r_g, r_h)
    assert r_g["iterations"] == r_h["iterations"], (r_g, r_h)
    assert r_g["status"] == r_h["status"], (r_g, r_h)
    assert abs(r_g["score"] - r_h["score"]) <= 1e-5 * abs(r_h["score"])
    assert np.linalg.norm(c_g - c_h) <= 1e-4 * max(np.linalg.norm(c_h), 1.0)
