"""Gradient check with the analytic curvature regulariser: 128x128x96
Gaussian-blob volumes (as the 64^3 registration workload), vox_per_rgn 6,
curvature lambda 0.005, the analytic gradient through the C ABI and through
the torch.autograd.Function binding.

Checks and their bars:
  binding       the autograd backward returns exactly the C ABI gradient
                and the forward value is the C ABI total score
  finite diff.  central differences of the total score (MSE in double +
                regulariser in double) with a 1e-3 mm step on 64 seeded
                control-point coefficients, against the analytic gradient
                with the trilinear-derivative moving gradient (the exact
                derivative of the trilinear score, the reference's flavour
                o); relative L2 error over the 64 components <= FD_L2 and
                every component within FD_ABS * max |quotient| of its
                difference quotient.  The quotient itself carries the kinks of the
                trilinear interpolant (voxels crossing a cell face between
                the two evaluations): both forms land at the same error,
                so it is not the tensor cores' split rounding.
  reference     score within 1e-5 and gradient within 1e-3 (relative L2) of
                the reference's own bspline_score() with the same regulariser
                (flavour g for the nearest-voxel gradient, o for trilinear)
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

FORMS = ["fp32", "tc"]
LAMBDA = 0.005
STEP = 1e-3          # mm
N_POINTS = 64
FD_L2 = 6e-3         # measured 3.2e-3 (FP32 form), 3.0e-3 (TC form)
FD_ABS = 5e-3        # measured 2.7e-3, 2.0e-3

needs_ref = pytest.mark.skipif(not O.ref_available(),
                               reason="reference build absent")


def c3_case(seed=synth.SEED_BASE + 2):
    fixed = synth.gaussian_blobs((128, 128, 96), seed=seed)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, seed + 1))
    grid = BsplineGrid.for_volume(fixed, 6)
    coeff = synth.random_coeff(grid, 1.0, seed + 2)
    return fixed, moving, grid, coeff


def points(grid, seed=synth.SEED_BASE + 2, n=N_POINTS):
    return np.sort(synth.rng(seed + 3).choice(grid.num_coeff, n,
                                              replace=False))


def total_f64(ctx, coeff, reg):
    s, _, _ = ctx.score_mse_f64(coeff)
    r, _ = ctx.regularize_f64(coeff, reg)
    return s + r


def fd_errors(form):
    """(analytic gradient at the points, difference quotients)."""
    torch = pytest.importorskip("torch")
    from plastimatch_b200.autograd import bspline_score
    fixed, moving, grid, coeff = c3_case()
    reg = P.reg_parms(curvature=LAMBDA)
    idx = points(grid)
    with P.Context(fixed, moving, grid, form=form,
                   mse_grad="trilinear") as ctx:
        ctx.set_images()
        c = torch.tensor(coeff, requires_grad=True)
        s = bspline_score(c, ctx, reg=reg)
        s.backward()
        g = c.grad.numpy().astype(np.float64)
        fd = np.zeros(len(idx))
        for n, i in enumerate(idx):
            cp, cm = coeff.copy(), coeff.copy()
            cp[i] += np.float32(STEP)
            cm[i] -= np.float32(STEP)
            h2 = float(cp[i]) - float(cm[i])      # the step as stored
            fd[n] = (total_f64(ctx, cp, reg) - total_f64(ctx, cm, reg)) / h2
    return g[idx], fd


@pytest.mark.parametrize("form", FORMS)
def test_autograd_binding_is_the_abi_gradient(form):
    torch = pytest.importorskip("torch")
    from plastimatch_b200.autograd import bspline_score
    fixed, moving, grid, coeff = c3_case()
    reg = P.reg_parms(curvature=LAMBDA)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        ts, tg, _, _ = ctx.score(coeff, reg=reg)
        for device in ("cpu", "cuda"):
            c = torch.tensor(coeff, device=device, requires_grad=True)
            s = bspline_score(c, ctx, reg=reg)
            (g,) = torch.autograd.grad(2.0 * s, c)
            assert float(s.detach()) == ts
            assert g.device.type == device
            np.testing.assert_array_equal(g.cpu().numpy(), 2.0 * tg)


@pytest.mark.parametrize("form", FORMS)
def test_gradient_against_finite_differences(form):
    g, fd = fd_errors(form)
    err = rel_err(g, fd)
    worst = float(np.max(np.abs(g - fd)))
    assert err <= FD_L2, (err, worst)
    assert worst <= FD_ABS * float(np.max(np.abs(fd))), (err, worst)


@needs_ref
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("mode,flavor", [("nearest", "g"),
                                         ("trilinear", "o")])
def test_gradient_against_reference(form, mode, flavor):
    fixed, moving, grid, coeff = c3_case()
    reg = P.reg_parms(curvature=LAMBDA)
    with P.Context(fixed, moving, grid, form=form, mse_grad=mode) as ctx:
        ctx.set_images()
        ts, tg, _, _ = ctx.score(coeff, reg=reg)
    ref = O.ref_score(grid, fixed, moving, coeff, flavor=flavor,
                      reg_impl="c", curvature=LAMBDA)
    assert abs(ts - ref.score) <= 1e-5 * abs(ref.score), (ts, ref.score)
    assert rel_err(tg, ref.grad) < 1e-3, rel_err(tg, ref.grad)
