"""Analytic regulariser and the whole cost function on the GPU.

Tolerances:
  regulariser score     relative 1e-6 against the reference (golden) and
                        the double-precision oracle
  regulariser gradient  relative 1e-6 (L2): the device adds the double
                        per-knot gradient into the float gradient once,
                        the reference adds its 64 double slot values one by
                        one
  total score/gradient  the MSE bars (score 1e-5, gradient 1e-3)
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

ALL = dict(curvature=0.7, diffusion=0.3, lame_1=0.4, lame_2=0.6,
           total_displacement=0.05, third_order=0.02,
           linear_elastic_multiplier=1.3, curvature_mixed_weight=0.8)


@pytest.mark.parametrize("name", golden_names("mse"))
def test_regularizer_golden(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid, form="fp32") as ctx:
        s, g = ctx.regularize(coeff, P.reg_parms(curvature=0.005))
    assert abs(s - rec["reg_score"]) <= 1e-6 * abs(rec["reg_score"])
    assert rel_err(g, rec["reg_grad"]) < 1e-6


@pytest.mark.parametrize("name", golden_names("mse"))
@pytest.mark.parametrize("which", ["all", "elastic", "third"])
def test_regularizer_every_term(name, which):
    kw = {"all": ALL, "elastic": dict(lame_1=1.0, lame_2=2.0),
          "third": dict(third_order=0.5, total_displacement=0.1)}[which]
    fixed, moving, grid, coeff, _ = load_golden(name)
    with P.Context(fixed, moving, grid, form="fp32") as ctx:
        s, g = ctx.regularize(coeff, P.reg_parms(**kw))
    r64 = O.port_reg(grid, fixed, coeff, O.penalties(**kw), precision="f64")
    assert abs(s - r64.score) <= 1e-6 * abs(r64.score)
    assert rel_err(g, r64.grad) < 1e-6


def test_regularizer_adds_into_gradient_and_switches_weights():
    fixed = synth.gaussian_blobs((40, 36, 30), spacing=(1.2, 1.0, 2.0), seed=5)
    grid = BsplineGrid.for_volume(fixed, (5, 6, 4))
    coeff = synth.random_coeff(grid, 1.5, 6)
    base = np.linspace(-1, 1, grid.num_coeff).astype(np.float32)
    with P.Context(fixed, fixed, grid, form="fp32") as ctx:
        for kw in (dict(curvature=0.01), ALL, {}):
            s, g = ctx.regularize(coeff, P.reg_parms(**kw), grad=base.copy())
            if not kw:
                assert s == 0.0
                np.testing.assert_array_equal(g, base)
                continue
            r64 = O.port_reg(grid, fixed, coeff, O.penalties(**kw),
                             precision="f64")
            assert abs(s - r64.score) <= 1e-6 * abs(r64.score)
            assert rel_err(g - base, r64.grad) < 1e-5


@pytest.mark.parametrize("form", ["fp32", "tc"])
@pytest.mark.parametrize("name", [n for n in golden_names("mse")])
def test_total_score_golden(form, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        ts, tg, sm, n = ctx.score(coeff, "mse", 1.0,
                                  P.reg_parms(curvature=0.005))
    assert abs(ts - rec["total_score"]) <= 1e-5 * abs(rec["total_score"])
    assert rel_err(tg, rec["total_grad"]) < 1e-3


@pytest.mark.parametrize("form", ["tc", "fp32"])
@pytest.mark.parametrize("with_reg", [True, False])
def test_score_device_path_matches_host_path(form, with_reg):
    """b200bsp_score with device outputs (the regulariser on a second
    stream, overlapping the tile kernel, combined by the finish kernel) is
    bit-identical to the host-output path (metric, then regulariser, in
    sequence)."""
    import torch
    fixed, moving, grid, coeff, rec = load_golden("mse_small")
    reg = P.reg_parms(curvature=0.005, diffusion=0.1) if with_reg else None
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        ts, g, sm, n = ctx.score(coeff, lam=0.7, reg=reg)
        d_c = torch.from_numpy(coeff).cuda()
        d_g = torch.zeros(grid.num_coeff, device="cuda")
        d_ts = torch.zeros(1, device="cuda")
        d_sm = torch.zeros(1, device="cuda")
        d_n = torch.zeros(1, dtype=torch.int64, device="cuda")
        import ctypes as C
        for _ in range(2):
            rc = P.lib().b200bsp_score(
                ctx._h, d_c.data_ptr(), 0, C.c_float(0.7),
                C.byref(reg) if reg is not None else None, d_ts.data_ptr(),
                d_g.data_ptr(), d_sm.data_ptr(), d_n.data_ptr())
            assert rc == 0
            torch.cuda.synchronize()
            assert float(d_ts.item()) == ts and float(d_sm.item()) == sm
            assert int(d_n.item()) == n
            assert np.array_equal(d_g.cpu().numpy(), g)
