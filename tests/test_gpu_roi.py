"""Image ROIs (uchar fixed / moving masks) on the GPU against the oracle and
the reference's ROI flavours (MSE i, MI h).

Bars (as for the evaluations without ROIs):
  score     relative 1e-5 against the double-precision oracle with the same
            ROIs
  gradient  relative 1e-3 (L2) against the double oracle and the
            reference's float output (golden record)
  num_vox   within 0.01 % (+2) of the reference's count: the fixed ROI test
            is computed in the reference's float arithmetic (bit for bit);
            a moving position within float rounding of a moving-ROI voxel
            face may land on the other side
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import (ROI_TAGS, golden_names, load_golden, load_rois,
                      pick_rois, rel_err)
from plastimatch_b200.geometry import Roi

pytestmark = pytest.mark.gpu

FORMS = ["tc", "fp32"]


def _check(s, g, n, f64, ref_grad, nv_ref):
    assert abs(n - nv_ref) <= 1e-4 * nv_ref + 2, (n, nv_ref)
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score), (s, f64.score)
    assert rel_err(g, f64.grad) < 1e-3, rel_err(g, f64.grad)
    assert rel_err(g, ref_grad) < 1e-3, rel_err(g, ref_grad)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("tag", ROI_TAGS)
@pytest.mark.parametrize("name", golden_names("roimask_mse"))
def test_mse_roi_golden(form, tag, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    fr, mr = pick_rois(tag, *load_rois(rec))
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        ctx.set_roi(fr, mr)
        s, g, n = ctx.score_mse(coeff)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=rec["moving_grad"],
                     precision="f64", fixed_roi=fr, moving_roi=mr)
    _check(s, g, n, f64, rec[f"{tag}_g_grad"], int(rec[f"{tag}_g_num_vox"]))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("tag", ROI_TAGS)
@pytest.mark.parametrize("name", golden_names("roimask_mi"))
def test_mi_roi_golden(form, tag, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    fr, mr = pick_rois(tag, *load_rois(rec))
    with P.Context(fixed, moving, grid, form=form, mi_bins=32) as ctx:
        ctx.set_images()
        ctx.set_roi(fr, mr)
        s, g, n, (fh, mh, jh) = ctx.score_mi(coeff, with_hist=True)
    f64 = O.port_mi(grid, fixed, moving, coeff, bins=32, precision="f64",
                    fixed_roi=fr, moving_roi=mr)
    _check(s, g, n, f64, rec[f"{tag}_mi_grad"], int(rec[f"{tag}_mi_num_vox"]))
    assert rel_err(jh, rec[f"{tag}_j_hist"]) < 1e-5


@pytest.mark.parametrize("form", FORMS)
def test_mse_roi_trilinear_gradient(form):
    """ROIs with the trilinear-derivative gradient (no reference flavour
    has both; checked against the double oracle)."""
    fixed, moving, grid, coeff, rec = load_golden("roimask_mse_small")
    fr, mr = load_rois(rec)
    with P.Context(fixed, moving, grid, form=form,
                   mse_grad="trilinear") as ctx:
        ctx.set_images()
        ctx.set_roi(fr, mr)
        s, g, n = ctx.score_mse(coeff)
    f64 = O.port_mse(grid, fixed, moving, coeff, grad_mode=1,
                     precision="f64", fixed_roi=fr, moving_roi=mr)
    assert abs(n - f64.num_vox) <= 1e-4 * f64.num_vox + 2
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score)
    assert rel_err(g, f64.grad) < 1e-3


def test_roi_set_replace_and_remove():
    """set_roi replaces the ROIs; no arguments remove them (the result is
    then the ROI-free one, bit for bit: the context returns to the kernel it
    used without ROIs); a geometry without its mask is an argument error."""
    fixed, moving, grid, coeff, rec = load_golden("roimask_mse_small")
    fr, mr = load_rois(rec)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        s0, g0, n0 = ctx.score_mse(coeff)
        ctx.set_roi(fr, mr)
        s1, g1, n1 = ctx.score_mse(coeff)
        ctx.set_roi(None, mr)
        s2, g2, n2 = ctx.score_mse(coeff)
        ctx.set_roi()
        s3, g3, n3 = ctx.score_mse(coeff)
        all_in = Roi.like(fixed, np.ones(fixed.img.shape, np.uint8))
        ctx.set_roi(all_in, None)
        s4, g4, n4 = ctx.score_mse(coeff)
        rc = P.lib().b200bsp_set_roi(ctx._h, None, fr.mask.ctypes.data,
                                     None, None)
        assert rc == -1                          # B200BSP_E_BADARG
    assert n1 < n2 < n0
    assert s3 == s0 and n3 == n0 and np.array_equal(g3, g0)
    # a mask that holds everywhere changes nothing but the kernel: ROIs run
    # on the x-lane kernel, the ROI-free context on the tile kernel, whose
    # tensor-core sums group the same products differently
    assert n4 == n0 and abs(s4 - s0) <= 1e-6 * abs(s0)
    assert rel_err(g4, g0) < 1e-5


@pytest.mark.parametrize("form", FORMS)
def test_headline_workload_with_window_roi(form):
    """The 256x256x128 CT phantom with a fixed ROI from an intensity window
    (body only, as a registration stage builds it from its MI window) and a
    moving ROI from the same window on the moving image."""
    import bench
    fixed, moving, grid, coeff = bench.make_workload()
    fr = Roi.from_window(fixed, -500.0, 3000.0)
    mr = Roi.from_window(moving, -500.0, 3000.0)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        ctx.set_roi(fr, mr)
        s, g, n = ctx.score_mse(coeff)
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg,
                     precision="f64", fixed_roi=fr, moving_roi=mr)
    assert abs(n - f64.num_vox) <= 1e-4 * f64.num_vox + 2
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score)
    assert rel_err(g, f64.grad) < 1e-3
    if O.ref_available():
        r = O.ref_metric(grid, fixed, moving, coeff, flavor="g", threads=8,
                         moving_grad=mg, fixed_roi=fr, moving_roi=mr)
        assert abs(n - r.num_vox) <= 1e-4 * r.num_vox + 2
        assert rel_err(g, r.grad) < 1e-3
