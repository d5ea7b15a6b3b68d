"""Dense vector field and warped moving image on the GPU against the
reference's golden outputs (bspline_interpolate_vf, bspline_warp linear).

Tolerances:
  field   max |difference| <= 1e-5 * (1 + max |field|) mm: the device sums
          the 64 knot terms with its own basis products and order
  warp    |difference| <= 1e-4 * max |moving| for all but 0.01% (+2) of the
          voxels: a voxel whose displaced position lies within float
          rounding of the moving image's edge may fall on the other side and
          take the default value instead of a sample (or the reverse)
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu


def _check_vf(vf, ref):
    tol = 1e-5 * (1.0 + float(np.abs(ref).max()))
    assert np.abs(vf - ref).max() <= tol, np.abs(vf - ref).max()


def _check_warp(w, ref, moving_img):
    bad = np.abs(w - ref) > 1e-4 * float(np.abs(moving_img).max())
    assert bad.sum() <= 1e-4 * ref.size + 2, bad.sum()


@pytest.mark.parametrize("name", golden_names("warp") + golden_names("vf"))
def test_interpolate_vf_golden(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        vf = ctx.interpolate_vf(coeff)
    _check_vf(vf, rec["vf"])
    if name.startswith("vf"):
        # outside the ROI the field is zero, as the reference leaves it
        assert (vf[rec["vf"] == 0] == 0).all()


@pytest.mark.parametrize("name", golden_names("warp"))
def test_warp_golden(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        w = ctx.warp(coeff, float(rec["default"]))
    _check_warp(w, rec["warped"], moving.img)
    assert (w == rec["default"]).any()


def test_warp_and_field_device_outputs_64cubed():
    torch = pytest.importorskip("torch")
    fixed = synth.gaussian_blobs((64, 60, 56), spacing=(1.0, 1.2, 1.5),
                                 seed=12)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, 13))
    grid = BsplineGrid.for_volume(fixed, (6, 5, 4))
    coeff = synth.random_coeff(grid, 2.5, 14)
    ref_w, ref_vf = O.port_warp(grid, fixed, moving, coeff, 3.5, with_vf=True)
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        w_h = ctx.warp(coeff, 3.5)
        vf_h = ctx.interpolate_vf(coeff)
        dc = torch.from_numpy(coeff).cuda()
        w_d = torch.zeros(fixed.npix, device="cuda")
        vf_d = torch.zeros(fixed.npix * 3, device="cuda")
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        P._check(P.lib().b200bsp_warp(ctx._h, dc.data_ptr(), 3.5,
                                      w_d.data_ptr()), ctx._h)
        P._check(P.lib().b200bsp_interpolate_vf(ctx._h, dc.data_ptr(),
                                                vf_d.data_ptr()), ctx._h)
        torch.cuda.synchronize()
    _check_vf(vf_h, ref_vf)
    _check_warp(w_h, ref_w, moving.img)
    np.testing.assert_array_equal(w_d.cpu().numpy().reshape(w_h.shape), w_h)
    np.testing.assert_array_equal(vf_d.cpu().numpy().reshape(vf_h.shape), vf_h)


def test_warp_rejects_partial_roi():
    fixed, moving, grid, coeff, rec = load_golden("vf_roi")
    with P.Context(fixed, moving, grid) as ctx:
        ctx.set_images()
        with pytest.raises(P.B200Error) as e:
            ctx.warp(coeff)
        assert e.value.code == -6
