"""Mattes MI (PVI-8) score + gradient on the GPU against the oracle.

Tolerances (float work, stated here as the bar):
  score      relative 1e-5 against the double-precision oracle
  gradient   relative 1e-3 (L2 norm of the difference over the norm of the
             reference) against the double oracle and the reference's float
             flavour g (golden record)
  histograms relative 1e-5 (L2) against the reference's pass-1 histograms;
             the device sums corner weights as integers in 2^-24 units, and its
             pass 1 takes world positions as origin + step * index where the
             reference accumulates x positions step by step
  num_vox    within 0.01% (+2), as for MSE
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

# "tc-xlane": the tensor-core form with its x-lane kernel pinned (the
# default runs MI on the tile kernel)
FORMS = ["fp32", "tc", "tc-xlane"]


def _context(fixed, moving, grid, form="tc", **kw):
    if form == "tc-xlane":
        return P.Context(fixed, moving, grid, form="tc", tc_kernel="xlane",
                         **kw)
    return P.Context(fixed, moving, grid, form=form, **kw)


def _check(s, g, n, f64, ref_grad, nv_ref):
    assert abs(n - nv_ref) <= 1e-4 * nv_ref + 2, (n, nv_ref)
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score), (s, f64.score)
    assert rel_err(g, f64.grad) < 1e-3, rel_err(g, f64.grad)
    assert rel_err(g, ref_grad) < 1e-3, rel_err(g, ref_grad)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", golden_names("mi"))
def test_mi_golden(form, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with _context(fixed, moving, grid, form=form, mi_bins=32) as ctx:
        ctx.set_images()
        s, g, n, (fh, mh, jh) = ctx.score_mi(coeff, with_hist=True)
    f64 = O.port_mi(grid, fixed, moving, coeff, bins=32, precision="f64")
    _check(s, g, n, f64, rec["mi_grad"], int(rec["mi_num_vox"]))
    assert rel_err(fh, rec["f_hist"]) < 1e-5
    assert rel_err(mh, rec["m_hist"]) < 1e-5
    assert rel_err(jh, rec["j_hist"]) < 1e-5


def _case(shape=(64, 64, 64), vpr=8, seed=20261205):
    fixed = synth.gaussian_blobs(shape, spacing=(1, 1, 1), seed=seed)
    g0 = BsplineGrid.for_volume(fixed, vpr)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, seed + 1))
    grid = BsplineGrid.for_volume(fixed, vpr)
    coeff = synth.random_coeff(grid, 1.0, seed + 2)
    return fixed, moving, grid, coeff


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("bins", [2, 32, 64])
def test_mi_64cubed_bins(form, bins):
    # tiles of 6 x 5 x 4 voxels: the tensor-core form runs its own passes
    fixed, moving, grid, coeff = _case(vpr=(6, 5, 4))
    with _context(fixed, moving, grid, form=form, mi_bins=bins) as ctx:
        ctx.set_images()
        s, g, n = ctx.score_mi(coeff)
        s2, g2, n2 = ctx.score_mi(coeff)
    f64 = O.port_mi(grid, fixed, moving, coeff, bins=bins, precision="f64")
    r32 = O.port_mi(grid, fixed, moving, coeff, bins=bins)
    _check(s, g, n, f64, r32.grad, r32.num_vox)
    # deterministic: fixed-point histograms and fixed-order gathers
    assert s == s2 and n == n2
    np.testing.assert_array_equal(g, g2)


@pytest.mark.parametrize("vpr", [(6, 5, 4), (5, 5, 5), (8, 8, 8), (9, 7, 6)])
def test_mi_tensor_core_form_matches_fp32_form(vpr):
    """The tensor-core MI passes (field and adjoint as GEMMs) against the
    FP32 tile passes: histograms within 1e-5 (L2), score 1e-5, gradient
    1e-3, voxel count within 0.01% (+2)."""
    fixed, moving, grid, coeff = _case(shape=(48, 40, 36), vpr=vpr, seed=3)
    out = []
    for form in FORMS:
        with _context(fixed, moving, grid, form=form) as ctx:
            ctx.set_images()
            out.append(ctx.score_mi(coeff, with_hist=True))
    s0, g0, n0, h0 = out[0]
    for s1, g1, n1, h1 in out[1:]:
        assert abs(n1 - n0) <= 1e-4 * n0 + 2, (n0, n1)
        assert abs(s1 - s0) <= 1e-5 * abs(s0), (s0, s1)
        assert rel_err(g1, g0) < 1e-3, rel_err(g1, g0)
        for a, b in zip(h1, h0):
            assert rel_err(a, b) < 1e-5


@pytest.mark.parametrize("form", FORMS)
def test_mi_no_overlap_and_roi_rejected(form):
    fixed, moving, grid, _ = _case(shape=(32, 32, 32), vpr=8, seed=9)
    with _context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        far = np.full(grid.num_coeff, 1e4, np.float32)
        s, g, n = ctx.score_mi(far)
        assert n == 0 and s == np.finfo(np.float32).max
        assert not g.any()
    roi = BsplineGrid.for_volume(fixed, 8, roi_offset=(2, 0, 0),
                                 roi_dim=(28, 32, 32))
    with _context(fixed, moving, roi, form=form) as ctx:
        ctx.set_images()
        with pytest.raises(P.B200Error) as e:
            ctx.score_mi(np.zeros(roi.num_coeff, np.float32))
        assert e.value.code == -6


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", golden_names("vopt_mi"))
def test_mi_vopt_golden(form, name):
    """V-optimal bins: the device's bin images come from the restated
    dynamic programme; the passes are those of equal spacing."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    with _context(fixed, moving, grid, form=form, mi_bins=32,
                   mi_hist="vopt") as ctx:
        ctx.set_images()
        s, g, n, (fh, mh, jh) = ctx.score_mi(coeff, with_hist=True)
    f64 = O.port_mi(grid, fixed, moving, coeff, bins=32, precision="f64",
                    hist="vopt")
    _check(s, g, n, f64, rec["mi_grad"], int(rec["mi_num_vox"]))
    assert rel_err(fh, rec["f_hist"]) < 1e-5
    assert rel_err(jh, rec["j_hist"]) < 1e-5


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("with_reg", [False, True])
def test_mi_score_device_path_matches_host_path(form, with_reg):
    """b200bsp_score with MI and device outputs (stream-ordered: both
    passes, the regulariser, the combine kernel) is bit-identical to the
    host-output path."""
    import ctypes as C
    import torch
    fixed, moving, grid, coeff = _case(vpr=(6, 5, 4))
    reg = P.reg_parms(curvature=0.005) if with_reg else None
    with _context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        ts, g, sm, n = ctx.score(coeff, metric="mi", lam=0.7, reg=reg)
        d_c = torch.from_numpy(coeff).cuda()
        d_g = torch.zeros(grid.num_coeff, device="cuda")
        d_ts = torch.zeros(1, device="cuda")
        d_sm = torch.zeros(1, device="cuda")
        d_n = torch.zeros(1, dtype=torch.int64, device="cuda")
        for _ in range(2):
            rc = P.lib().b200bsp_score(
                ctx._h, d_c.data_ptr(), 1, C.c_float(0.7),
                C.byref(reg) if reg is not None else None, d_ts.data_ptr(),
                d_g.data_ptr(), d_sm.data_ptr(), d_n.data_ptr())
            assert rc == 0
            torch.cuda.synchronize()
            assert float(d_ts.item()) == ts and float(d_sm.item()) == sm
            assert int(d_n.item()) == n
            assert np.array_equal(d_g.cpu().numpy(), g)
