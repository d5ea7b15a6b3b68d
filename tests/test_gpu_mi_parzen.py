"""Mattes MI with cubic B-spline Parzen windows on the GPU against the
double-precision oracle (the published method, Mattes et al. IEEE TMI 2003;
the reference has no Parzen flavour, so parity is against the restatement).

Bars: score relative 1e-5, gradient relative L2 1e-3, joint histogram
relative L2 1e-5, voxel count within 0.01% (+2) -- as for PVI-8 MI.  The
oracle's own gradient is checked against its central differences in
tests/test_oracle_parzen.py, so these bars also tie the device gradient to
the derivative of the score.
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid, Volume

pytestmark = pytest.mark.gpu

FORMS = ["fp32", "tc"]


def _case(shape=(48, 40, 36), vpr=(6, 5, 4), seed=61, dcos=None, roi=None):
    fixed = synth.gaussian_blobs(shape, spacing=(1.0, 1.2, 1.5), seed=seed)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.5, seed + 1))
    # a monotone intensity remap, as in a multi-modal pair
    moving = synth.intensity_remap(moving, 0.7, 5.0, seed + 2)
    if dcos is not None:
        fixed = Volume(fixed.img, origin=fixed.origin, spacing=fixed.spacing,
                       dcos=dcos)
        moving = Volume(moving.img, origin=moving.origin,
                        spacing=moving.spacing, dcos=dcos)
    kw = {} if roi is None else dict(roi_offset=roi[0], roi_dim=roi[1])
    grid = BsplineGrid.for_volume(fixed, vpr, **kw)
    coeff = synth.random_coeff(grid, 1.0, seed + 3)
    return fixed, moving, grid, coeff


def _check(out, ref):
    s, g, n, (fh, mh, jh) = out
    assert abs(n - ref.num_vox) <= 1e-4 * ref.num_vox + 2, (n, ref.num_vox)
    assert abs(s - ref.score) <= 1e-5 * abs(ref.score), (s, ref.score)
    assert rel_err(g, ref.grad) < 1e-3, rel_err(g, ref.grad)
    assert rel_err(jh, ref.j_hist) < 1e-5, rel_err(jh, ref.j_hist)
    assert rel_err(mh, ref.m_hist) < 1e-5
    assert rel_err(fh, ref.f_hist) < 1e-5


CASES = {
    "axis_small_tiles": dict(),
    "tiles_of_512": dict(vpr=(8, 8, 8)),
    "rotated": dict(dcos=(0.0, 1.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0)),
    "roi": dict(roi=((4, 3, 2), (36, 30, 28))),
    "rotated_tiles_of_512": dict(vpr=(8, 8, 8), dcos=(
        0.0, 1.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0)),
}


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("bins", [16, 32])
def test_parzen_mi_against_oracle(form, case, bins):
    fixed, moving, grid, coeff = _case(**CASES[case])
    with P.Context(fixed, moving, grid, form=form, mi_bins=bins,
                   mi_window="parzen") as ctx:
        ctx.set_images()
        out = ctx.score_mi(coeff, with_hist=True)
        again = ctx.score_mi(coeff)
    ref = O.port_mi_parzen(grid, fixed, moving, coeff, bins=bins)
    _check(out, ref)
    # deterministic
    assert again[0] == out[0] and again[2] == out[2]
    np.testing.assert_array_equal(again[1], out[1])


def test_parzen_tensor_core_form_matches_fp32_form():
    fixed, moving, grid, coeff = _case(shape=(64, 56, 40), vpr=(5, 5, 5),
                                       seed=71)
    out = []
    for form in FORMS:
        with P.Context(fixed, moving, grid, form=form,
                       mi_window="parzen") as ctx:
            ctx.set_images()
            out.append(ctx.score_mi(coeff, with_hist=True))
    (s0, g0, n0, h0), (s1, g1, n1, h1) = out
    assert abs(n1 - n0) <= 1e-4 * n0 + 2
    assert abs(s1 - s0) <= 1e-5 * abs(s0)
    assert rel_err(g1, g0) < 1e-3
    assert rel_err(h1[2], h0[2]) < 1e-5


def test_parzen_rejects_too_few_bins():
    fixed, moving, grid, _ = _case()
    with pytest.raises(P.B200Error):
        P.Context(fixed, moving, grid, mi_bins=4, mi_window="parzen")
