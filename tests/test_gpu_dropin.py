"""The drop-in exercised from the reference side.

oracle/ref/b200_adapter.cxx holds the two functions a Plastimatch
maintainer adds (bspline_b200_state_create at Bspline_state's device-state
hook, bspline_score_b200 as the new threading flavour), compiled against
the reference's own headers and linked with the reference build and
libplastimatch_b200.so.  Each case builds the reference's Bspline_xform /
Bspline_parms / Bspline_state / Metric_state as Bspline_optimize::optimize
does, scores it through the adapter and through the reference's own
bspline_score_mse / _mi dispatcher (CPU flavour), and compares the
Bspline_score fields they write (curr_smetric, curr_smetric_grad,
curr_num_vox) at the library's bars: score 1e-5 relative, gradient 1e-3
relative (L2), voxel count within 0.01 % (+2).
"""
import pytest

import oracle as O
from conftest import load_golden, load_rois, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.adapter_available(),
                                 reason="reference-side adapter not built")]


def _check(b, r):
    assert abs(b.num_vox - r.num_vox) <= 1e-4 * r.num_vox + 2, (b.num_vox, r.num_vox)
    assert abs(b.score - r.score) <= 1e-5 * abs(r.score), (b.score, r.score)
    assert rel_err(b.grad, r.grad) < 1e-3, rel_err(b.grad, r.grad)


@pytest.mark.parametrize("name", ["mse_small", "mse_roi", "mse_dcos",
                                  "mse_vpr8"])
def test_dropin_mse(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    b, r = O.adapter_compare(grid, fixed, moving, coeff, flavor="g")
    assert r.num_vox == rec["g_num_vox"]          # the reference's flavour g
    _check(b, r)


@pytest.mark.parametrize("name", ["mi_small", "mi_dcos", "mi_partial"])
def test_dropin_mi(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    b, r = O.adapter_compare(grid, fixed, moving, coeff, flavor="g",
                             metric="mi")
    _check(b, r)


def test_dropin_mi_vopt():
    fixed, moving, grid, coeff, rec = load_golden("vopt_mi_small")
    b, r = O.adapter_compare(grid, fixed, moving, coeff, flavor="g",
                             metric="mi", hist="vopt")
    _check(b, r)


@pytest.mark.parametrize("name,metric", [("roimask_mse_small", "mse"),
                                         ("roimask_mse_dcos", "mse"),
                                         ("roimask_mi_small", "mi")])
def test_dropin_with_rois(name, metric):
    """ROIs on the metric state: the reference dispatches to its ROI
    flavours (MSE i, MI h); the adapter forwards the same masks."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    fr, mr = load_rois(rec)
    b, r = O.adapter_compare(grid, fixed, moving, coeff, flavor="g",
                             metric=metric, fixed_roi=fr, moving_roi=mr)
    _check(b, r)
