"""Image ROIs (uchar fixed / moving masks) in the oracle, pinned to the
reference's ROI flavours.

The roimask_* golden cases hold a fixed ROI built from an intensity window
and a moving ROI on its own coarser, shifted grid, with the compiled
reference's outputs for the fixed ROI alone (tag f), the moving ROI alone
(m) and both (fm): MSE flavour i (chosen by the reference's dispatcher for
'g' when ROIs are set) and k (for 'c'), MI flavour h.  The C restatement
must reproduce them bit for bit; the double-precision one within float
rounding (score 1e-5, gradient 1e-3, the device bars).
"""
import numpy as np
import pytest

import oracle as O
from conftest import (ROI_TAGS, golden_names, load_golden, load_rois,
                      pick_rois, rel_err)


@pytest.mark.parametrize("tag", ROI_TAGS)
@pytest.mark.parametrize("name", golden_names("roimask_mse"))
def test_port_mse_roi_bit_exact(name, tag):
    fixed, moving, grid, coeff, rec = load_golden(name)
    fr, mr = pick_rois(tag, *load_rois(rec))
    r = O.port_mse(grid, fixed, moving, coeff, moving_grad=rec["moving_grad"],
                   fixed_roi=fr, moving_roi=mr)
    assert np.float32(r.score) == rec[f"{tag}_g_score"]
    assert r.num_vox == rec[f"{tag}_g_num_vox"]
    np.testing.assert_array_equal(r.grad, rec[f"{tag}_g_grad"])
    r64 = O.port_mse(grid, fixed, moving, coeff,
                     moving_grad=rec["moving_grad"], fixed_roi=fr,
                     moving_roi=mr, precision="f64")
    assert abs(r64.num_vox - r.num_vox) <= 2
    assert abs(r64.score - r.score) <= 1e-5 * abs(r.score)
    assert rel_err(r64.grad, r.grad) < 1e-3


@pytest.mark.parametrize("tag", ROI_TAGS)
@pytest.mark.parametrize("name", [n for n in golden_names("roimask_mse")
                                  if "dcos" not in n])
def test_reference_roi_flavour_k_matches_i(name, tag):
    """With ROIs the reference's 'c' runs flavour k, its voxel-serial form:
    same voxels as flavour i, sums in another order.  (Not on rotated
    grids: k accumulates world positions along x (LOOP_X) where i computes
    them from the index, and inside_roi floors projections that land on
    integers, so the rounding picks other neighbours there.)"""
    fixed, moving, grid, coeff, rec = load_golden(name)
    if f"{tag}_c_score" not in rec:
        pytest.skip("flavour k needs the grid to cover the image")
    assert rec[f"{tag}_c_num_vox"] == rec[f"{tag}_g_num_vox"]
    assert abs(rec[f"{tag}_c_score"] - rec[f"{tag}_g_score"]) \
        <= 1e-6 * abs(rec[f"{tag}_g_score"])
    assert rel_err(rec[f"{tag}_c_grad"], rec[f"{tag}_g_grad"]) < 1e-5


@pytest.mark.parametrize("tag", ROI_TAGS)
@pytest.mark.parametrize("name", golden_names("roimask_mi"))
def test_port_mi_roi_bit_exact(name, tag):
    fixed, moving, grid, coeff, rec = load_golden(name)
    fr, mr = pick_rois(tag, *load_rois(rec))
    r = O.port_mi(grid, fixed, moving, coeff, bins=32, fixed_roi=fr,
                  moving_roi=mr)
    assert np.float32(r.score) == rec[f"{tag}_mi_score"]
    assert r.num_vox == rec[f"{tag}_mi_num_vox"]
    np.testing.assert_array_equal(r.j_hist, rec[f"{tag}_j_hist"])
    np.testing.assert_array_equal(r.grad, rec[f"{tag}_mi_grad"])
    r64 = O.port_mi(grid, fixed, moving, coeff, bins=32, fixed_roi=fr,
                    moving_roi=mr, precision="f64")
    assert abs(r64.score - r.score) <= 1e-5 * abs(r.score)
    assert rel_err(r64.grad, r.grad) < 1e-3


def test_rois_change_the_voxel_set():
    """The fixture's ROIs are not trivial: each removes voxels."""
    for name in golden_names("roimask"):
        rec = load_golden(name)[4]
        key = "g" if name.startswith("roimask_mse") else "mi"
        n_f = rec[f"f_{key}_num_vox"]
        n_m = rec[f"m_{key}_num_vox"]
        n_fm = rec[f"fm_{key}_num_vox"]
        assert n_fm < min(n_f, n_m), (name, n_f, n_m, n_fm)


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
def test_reference_roi_entry_reproduces_golden():
    fixed, moving, grid, coeff, rec = load_golden("roimask_mse_small")
    fr, mr = load_rois(rec)
    r = O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                     moving_grad=rec["moving_grad"], fixed_roi=fr,
                     moving_roi=mr)
    np.testing.assert_array_equal(r.grad, rec["fm_g_grad"])


@pytest.mark.parametrize("name", golden_names("vopt_mi"))
def test_port_mi_vopt_bit_exact(name):
    """V-optimal bins (Bspline_parms::mi_hist_type = HIST_VOPT): the
    restated dynamic programme and key lookup reproduce the reference's MI
    flavour g bit for bit; the double restatement within float rounding."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mi(grid, fixed, moving, coeff, bins=32, hist="vopt")
    assert np.float32(r.score) == rec["mi_score"]
    assert r.num_vox == rec["mi_num_vox"]
    np.testing.assert_array_equal(r.f_hist, rec["f_hist"])
    np.testing.assert_array_equal(r.m_hist, rec["m_hist"])
    np.testing.assert_array_equal(r.j_hist, rec["j_hist"])
    np.testing.assert_array_equal(r.grad, rec["mi_grad"])
    r64 = O.port_mi(grid, fixed, moving, coeff, bins=32, hist="vopt",
                    precision="f64")
    assert abs(r64.score - r.score) <= 1e-5 * abs(r.score)
    assert rel_err(r64.grad, r.grad) < 1e-3
    # the bins differ from equal spacing on these images
    e = O.port_mi(grid, fixed, moving, coeff, bins=32)
    assert not np.array_equal(e.j_hist, r.j_hist)
