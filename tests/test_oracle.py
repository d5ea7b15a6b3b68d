"""The oracle pinned against the reference's own outputs.

The golden vectors in tests/golden/ were produced by the reference's
compiled CPU flavours (tests/golden/make_golden.py).  The C restatement
keeps the reference's float operation order, so it must reproduce them bit
for bit; the double-precision restatement must agree to within float
rounding.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden_names, load_golden, rel_err


@pytest.mark.parametrize("name", golden_names("mse"))
def test_port_mse_g_bit_exact(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mse(grid, fixed, moving, coeff, moving_grad=rec["moving_grad"])
    assert np.float32(r.score) == rec["g_score"]
    assert r.num_vox == rec["g_num_vox"]
    np.testing.assert_array_equal(r.grad, rec["g_grad"])


@pytest.mark.parametrize("name", [n for n in golden_names("mse") if n != "mse_roi"])
def test_port_mse_o_bit_exact(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mse(grid, fixed, moving, coeff, grad_mode=1)
    assert np.float32(r.score) == rec["o_score"]
    np.testing.assert_array_equal(r.grad, rec["o_grad"])


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
@pytest.mark.parametrize("flavor", ["p", "q", "r"])
@pytest.mark.parametrize("name", [n for n in golden_names("mse") if n != "mse_roi"])
def test_reference_flavours_pqr_equal_o(name, flavor):
    """The reference's flavours p, q and r compute flavour o's MSE (the
    exact trilinear-derivative gradient) and differ from it only in the
    order of float sums: same voxel count, score within 1e-6 relative,
    gradient within 1e-5 relative (L2).  The restatement of o therefore
    checks all four."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.ref_metric(grid, fixed, moving, coeff, flavor=flavor)
    assert r.num_vox == rec["o_num_vox"]
    assert abs(r.score - rec["o_score"]) <= 1e-6 * abs(rec["o_score"])
    assert rel_err(r.grad, rec["o_grad"]) < 1e-5


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
@pytest.mark.parametrize("name", [n for n in golden_names("mse") if n != "mse_roi"])
def test_reference_flavour_k_equals_c(name):
    """MSE flavour k is flavour c bit for bit (same voxel-serial sums)."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.ref_metric(grid, fixed, moving, coeff, flavor="k")
    assert np.float32(r.score) == rec["c_score"]
    assert r.num_vox == rec["c_num_vox"]
    np.testing.assert_array_equal(r.grad, rec["c_grad"])


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
@pytest.mark.parametrize("name", [n for n in golden_names("mi")
                                  if n != "mi_partial"])
def test_reference_mi_flavours_equal_g(name):
    """The reference's MI flavours compute flavour g's PVI-8 MI: same score
    and voxel count, gradient within 1e-5 relative (L2), so the device's
    g semantics stand for them, when the grid's ROI is the whole image.
    Exception: d, e, f and i ignore the direction cosines and differ from g
    (and from the others) on rotated grids."""
    fixed, moving, grid, coeff, rec = load_golden(name)
    rotated = not np.allclose(np.asarray(fixed.dcos).reshape(3, 3), np.eye(3))
    for flavor in "cdefhikl":
        r = O.ref_metric(grid, fixed, moving, coeff, flavor=flavor,
                         metric="mi", bins=32)
        same = np.float32(r.score) == rec["mi_score"] \
            and r.num_vox == rec["mi_num_vox"] \
            and rel_err(r.grad, rec["mi_grad"]) < 1e-5
        assert same != (rotated and flavor in "defi"), flavor


@pytest.mark.parametrize("name", golden_names("mse"))
def test_port_mse_f64_close(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mse(grid, fixed, moving, coeff, moving_grad=rec["moving_grad"],
                   precision="f64")
    assert abs(r.score - rec["g_score"]) <= 1e-5 * abs(rec["g_score"])
    assert rel_err(r.grad, rec["g_grad"]) < 1e-4


@pytest.mark.parametrize("name", golden_names("mse"))
def test_port_volume_grad_bit_exact(name):
    _, moving, _, _, rec = load_golden(name)
    np.testing.assert_array_equal(O.port_volume_grad(moving), rec["moving_grad"])


@pytest.mark.parametrize("name", golden_names("mse"))
def test_port_regularizer_bit_exact(name):
    fixed, _, grid, coeff, rec = load_golden(name)
    r = O.port_reg(grid, fixed, coeff, O.penalties(curvature=0.005))
    assert np.float32(r.score) == rec["reg_score"]
    np.testing.assert_array_equal(r.grad, rec["reg_grad"])
    r64 = O.port_reg(grid, fixed, coeff, O.penalties(curvature=0.005),
                     precision="f64")
    assert abs(r64.score - rec["reg_score"]) <= 1e-6 * abs(rec["reg_score"])
    assert rel_err(r64.grad, rec["reg_grad"]) < 1e-6


@pytest.mark.parametrize("name", golden_names("mse"))
def test_total_score_is_metric_plus_regularizer(name):
    """bspline_score(): total = lambda*smetric + rmetric, grads likewise."""
    _, _, _, _, rec = load_golden(name)
    assert abs(float(rec["total_score"]) - (float(rec["g_score"])
               + float(rec["reg_score"]))) <= 1e-6 * abs(float(rec["total_score"]))
    np.testing.assert_allclose(rec["total_grad"], rec["g_grad"] + rec["reg_grad"],
                               rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("name", golden_names("mi"))
def test_port_mi_bit_exact(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mi(grid, fixed, moving, coeff, bins=32)
    np.testing.assert_array_equal(r.f_hist, rec["f_hist"])
    np.testing.assert_array_equal(r.m_hist, rec["m_hist"])
    np.testing.assert_array_equal(r.j_hist, rec["j_hist"])
    assert np.float32(r.score) == rec["mi_score"]
    assert r.num_vox == rec["mi_num_vox"]
    np.testing.assert_array_equal(r.grad, rec["mi_grad"])


@pytest.mark.parametrize("name", golden_names("mi"))
def test_port_mi_f64_close(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.port_mi(grid, fixed, moving, coeff, bins=32, precision="f64")
    assert abs(r.score - rec["mi_score"]) <= 1e-5 * abs(rec["mi_score"])
    assert rel_err(r.grad, rec["mi_grad"]) < 1e-3


@pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("name", golden_names("mse_small"))
def test_reference_reproduces_golden(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    r = O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                     moving_grad=rec["moving_grad"])
    np.testing.assert_array_equal(r.grad, rec["g_grad"])


WARP_GOLDEN = golden_names("warp") + golden_names("vf")


@pytest.mark.parametrize("name", WARP_GOLDEN)
def test_port_interpolate_vf_bit_exact(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    np.testing.assert_array_equal(O.port_interpolate_vf(grid, fixed, coeff),
                                  rec["vf"])


@pytest.mark.parametrize("name", golden_names("warp"))
def test_port_warp_bit_exact(name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    w, vf = O.port_warp(grid, fixed, moving, coeff, float(rec["default"]),
                        with_vf=True)
    np.testing.assert_array_equal(w, rec["warped"])
    np.testing.assert_array_equal(vf, rec["warp_vf"])
    # some voxels land outside the moving image and keep the default
    assert (w == rec["default"]).any() and (w != rec["default"]).any()


def test_port_warp_rejects_partial_roi():
    fixed, moving, grid, coeff, rec = load_golden("vf_roi")
    with pytest.raises(RuntimeError):
        O.port_warp(grid, fixed, moving, coeff)


def _resample_case(name):
    from plastimatch_b200.geometry import Volume
    import os
    from conftest import GOLDEN
    r = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    v = Volume(r["img"], origin=tuple(float(x) for x in r["origin"]),
               spacing=tuple(float(x) for x in r["spacing"]))
    return v, str(r["mode"]), tuple(float(x) for x in r["rate"]), r


@pytest.mark.parametrize("name", golden_names("resample"))
def test_port_resample_bit_exact(name):
    v, mode, rate, rec = _resample_case(name)
    out = O.port_resample(v, mode, rate)
    assert out.dim == tuple(int(x) for x in rec["out_dim"])
    np.testing.assert_array_equal(np.float32(out.origin), rec["out_origin"])
    np.testing.assert_array_equal(np.float32(out.spacing), rec["out_spacing"])
    np.testing.assert_array_equal(out.img, rec["out"])
