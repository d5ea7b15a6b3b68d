"""MSE score + gradient on the GPU against the oracle.

Tolerances (float work, stated here as the bar):
  score     relative 1e-5 against the double-precision oracle
  gradient  relative 1e-3 (L2 norm of the difference over the norm of the
            reference) against both the double oracle and the reference's
            float flavour g / o
  num_vox   within 0.01% (+2): a voxel whose moving position lies within
            float rounding of a cell edge or of the inside bound may land
            on the other side.
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid, Volume

pytestmark = pytest.mark.gpu

FORMS = ["fp32", "tc"]


def check(score, grad, nvox, f64, ref32, nv_ref):
    assert abs(nvox - nv_ref) <= 1e-4 * nv_ref + 2, (nvox, nv_ref)
    assert abs(score - f64.score) <= 1e-5 * abs(f64.score), (score, f64.score)
    assert rel_err(grad, f64.grad) < 1e-3, rel_err(grad, f64.grad)
    assert rel_err(grad, ref32) < 1e-3, rel_err(grad, ref32)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", golden_names("mse"))
def test_mse_golden(form, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        s, g, n = ctx.score_mse(coeff)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=rec["moving_grad"],
                     precision="f64")
    check(s, g, n, f64, rec["g_grad"], int(rec["g_num_vox"]))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", [n for n in golden_names("mse") if n != "mse_roi"])
def test_mse_trilinear_gradient_golden(form, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid, form=form, mse_grad="trilinear") as ctx:
        ctx.set_images()
        s, g, n = ctx.score_mse(coeff)
    f64 = O.port_mse(grid, fixed, moving, coeff, grad_mode=1, precision="f64")
    check(s, g, n, f64, rec["o_grad"], int(rec["o_num_vox"]))


def test_device_moving_gradient_matches_reference():
    for name in golden_names("mse"):
        _, moving, _, _, rec = load_golden(name)
        np.testing.assert_array_equal(P.volume_grad(moving), rec["moving_grad"])


def _c1_case(seed=20261204):
    fixed = synth.gaussian_blobs((64, 64, 64), spacing=(1, 1, 1), seed=seed)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0, synth.random_coeff(g0, 2.0, seed + 1))
    grid = BsplineGrid.for_volume(fixed, 8)
    coeff = synth.random_coeff(grid, 1.0, seed + 2)
    return fixed, moving, grid, coeff


@pytest.mark.parametrize("form", FORMS)
def test_mse_64cubed_vpr8(form):
    fixed, moving, grid, coeff = _c1_case()
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        s, g, n = ctx.score_mse(coeff)
        s2, g2, n2 = ctx.score_mse(coeff)
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg, precision="f64")
    r32 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    check(s, g, n, f64, r32.grad, r32.num_vox)
    # deterministic: fixed reduction order, no float atomics
    assert s == s2 and n == n2
    np.testing.assert_array_equal(g, g2)


@pytest.mark.parametrize("vpr", [(9, 9, 7), (10, 10, 10)])
def test_mse_large_tiles_tensor_core_form(vpr):
    # 567 and 1000 voxels per tile: five and eight 128-voxel blocks, the
    # tensor-core kernel's non-pipelined path (a 10 mm grid at 1 mm spacing)
    fixed, moving, _, _ = _c1_case(seed=23)
    grid = BsplineGrid.for_volume(fixed, vpr)
    coeff = synth.random_coeff(grid, 1.0, 24)
    with P.Context(fixed, moving, grid, form="tc") as ctx:
        ctx.set_images()
        s, g, n = ctx.score_mse(coeff)
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg, precision="f64")
    r32 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    check(s, g, n, f64, r32.grad, r32.num_vox)


@pytest.mark.parametrize("form", FORMS)
def test_mse_zero_coefficients_and_no_overlap(form):
    fixed, moving, grid, _ = _c1_case(seed=7)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        z = np.zeros(grid.num_coeff, np.float32)
        s, g, n = ctx.score_mse(z)
        assert n == fixed.npix
        # push every voxel outside the moving image: reference returns
        # FLT_MAX and a zero gradient
        far = np.full(grid.num_coeff, 1e4, np.float32)
        s, g, n = ctx.score_mse(far)
        assert n == 0 and s == np.finfo(np.float32).max
        assert not g.any()


@pytest.mark.parametrize("form", FORMS)
def test_mse_device_pointers_are_stream_ordered(form):
    torch = pytest.importorskip("torch")
    fixed, moving, grid, coeff = _c1_case(seed=11)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        ctx.set_images()
        s_h, g_h, n_h = ctx.score_mse(coeff)
        dc = torch.from_numpy(coeff).cuda()
        gd = torch.zeros(grid.num_coeff, device="cuda")
        sd = torch.zeros(1, device="cuda")
        nd = torch.zeros(1, dtype=torch.int64, device="cuda")
        ctx.score_mse(dc, grad_out=gd, score_out=sd, nvox_out=nd)
        torch.cuda.synchronize()
        assert float(sd.item()) == s_h and int(nd.item()) == n_h
        np.testing.assert_array_equal(gd.cpu().numpy(), g_h)


@pytest.mark.parametrize("form", FORMS)
def test_mse_page_locked_host_outputs(form):
    """Page-locked (mapped) host buffers are written in place by the device;
    the results equal those through pageable buffers, float and double."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    fixed, moving, grid, coeff = _c1_case(seed=12)
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        s_h, g_h, n_h = ctx.score_mse(coeff)
        hc = torch.from_numpy(coeff).pin_memory()
        for dtype, fn in ((torch.float32, P.lib().b200bsp_score_mse),
                          (torch.float64, P.lib().b200bsp_score_mse_f64)):
            hg = torch.full((grid.num_coeff,), 7.0, dtype=dtype).pin_memory()
            sc = C.c_float() if dtype == torch.float32 else C.c_double()
            nv = C.c_int64()
            P._check(fn(ctx._h, hc.data_ptr(), C.addressof(sc), hg.data_ptr(),
                        C.addressof(nv)), ctx._h)
            assert nv.value == n_h
            if dtype == torch.float32:
                assert sc.value == s_h
                np.testing.assert_array_equal(hg.numpy(), g_h)
            else:
                s64, g64, n64 = ctx.score_mse_f64(coeff)
                assert sc.value == s64
                np.testing.assert_array_equal(hg.numpy(), g64)


@pytest.mark.parametrize("shape,vpr", [((96, 80, 48), (5, 5, 5)),
                                       ((200, 64, 40), (4, 4, 4))])
def test_autotune_keeps_parity(shape, vpr):
    """The autotuner's batch split changes only how tiles are grouped: the
    results stay within the bars, repeat exactly, and the chosen split is
    one the kernel supports (at least 3 tiles per batch)."""
    fixed = synth.gaussian_blobs(shape, spacing=(1.0, 1.0, 2.0), seed=41)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.5, 42))
    grid = BsplineGrid.for_volume(fixed, vpr)
    coeff = synth.random_coeff(grid, 1.0, 43)
    with P.Context(fixed, moving, grid, form="tc") as ctx:
        ctx.set_images()
        t = ctx.autotune(coeff, evals=2)
        s, g, n = ctx.score_mse(coeff)
        s2, g2, n2 = ctx.score_mse(coeff)
    assert 3 <= t <= 26
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg, precision="f64")
    r32 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    check(s, g, n, f64, r32.grad, r32.num_vox)
    assert s == s2 and n == n2
    np.testing.assert_array_equal(g, g2)
