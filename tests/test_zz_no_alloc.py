"""b200bsp_score_mse_static (no context, no allocation) against the context
entry point b200bsp_score_mse with the FP32 form.

Tolerances: score relative 1e-6, gradient relative 1e-6 (L2), num_vox
exact -- both entry points run the same kernels, so they agree far inside
these bars.  Each case makes two calls in a row on the shared static
scratch and checks both.
"""
import numpy as np
import pytest

import plastimatch_b200 as P
from conftest import load_golden, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _blob_case(shape, vpr, seed):
    fixed = synth.gaussian_blobs(shape, spacing=(1, 1, 1), seed=seed)
    g0 = BsplineGrid.for_volume(fixed, vpr)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, seed + 1))
    grid = BsplineGrid.for_volume(fixed, vpr)
    coeff = synth.random_coeff(grid, 1.0, seed + 2)
    return fixed, moving, grid, coeff


def _dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def _static_twice(fixed, moving, grid, coeff, mse_grad, mgrad):
    df, dm, dc = _dev(fixed.img), _dev(moving.img), _dev(coeff)
    dg = _dev(mgrad) if mgrad is not None else None
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for _ in range(2):
        grad = torch.full((grid.num_coeff,), float("nan"), device="cuda")
        score = torch.zeros(1, device="cuda")
        nvox = torch.zeros(1, dtype=torch.int64, device="cuda")
        P.score_mse_static(fixed, moving, grid, df, dm, dc, grad, score, nvox,
                           moving_grad=dg, mse_grad=mse_grad, stream=stream)
        out.append((grad, score, nvox))
    torch.cuda.synchronize()
    return [(float(s.item()), g.cpu().numpy(), int(n.item()))
            for g, s, n in out]


def _context(fixed, moving, grid, coeff, mse_grad, mgrad):
    with P.Context(fixed, moving, grid, form="fp32", mse_grad=mse_grad) as ctx:
        ctx.set_images(moving_grad=mgrad)
        return ctx.score_mse(coeff)


def _agree(static, ref):
    s0, g0, n0 = ref
    for s, g, n in static:
        assert n == n0
        assert abs(s - s0) <= 1e-6 * abs(s0), (s, s0)
        assert rel_err(g, g0) < 1e-6


@pytest.mark.parametrize("mse_grad", ["nearest", "trilinear"])
def test_static_matches_context_64cubed(mse_grad):
    fixed, moving, grid, coeff = _blob_case((64, 64, 64), 8, 31)
    mgrad = P.volume_grad(moving) if mse_grad == "nearest" else None
    ref = _context(fixed, moving, grid, coeff, mse_grad, mgrad)
    _agree(_static_twice(fixed, moving, grid, coeff, mse_grad, mgrad), ref)


def test_static_matches_context_golden_dcos_roi():
    for name in ("mse_dcos", "mse_roi"):
        fixed, moving, grid, coeff, rec = load_golden(name)
        mgrad = rec["moving_grad"]
        ref = _context(fixed, moving, grid, coeff, "nearest", mgrad)
        _agree(_static_twice(fixed, moving, grid, coeff, "nearest", mgrad),
               ref)


def test_static_near_the_tile_limit():
    # 128 x 128 x 96 with 6-voxel tiles: 22 * 22 * 16 = 7744 tiles
    fixed, moving, grid, coeff = _blob_case((128, 128, 96), 6, 77)
    assert grid.rdims[0] * grid.rdims[1] * grid.rdims[2] == 7744
    mgrad = P.volume_grad(moving)
    ref = _context(fixed, moving, grid, coeff, "nearest", mgrad)
    _agree(_static_twice(fixed, moving, grid, coeff, "nearest", mgrad), ref)


def test_static_allocates_nothing_after_first_call():
    fixed, moving, grid, coeff = _blob_case((48, 48, 48), 6, 5)
    df, dm, dc = _dev(fixed.img), _dev(moving.img), _dev(coeff)
    grad = torch.zeros(grid.num_coeff, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    P.score_mse_static(fixed, moving, grid, df, dm, dc, grad,
                       mse_grad="trilinear", stream=stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        P.score_mse_static(fixed, moving, grid, df, dm, dc, grad,
                           mse_grad="trilinear", stream=stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_rejects_oversized_grid_and_host_memory():
    fixed, moving, grid, coeff = _blob_case((100, 100, 100), 4, 3)
    assert grid.rdims[0] * grid.rdims[1] * grid.rdims[2] > 8192
    df, dm, dc = _dev(fixed.img), _dev(moving.img), _dev(coeff)
    grad = torch.zeros(grid.num_coeff, device="cuda")
    with pytest.raises(P.B200Error) as e:
        P.score_mse_static(fixed, moving, grid, df, dm, dc, grad,
                           mse_grad="trilinear")
    assert e.value.code == -6 and "8192" in str(e.value)
    small = BsplineGrid.for_volume(fixed, 10)
    host_grad = np.zeros(small.num_coeff, np.float32)
    with pytest.raises(P.B200Error) as e:
        P.score_mse_static(fixed, moving, small, df, dm,
                           _dev(np.zeros(small.num_coeff, np.float32)),
                           host_grad, mse_grad="trilinear")
    assert e.value.code == -1
