"""Failure detection without a GPU fault.

* A bounded device-side wait that runs out: the x-lane tensor-core
  kernel's tensor-core warp withholds its MMAs (b200bsp_set_wait_limit's
  testing aid, refused on a context on the tile kernel), so the compute warps' first wait -- on a barrier nothing completes
  -- gives up after a short poll limit.  The call returns
  B200BSP_E_TIMEOUT, the kernel has released its TMEM (the next
  evaluation's allocation succeeds) and the same context then scores
  exactly as before.
* An allocation failure at create, injected on the host
  (b200bsp_debug_fail_alloc): B200BSP_E_OOM, and everything allocated
  before it is released again.
* Non-finite coefficients: the voxels whose displacement is not finite
  fail the inside test and drop out; the call succeeds with a finite score
  and gradient.  (The reference's is_inside lets NaN through and then
  reads outside its image; a defined result is the library's choice.)  The
  FP32 form loses the knot's 64 tiles; the tensor-core form's x contraction
  is one dense product per row of tiles, whose zeros off the band times a
  NaN are NaN, so it loses every row of tiles that holds the knot.
"""
import ctypes as C

import numpy as np
import pytest

import plastimatch_b200 as P
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

E_OOM, E_TIMEOUT, E_UNSUPPORTED = -2, -4, -6


def _case(seed=5):
    fixed = synth.gaussian_blobs((48, 40, 32), spacing=(1.0, 1.1, 1.3),
                                 seed=seed)
    g0 = BsplineGrid.for_volume(fixed, (8, 7, 6))
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, seed + 1))
    grid = BsplineGrid.for_volume(fixed, 5)
    return fixed, moving, grid, synth.random_coeff(grid, 1.5, seed + 2)


def _score(ctx, coeff):
    s = C.c_float()
    n = C.c_int64()
    g = np.zeros(ctx.num_coeff, np.float32)
    rc = P.lib().b200bsp_score_mse(ctx._h, coeff.ctypes.data, C.addressof(s),
                                   g.ctypes.data, C.addressof(n))
    return rc, s.value, g, n.value


def test_withholding_mmas_needs_the_xlane_kernel():
    fixed, moving, grid, coeff = _case()
    with P.Context(fixed, moving, grid, form="tc", tc_kernel="tile") as ctx:
        ctx.set_images()
        lib = P.lib()
        assert lib.b200bsp_set_wait_limit(ctx._h, 1000, 1) == E_UNSUPPORTED
        rc, s0, g0, n0 = _score(ctx, coeff)        # nothing was withheld
        assert rc == 0 and n0 > 0


def test_optimiser_reports_wait_expiry_and_context_recovers():
    """A registration whose evaluations give up (MMAs withheld) ends with
    B200BSP_E_TIMEOUT, not with a result; with the default limit restored
    the same context registers exactly as a fresh one does."""
    fixed, moving, grid, coeff = _case()
    x0 = np.zeros(grid.num_coeff, np.float32)
    with P.Context(fixed, moving, grid, form="tc", tc_kernel="xlane") as ctx:
        ctx.set_images()
        c0, r0 = ctx.optimize_lbfgs(x0, max_its=5, max_feval=10)
        lib = P.lib()
        assert lib.b200bsp_set_wait_limit(ctx._h, 1000, 1) == 0
        with pytest.raises(P.B200Error) as ei:
            ctx.optimize_lbfgs(x0, max_its=5, max_feval=10)
        assert ei.value.code == E_TIMEOUT
        assert lib.b200bsp_set_wait_limit(ctx._h, 0, 0) == 0
        c1, r1 = ctx.optimize_lbfgs(x0, max_its=5, max_feval=10)
    assert r1["fevals"] == r0["fevals"] and r1["score"] == r0["score"]
    assert np.array_equal(c1, c0)


def test_wait_expiry_times_out_and_context_recovers():
    fixed, moving, grid, coeff = _case()
    # withholding the MMAs is the x-lane kernel's testing aid
    with P.Context(fixed, moving, grid, form="tc", tc_kernel="xlane") as ctx:
        ctx.set_images()
        rc, s0, g0, n0 = _score(ctx, coeff)
        assert rc == 0
        lib = P.lib()
        for _ in range(2):
            assert lib.b200bsp_set_wait_limit(ctx._h, 1000, 1) == 0
            rc, _, _, _ = _score(ctx, coeff)
            assert rc == E_TIMEOUT
            assert b"gave up" in lib.b200bsp_last_error(ctx._h)
            assert lib.b200bsp_set_wait_limit(ctx._h, 0, 0) == 0
            rc, s1, g1, n1 = _score(ctx, coeff)
            assert rc == 0
            assert s1 == s0 and n1 == n0 and np.array_equal(g1, g0)


def test_wait_limit_option_rejects_negative():
    fixed, moving, grid, _ = _case()
    with pytest.raises(P.B200Error):
        P.Context(fixed, moving, grid, wait_limit=-1)


def test_allocation_failure_at_create_releases_everything():
    import torch
    torch.cuda.init()
    fixed, moving, grid, _ = _case()
    lib = P.lib()
    with P.Context(fixed, moving, grid) as warm:   # CUDA context, kernels loaded
        warm.set_images()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for nth in (1, 3, 6, 9):
        lib.b200bsp_debug_fail_alloc(nth)
        with pytest.raises(P.B200Error) as e:
            P.Context(fixed, moving, grid)
        assert e.value.code == E_OOM
        assert "injected" in str(e.value)
    lib.b200bsp_debug_fail_alloc(0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free1 - free0) <= 8 << 20, (free0, free1)
    with P.Context(fixed, moving, grid) as ctx:      # and creation works again
        ctx.set_images()


@pytest.mark.parametrize("form", ["tc", "fp32"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_coefficient_drops_its_voxels(form, bad):
    fixed, moving, grid, coeff = _case()
    with P.Context(fixed, moving, grid, form=form) as ctx:
        ctx.set_images()
        s0, g0, n0 = ctx.score_mse(coeff)
        c = coeff.copy()
        k = (grid.cdims[2] // 2 * grid.cdims[1] + grid.cdims[1] // 2) \
            * grid.cdims[0] + grid.cdims[0] // 2
        c[3 * k] = bad
        s, g, n = ctx.score_mse(c)
    assert np.isfinite(s) and np.all(np.isfinite(g))
    # the knot's 64 tiles of 125 voxels drop out (FP32 form), or the 16
    # rows of tiles along x through them (tensor-core form)
    limit = 64 * 125 if form == "fp32" else 16 * grid.rdims[0] * 125
    assert 0 < n0 - n <= limit, (n0 - n, limit)
