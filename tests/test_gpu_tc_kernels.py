"""The tensor-core form's two MSE kernels pinned one at a time
(b200bsp_opts.tc_kernel): the x-lane kernel (voxel x on the TMEM lanes) and
the tile kernel (one tile's 125 voxels on the lanes) each meet the MSE
bars on the golden cases and on the benchmark workload, whatever batch
split the autotuner picks; b200bsp_mse_kernel reports the kernel that
runs.

Bars as for the MSE evaluations: score relative 1e-5 against the double
oracle, gradient relative 1e-3 (L2) against the double oracle and the
reference's float flavour g, num_vox within 0.01 % (+2).
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden, load_rois, rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

KERNELS = ["xlane", "tile"]


def _check(s, g, n, f64, ref_grad, nv_ref):
    assert abs(n - nv_ref) <= 1e-4 * nv_ref + 2, (n, nv_ref)
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score), (s, f64.score)
    assert rel_err(g, f64.grad) < 1e-3, rel_err(g, f64.grad)
    assert rel_err(g, ref_grad) < 1e-3, rel_err(g, ref_grad)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", golden_names("mse"))
def test_pinned_kernel_golden(kernel, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    with P.Context(fixed, moving, grid, tc_kernel=kernel) as ctx:
        ctx.set_images(moving_grad=rec["moving_grad"])
        assert ctx.mse_kernel()[0] == kernel
        s, g, n = ctx.score_mse(coeff)
        ctx.autotune(coeff, evals=1)
        assert ctx.mse_kernel()[0] == kernel         # tuning stays pinned
        s2, g2, n2 = ctx.score_mse(coeff)
    f64 = O.port_mse(grid, fixed, moving, coeff,
                     moving_grad=rec["moving_grad"], precision="f64")
    for a in ((s, g, n), (s2, g2, n2)):
        _check(*a, f64, rec["g_grad"], int(rec["g_num_vox"]))


@pytest.mark.parametrize("kernel", KERNELS)
def test_pinned_kernel_headline_workload(kernel):
    import bench
    fixed, moving, grid, coeff = bench.make_workload()
    with P.Context(fixed, moving, grid, tc_kernel=kernel) as ctx:
        ctx.set_images()
        ctx.autotune(coeff, evals=2)
        name, tiles, batches = ctx.mse_kernel()
        s, g, n = ctx.score_mse(coeff)
    assert name == kernel and tiles >= 1 and batches >= 1
    mg = O.port_volume_grad(moving)
    f64 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg,
                     precision="f64")
    r32 = O.port_mse(grid, fixed, moving, coeff, moving_grad=mg)
    assert abs(n - r32.num_vox) <= 1e-4 * r32.num_vox + 2
    assert abs(s - f64.score) <= 1e-5 * abs(f64.score)
    assert rel_err(g, r32.grad) < 1e-3, rel_err(g, r32.grad)
    assert rel_err(g, f64.grad) <= rel_err(r32.grad, f64.grad) + 1e-4


def test_kernel_choice_errors():
    fixed, moving, grid, coeff, rec = load_golden("roimask_mse_small")
    fr, mr = load_rois(rec)
    with P.Context(fixed, moving, grid, tc_kernel="tile") as ctx:
        ctx.set_images()
        with pytest.raises(P.B200Error) as e:
            ctx.set_roi(fr, mr)                  # no ROI tests in the tile kernel
        assert e.value.code == -6                # B200BSP_E_UNSUPPORTED
    with P.Context(fixed, moving, grid, form="fp32") as ctx:
        assert ctx.mse_kernel()[0] == "fp32"
    # vox_per_rgn[1] = 12 is outside the x-lane kernel's 3..10
    f = synth.gaussian_blobs((40, 48, 24), spacing=(1, 1, 1), seed=3)
    g12 = BsplineGrid.for_volume(f, (5, 12, 5))
    with pytest.raises(P.B200Error) as e:
        P.Context(f, f, g12, tc_kernel="xlane")
    assert e.value.code == -6
    with P.Context(f, f, g12) as ctx:            # auto: the tile kernel
        assert ctx.mse_kernel()[0] == "tile"
