"""Batched registrations: contexts of uneven sizes and grids evaluated by one
graph launch, and L-BFGS registrations advancing together.

Bar: bit-identical to the same contexts run one at a time (the tile passes
do the same arithmetic whatever share of the SMs they get; the score and
gradient partial sums are per tile batch, so their order does not depend on
the grid), and so are whole L-BFGS runs (iterations, evaluations, status,
final coefficients and score).
"""
import numpy as np
import pytest

import plastimatch_b200 as P
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

pytestmark = pytest.mark.gpu

FORMS = ["fp32", "tc"]

# (dims, spacing, vox_per_rgn): axis-aligned tiles of <= 128 voxels, one of
# 512 voxels (the tensor-core form's non-pipelined path), a trilinear one
SHAPES = [((40, 36, 30), (1.2, 1.0, 2.0), (5, 5, 5)),
          ((48, 40, 36), (1.0, 1.0, 1.5), (6, 5, 4)),
          ((32, 32, 32), (1.0, 1.0, 1.0), (8, 8, 8)),
          ((56, 48, 40), (1.5, 1.5, 2.5), (4, 4, 4))]


def registrations(seed=31):
    out = []
    for k, (dim, sp, vpr) in enumerate(SHAPES):
        fixed = synth.gaussian_blobs(dim, spacing=sp, seed=seed + 10 * k)
        g0 = BsplineGrid.for_volume(fixed, 8)
        moving = synth.warp_trilinear(fixed, fixed, g0,
                                      synth.random_coeff(g0, 1.5,
                                                         seed + 10 * k + 1))
        grid = BsplineGrid.for_volume(fixed, vpr)
        coeff = synth.random_coeff(grid, 0.5, seed + 10 * k + 2)
        out.append((fixed, moving, grid, coeff))
    return out


def open_contexts(regs, form):
    ctxs = []
    for k, (fixed, moving, grid, _) in enumerate(regs):
        mode = "trilinear" if k == 3 else "nearest"
        ctxs.append(P.Context(fixed, moving, grid, form=form,
                              mse_grad=mode).set_images())
    return ctxs


@pytest.mark.parametrize("form", FORMS)
def test_batch_evaluation_equals_single_contexts(form):
    torch = pytest.importorskip("torch")
    regs = registrations()
    ctxs = open_contexts(regs, form)
    try:
        single = [c.score_mse(r[3]) for c, r in zip(ctxs, regs)]
        with P.Batch(ctxs) as b:
            coeffs = [torch.from_numpy(r[3]).cuda() for r in regs]
            grads = [torch.zeros(c.num_coeff, device="cuda") for c in ctxs]
            scores = torch.zeros(len(ctxs), device="cuda")
            nvox = torch.zeros(len(ctxs), dtype=torch.int64, device="cuda")
            for _ in range(2):      # capture, then replay
                grads[0].fill_(7.0)
                b.score_mse(coeffs, grads, scores, nvox)
                for k, (s, g, n) in enumerate(single):
                    assert float(scores[k]) == s
                    assert int(nvox[k]) == n
                    np.testing.assert_array_equal(grads[k].cpu().numpy(), g)
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("form", FORMS)
def test_batched_lbfgs_equals_single_registrations(form):
    regs = registrations(seed=57)
    parms = dict(max_its=5, max_feval=20)
    ref = []
    ctxs = open_contexts(regs, form)
    try:
        for c, r in zip(ctxs, regs):
            ref.append(c.optimize_lbfgs(r[3].copy(), **parms))
        coeffs = [r[3].copy() for r in regs]
        with P.Batch(ctxs) as b:
            res = b.optimize_lbfgs(coeffs, **parms)
        for (x1, r1), x2, r2 in zip(ref, coeffs, res):
            assert r2["iterations"] == r1["iterations"]
            assert r2["fevals"] == r1["fevals"]
            assert r2["status"] == r1["status"]
            assert r2["score"] == r1["score"]
            np.testing.assert_array_equal(x2, x1)
    finally:
        for c in ctxs:
            c.close()


def test_batch_rejects_bad_arguments():
    regs = registrations()[:1]
    ctxs = open_contexts(regs, "tc")
    try:
        with pytest.raises(P.B200Error):
            P.Batch([ctxs[0], ctxs[0]])
        with P.Batch(ctxs) as b:
            with pytest.raises(P.B200Error) as e:
                # host buffers are refused: batch buffers live on the device
                b.score_mse([regs[0][3]], [np.zeros(ctxs[0].num_coeff,
                                                    np.float32)],
                            np.zeros(1, np.float32))
            assert e.value.code == -1
    finally:
        for c in ctxs:
            c.close()
