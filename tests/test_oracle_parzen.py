"""The Parzen-window MI oracle (a restatement of Mattes et al., IEEE TMI
22(1) 2003; the reference has no Parzen flavour) checked against itself:
its analytic gradient against central differences of its score (double
precision; relative L2 below 1e-3 on seeded control points -- measured
1e-4, all of it from the few voxels whose sample crosses a trilinear cell
face between the two evaluations, where the score has a kink), and its
histograms against their defining sums."""
import numpy as np

import oracle as O
from conftest import rel_err
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid


def _case():
    fixed = synth.gaussian_blobs((24, 20, 18), seed=3)
    g0 = BsplineGrid.for_volume(fixed, 6)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.5, 4))
    moving = synth.intensity_remap(moving, 1.6, 3.0, 9)
    grid = BsplineGrid.for_volume(fixed, (5, 4, 4))
    coeff = synth.random_coeff(grid, 0.5, 5)
    return fixed, moving, grid, coeff


def test_parzen_gradient_is_the_derivative_of_the_score():
    fixed, moving, grid, coeff = _case()
    r = O.port_mi_parzen(grid, fixed, moving, coeff, bins=16)
    idx = synth.rng(8).choice(grid.num_coeff, 24, replace=False)
    fd = []
    for i in idx:
        cp, cm = coeff.copy(), coeff.copy()
        cp[i] += np.float32(1e-3)
        cm[i] -= np.float32(1e-3)
        h2 = float(cp[i]) - float(cm[i])
        fd.append((O.port_mi_parzen(grid, fixed, moving, cp, 16).score
                   - O.port_mi_parzen(grid, fixed, moving, cm, 16).score) / h2)
    assert rel_err(r.grad[idx], np.array(fd)) < 1e-3


def test_parzen_histograms_are_consistent():
    fixed, moving, grid, coeff = _case()
    r = O.port_mi_parzen(grid, fixed, moving, coeff, bins=16)
    # the cubic window is a partition of unity: one unit of weight per voxel
    assert abs(r.j_hist.sum() - r.num_vox) <= 1e-9 * r.num_vox
    assert np.allclose(r.f_hist, r.j_hist.sum(axis=1))
    # padding bins: the fixed box window never uses the outer two bins
    assert not r.j_hist[:2].any() and not r.j_hist[-2:].any()
    assert -np.log(16) <= r.score <= 0.0
