"""The multi-resolution driver's host logic: carrying a transform from one
level's B-spline grid to the next (interpolation at the new knots).

An affine displacement field is reproduced exactly by cubic B-splines, so
carried from a coarse grid to a finer, shifted one it must come out the
same at every voxel (up to float rounding); a general field must agree at
the new grid's interior knots, where it is interpolated."""
import numpy as np

import oracle as O
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid, Volume
from plastimatch_b200.pipeline import refine_coefficients


def _affine_coeff(grid, a, b):
    """Coefficients of the field d(x) = A x + b: a cubic B-spline
    reproduces linear functions with coefficients equal to the function at
    each knot's centre (knot k of an axis sits at p = k - 1 spacings from
    the ROI origin)."""
    cx, cy, cz = grid.cdims
    o = np.asarray(grid.img_origin) + np.asarray(grid.roi_offset) * np.asarray(grid.img_spacing)
    gs = np.asarray(grid.grid_spac)
    k = np.stack(np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx),
                             indexing="ij"), axis=-1)[..., ::-1]
    x = o + (k - 1) * gs
    return (x @ a.T + b).astype(np.float32).ravel()


def test_affine_field_is_carried_exactly():
    coarse = Volume(np.zeros((10, 12, 14), np.float32), origin=(-3.0, 2.0, 1.0),
                    spacing=(4.0, 4.0, 5.0))
    fine = Volume(np.zeros((40, 48, 56), np.float32), origin=(-4.5, 0.5, -1.0),
                  spacing=(1.0, 1.0, 1.25))
    g0 = BsplineGrid.for_volume(coarse, (4, 4, 4))
    g1 = BsplineGrid.for_volume(fine, (7, 6, 5))
    a = np.array([[0.01, -0.02, 0.005], [0.0, 0.015, -0.01],
                  [0.02, 0.0, -0.005]])
    b = np.array([1.5, -0.75, 0.25])
    c1 = refine_coefficients(_affine_coeff(g0, a, b), g0, g1)
    np.testing.assert_allclose(c1, _affine_coeff(g1, a, b), atol=2e-5)
    vf = O.port_interpolate_vf(g1, fine, c1).reshape(-1, 3)
    nx, ny, nz = fine.dim
    k = np.stack(np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx),
                             indexing="ij"), axis=-1)[..., ::-1].reshape(-1, 3)
    x = np.asarray(fine.origin) + k * np.asarray(fine.spacing)
    np.testing.assert_allclose(vf, x @ a.T + b, atol=1e-4)


def test_general_field_matches_at_interior_knots():
    vol = synth.gaussian_blobs((40, 36, 30), spacing=(1.0, 1.0, 1.5), seed=2)
    g0 = BsplineGrid.for_volume(vol, (10, 9, 6))
    g1 = BsplineGrid.for_volume(vol, (5, 4, 3))
    c0 = synth.random_coeff(g0, 2.0, 3)
    c1 = refine_coefficients(c0, g0, g1)
    vf0 = O.port_interpolate_vf(g0, vol, c0).reshape(30, 36, 40, 3)
    vf1 = O.port_interpolate_vf(g1, vol, c1).reshape(30, 36, 40, 3)
    # interior knots of g1 fall on voxels k * vox_per_rgn (from the origin)
    zs = np.arange(0, 30, 3)
    ys = np.arange(0, 36, 4)
    xs = np.arange(0, 40, 5)
    sel = np.ix_(zs, ys, xs)
    np.testing.assert_allclose(vf1[sel], vf0[sel], atol=1e-4)
    # and the two fields stay close in between
    assert np.abs(vf1 - vf0).max() < 0.1 * np.abs(vf0).max()
