"""Multi-resolution registration driver over the library's entry points.

Plastimatch runs a registration as stages: each stage subsamples both
images (registration_resample_volume), lays a B-spline grid of a given
spacing in mm over the fixed image, carries the previous stage's transform
over to that grid and optimises.  This module strings the device pieces
together the same way -- pyramid levels by b200bsp_resample, one context per
level, the device L-BFGS -- with the stage-to-stage carry-over done here on
the host.

The carry-over is cubic B-spline interpolation: the previous field is
evaluated at the new grid's interior knots and new coefficients are solved
so that the new field passes through those values, with the two outer
knots of every axis continuing the next two linearly.  (Plastimatch does
this step through ITK's B-spline resampling; ITK is outside this library,
and interpolation at the knots is the same idea on the tensor grid.)
"""
from __future__ import annotations

import time

import numpy as np

from . import Context, pyramid_level
from .geometry import BsplineGrid, Volume

__all__ = ["refine_coefficients", "register_pyramid"]


def _basis(u):
    """The four cubic B-spline basis weights at local coordinate u."""
    return np.stack([(1 - u) ** 3 / 6.0,
                     (3 * u ** 3 - 6 * u ** 2 + 4) / 6.0,
                     (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6.0,
                     u ** 3 / 6.0], axis=-1)


def _eval_matrix(pos, n_old):
    """Rows: the old field along one axis at grid coordinates `pos` (in old
    grid spacings from the old ROI origin) as weights on the n_old knots;
    beyond the old tiles the end tile's polynomial continues."""
    rd = n_old - 3
    t = np.clip(np.floor(pos).astype(np.int64), 0, rd - 1)
    w = _basis(pos - t)
    m = np.zeros((len(pos), n_old))
    for i in range(4):
        np.add.at(m, (np.arange(len(pos)), t + i), w[:, i])
    return m


def _interp_system(n):
    """Cubic B-spline interpolation on knots 1..n-2 (values at the knot
    centres: (c[k-1] + 4 c[k] + c[k+1]) / 6) with linear continuation at
    both ends: c0 - 2 c1 + c2 = 0, c[n-1] - 2 c[n-2] + c[n-3] = 0."""
    a = np.zeros((n, n))
    for k in range(1, n - 1):
        a[k, k - 1:k + 2] = (1 / 6.0, 4 / 6.0, 1 / 6.0)
    a[0, 0:3] = (1.0, -2.0, 1.0)
    a[n - 1, n - 3:n] = (1.0, -2.0, 1.0)
    return a


def refine_coefficients(coeff_old, grid_old: BsplineGrid,
                        grid_new: BsplineGrid) -> np.ndarray:
    """Coefficients on grid_new whose field interpolates grid_old's field
    (coeff_old, xyz interleaved per knot) at grid_new's interior knots.
    Both grids must share their direction cosines."""
    if not np.allclose(grid_old.dcos, grid_new.dcos):
        raise ValueError("grids must share direction cosines")
    dc = np.asarray(grid_new.dcos, np.float64).reshape(3, 3)
    # ROI origins and knot spacing along the (rotated) grid axes
    def roi_origin(g):
        o = np.asarray(g.img_origin, np.float64)
        off = np.asarray(g.roi_offset, np.float64) * np.asarray(g.img_spacing)
        return o + dc @ off
    o_old, o_new = roi_origin(grid_old), roi_origin(grid_new)
    shift = dc.T @ (o_new - o_old)          # new ROI origin in the old frame
    ops = []
    for d in range(3):
        n_new, n_old = grid_new.cdims[d], grid_old.cdims[d]
        gs_new, gs_old = grid_new.grid_spac[d], grid_old.grid_spac[d]
        k = np.arange(1, n_new - 1)
        pos = (shift[d] + (k - 1) * gs_new) / gs_old
        rhs = np.zeros((n_new, n_old))
        rhs[1:n_new - 1] = _eval_matrix(pos, n_old)
        ops.append(np.linalg.solve(_interp_system(n_new), rhs))
    cx, cy, cz = grid_old.cdims
    c = np.asarray(coeff_old, np.float64).reshape(cz, cy, cx, 3)
    out = np.einsum("zc,yb,xa,cbad->zyxd", ops[2], ops[1], ops[0], c,
                    optimize=True)
    return out.astype(np.float32).ravel()


def register_pyramid(fixed: Volume, moving: Volume, levels=(4, 2, 1),
                     grid_mm=10.0, metric="mi", mi_window="parzen",
                     mi_bins=32, its=50, max_feval=None, form="tc",
                     mode="voxel", epsilon=0.0, device=0):
    """Register moving onto fixed through the subsampling levels (voxel
    factors, coarse to fine), a grid of `grid_mm` at every level, `its`
    L-BFGS iterations per level.  `epsilon` is liblbfgs's gradient test
    (|g| / max(1, |x|)); its default 1e-5 would stop an MI registration at
    once (MI gradients are small), so levels run their iterations unless a
    value is given.  Returns (coefficients, finest grid, one record per
    level: dims, vox_per_rgn, evaluations, status, first and last score,
    seconds)."""
    coeff, grid_prev, history = None, None, []
    for lv in levels:
        t0 = time.perf_counter()
        f = pyramid_level(fixed, mode, (lv, lv, lv), device=device)
        m = pyramid_level(moving, mode, (lv, lv, lv), device=device)
        grid = BsplineGrid.for_grid_spacing(f, grid_mm)
        x0 = (np.zeros(grid.num_coeff, np.float32) if coeff is None
              else refine_coefficients(coeff, grid_prev, grid))
        with Context(f, m, grid, form=form, mi_bins=mi_bins,
                     mi_window=mi_window, device=device) as ctx:
            ctx.set_images()
            s0 = (ctx.score_mi(x0) if metric == "mi" else ctx.score_mse(x0))[0]
            coeff, res = ctx.optimize_lbfgs(
                x0, metric=metric, max_its=its, epsilon=epsilon,
                max_feval=max_feval if max_feval else 2 * its + 10)
        history.append({"level": lv, "dim": list(f.dim),
                        "vox_per_rgn": list(grid.vox_per_rgn),
                        "fevals": res["fevals"], "status": res["status"],
                        "first_score": float(s0),
                        "last_score": float(res["score"]),
                        "seconds": time.perf_counter() - t0})
        grid_prev = grid
    return coeff, grid_prev, history
