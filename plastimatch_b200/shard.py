"""Multi-GPU forms of the MSE and Mattes MI cost functions.

Replicas (independent registrations, one per GPU) need nothing from this
module: each process creates its own Context.

Z-slabs split ONE volume's tile grid along z across the ranks of a process
group.  A slab of whole tiles [tz0, tz1) is the same computation as the
reference's tile loop (src/register/bspline_mse.cxx:519-720) restricted to
those tiles: a grid whose ROI is the slab has the same tiles, the same basis
tables and the same voxel positions (positions come from the fixed image's
origin, not the ROI's), and its knots are the global knot planes
tz0 .. tz1 + 2.  Each rank therefore evaluates its slab with an ordinary
context, and one all-reduce of the raw sums -- sum of diff^2, the voxel
count and the unnormalised gradient, in double precision -- gives the global
result, normalised afterwards as bspline_score_normalize (:43-72) does.

Mattes MI needs the whole volume's histograms before its gradient pass, so
a slab evaluation is two calls around two all-reduces: pass 1 on every slab
(b200bsp_mi_hist: exact integer histograms), one all-reduce of the
histograms (the sum is the whole ROI's, bit for bit), pass 2 on every slab
with the summed histograms (b200bsp_mi_grad: the score and the slab's part
of the gradient), one all-reduce of the gradient.

No tensor-core work crosses GPUs and no GPU reads another's memory; the only
exchanges are the all-reduces (NCCL over NVLink on GPUs, gloo on CPU).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from .geometry import BsplineGrid, Volume

FLT_MAX = float(np.finfo(np.float32).max)


@dataclass(frozen=True)
class Slab:
    """Tiles [tz0, tz1) of the global grid along z (empty when equal)."""
    rank: int
    tz0: int
    tz1: int

    @property
    def empty(self) -> bool:
        return self.tz1 <= self.tz0


def plan_slabs(grid: BsplineGrid, world: int) -> list[Slab]:
    """Split the grid's z tiles into `world` contiguous slabs, sizes
    differing by at most one tile (ranks beyond the tile count get none)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    nz = grid.rdims[2]
    base, extra = divmod(nz, world)
    out, t = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append(Slab(r, t, t + n))
        t += n
    return out


def slab_grid(grid: BsplineGrid, slab: Slab) -> BsplineGrid:
    """The grid over the slab: same x/y ROI, z ROI cut to the slab's tiles."""
    if slab.empty:
        raise ValueError("empty slab has no grid")
    vz = grid.vox_per_rgn[2]
    z0 = grid.roi_offset[2] + slab.tz0 * vz
    z1 = grid.roi_offset[2] + min(slab.tz1 * vz, grid.roi_dim[2])
    g = BsplineGrid(grid.img_origin, grid.img_spacing, grid.img_dim,
                    (grid.roi_offset[0], grid.roi_offset[1], z0),
                    (grid.roi_dim[0], grid.roi_dim[1], z1 - z0),
                    grid.vox_per_rgn, grid.dcos)
    assert g.rdims[2] == slab.tz1 - slab.tz0
    return g


def slab_coeff(grid: BsplineGrid, slab: Slab, coeff: np.ndarray) -> np.ndarray:
    """The slab's coefficients: global knot planes tz0 .. tz1 + 2."""
    cx, cy, cz = grid.cdims
    c = np.asarray(coeff).reshape(cz, cy, cx, 3)
    return np.ascontiguousarray(c[slab.tz0:slab.tz1 + 3]).reshape(-1)


def scatter_grad(grid: BsplineGrid, slab: Slab, local: np.ndarray,
                 out: np.ndarray) -> np.ndarray:
    """Add a slab's gradient into the global gradient vector `out`."""
    cx, cy, cz = grid.cdims
    o = out.reshape(cz, cy, cx, 3)
    o[slab.tz0:slab.tz1 + 3] += np.asarray(local).reshape(-1, cy, cx, 3)
    return out


# An evaluator returns the slab's raw sums: (sum of diff^2, unnormalised
# gradient sum_v dc/dv * basis as float64, voxel count).
Evaluator = Callable[[BsplineGrid, np.ndarray], tuple]


def context_evaluator(fixed: Volume, moving: Volume, form: str = "tc",
                      mse_grad: str = "nearest", device: int = 0,
                      moving_grad: Optional[np.ndarray] = None) -> Evaluator:
    """Evaluate slabs on the GPU through a Context per slab grid (created on
    first use and kept).  The context's double-precision outputs are
    normalised; the raw sums are recovered as score * N and grad * N / 2."""
    from . import Context
    cache = {}

    def run(g: BsplineGrid, coeff: np.ndarray):
        key = (g.roi_offset, g.roi_dim)
        if key not in cache:
            ctx = Context(fixed, moving, g, form=form, mse_grad=mse_grad,
                          device=device)
            ctx.set_images(moving_grad=moving_grad)
            cache[key] = ctx
        s, grad, n = cache[key].score_mse_f64(coeff)
        if n < 1:
            return 0.0, np.zeros_like(grad), 0
        return s * n, grad * (n / 2.0), n

    run.contexts = cache
    return run


class ContextMiEvaluator:
    """MI passes of slabs on the GPU through a Context per slab grid: hist()
    returns the slab's integer histograms, grad() the score of the given
    (summed) histograms and the slab's gradient part in double."""

    def __init__(self, fixed: Volume, moving: Volume, form: str = "tc",
                 mi_bins: int = 32, mi_window: str = "pvi8", device: int = 0):
        self.fixed, self.moving = fixed, moving
        self.kw = dict(form=form, mi_bins=mi_bins, mi_window=mi_window,
                       device=device)
        self.contexts = {}

    def _ctx(self, g: BsplineGrid):
        from . import Context
        key = (g.roi_offset, g.roi_dim)
        if key not in self.contexts:
            ctx = Context(self.fixed, self.moving, g, **self.kw)
            ctx.set_images()
            self.contexts[key] = ctx
        return self.contexts[key]

    def hist(self, g: BsplineGrid, coeff: np.ndarray) -> np.ndarray:
        return self._ctx(g).mi_hist(coeff)

    def grad(self, g: BsplineGrid, coeff: np.ndarray, hist: np.ndarray):
        return self._ctx(g).mi_grad(coeff, hist)

    hist_dtype = np.int64

    def hist_len(self) -> int:
        b = self.kw["mi_bins"]
        return 2 * b + b * b + 1


class SlabScorer:
    """MSE score + gradient of one volume sharded by z-slab over a
    torch.distributed process group (every rank calls score_mse with the
    same coefficients and receives the same global result)."""

    def __init__(self, grid: BsplineGrid, evaluate: Evaluator, group=None,
                 device=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.grid = grid
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.slab = plan_slabs(grid, self.world)[self.rank]
        self.local_grid = None if self.slab.empty else slab_grid(grid, self.slab)
        self.evaluate = evaluate
        self.device = device

    def score_mse(self, coeff: np.ndarray):
        """(score, gradient float32, num_vox), as b200bsp_score_mse."""
        import torch
        n = self.grid.num_coeff
        buf = np.zeros(n + 2, np.float64)
        if not self.slab.empty:
            s, g, nv = self.evaluate(self.local_grid,
                                     slab_coeff(self.grid, self.slab, coeff))
            scatter_grad(self.grid, self.slab, g, buf[:n])
            buf[n] = s
            buf[n + 1] = nv
        t = torch.from_numpy(buf)
        if self.device is not None:
            t = t.to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        buf = t.cpu().numpy()
        nv = int(round(buf[n + 1]))
        if nv < 1:
            return FLT_MAX, np.zeros(n, np.float32), 0
        score = buf[n] / nv
        grad = (2.0 * buf[:n] / nv).astype(np.float32)
        return float(np.float32(score)), grad, nv

    def score_mi(self, coeff: np.ndarray, mi_eval):
        """(score, gradient float32, num_vox), as b200bsp_score_mi over the
        whole ROI.  mi_eval: hist(grid, coeff) -> histograms (the count
        last; of type mi_eval.hist_dtype, float64 when absent),
        grad(grid, coeff, hist) -> (score, slab gradient, num_vox),
        hist_len()."""
        import torch
        n = self.grid.num_coeff
        c_local = None
        if self.slab.empty:
            # zeros of the evaluator's histogram type: every rank must pass
            # the same dtype to the all-reduce
            h = np.zeros(mi_eval.hist_len(),
                         getattr(mi_eval, "hist_dtype", np.float64))
        else:
            c_local = slab_coeff(self.grid, self.slab, coeff)
            h = np.asarray(mi_eval.hist(self.local_grid, c_local))
        t = torch.from_numpy(np.ascontiguousarray(h))
        if self.device is not None:
            t = t.to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        h = t.cpu().numpy()
        buf = np.zeros(n + 1, np.float64)
        if not self.slab.empty:
            s, g, _ = mi_eval.grad(self.local_grid, c_local, h)
            scatter_grad(self.grid, self.slab, g, buf[:n])
            if self.rank == 0:
                buf[n] = s
        t = torch.from_numpy(buf)
        if self.device is not None:
            t = t.to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        buf = t.cpu().numpy()
        nv = int(round(float(h[-1])))
        if nv < 1:
            return FLT_MAX, np.zeros(n, np.float32), 0
        return float(np.float32(buf[n])), buf[:n].astype(np.float32), nv
