"""Z-slab sharding of one volume over a process group (host logic).

Runs as gloo ranks on CPU; each rank evaluates its slab with the oracle
(double precision) and the all-reduced result must equal the oracle's
whole-volume evaluation: exact voxel count, score and gradient within
relative 1e-6 (they are returned in float32, as the reference reports them;
the slab decomposition itself is exact and only the summation order
differs).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from conftest import load_golden, rel_err
from plastimatch_b200 import shard, synth
from plastimatch_b200.geometry import BsplineGrid


def _case():
    fixed = synth.gaussian_blobs((24, 22, 37), spacing=(1.0, 1.1, 0.9),
                                 seed=41)
    g0 = BsplineGrid.for_volume(fixed, 6)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.5, 42))
    grid = BsplineGrid.for_volume(fixed, (5, 6, 4), roi_offset=(1, 0, 2),
                                  roi_dim=(22, 22, 33))
    coeff = synth.random_coeff(grid, 1.0, 43)
    return fixed, moving, grid, coeff


def oracle_evaluator(fixed, moving, mgrad):
    def run(g, c):
        r = O.port_mse(g, fixed, moving, c, moving_grad=mgrad,
                       precision="f64")
        n = r.num_vox
        if n < 1:
            return 0.0, np.zeros(g.num_coeff), 0
        return r.score * n, r.grad * (n / 2.0), n
    return run


def test_plan_covers_every_tile_once():
    _, _, grid, _ = _case()
    for world in (1, 2, 3, 8, 9, 20):
        slabs = shard.plan_slabs(grid, world)
        assert len(slabs) == world
        assert slabs[0].tz0 == 0 and slabs[-1].tz1 == grid.rdims[2]
        for a, b in zip(slabs, slabs[1:]):
            assert a.tz1 == b.tz0
        sizes = [s.tz1 - s.tz0 for s in slabs]
        assert max(sizes) - min(sizes) <= 1


def test_slab_grids_tile_the_roi():
    fixed, _, grid, coeff = _case()
    slabs = [s for s in shard.plan_slabs(grid, 3) if not s.empty]
    z = grid.roi_offset[2]
    acc = np.zeros(grid.num_coeff)
    for s in slabs:
        g = shard.slab_grid(grid, s)
        assert g.roi_offset[2] == z and g.rdims[:2] == grid.rdims[:2]
        z += g.roi_dim[2]
        c = shard.slab_coeff(grid, s, coeff)
        assert c.size == g.num_coeff
        shard.scatter_grad(grid, s, np.ones(g.num_coeff), acc)
    assert z == grid.roi_offset[2] + grid.roi_dim[2]
    # interior knot planes are shared by the tiles of neighbouring slabs
    assert acc.max() == 2 and acc.min() == 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, name, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if name == "blobs":
            fixed, moving, grid, coeff = _case()
        else:
            fixed, moving, grid, coeff, _ = load_golden(name)
        mgrad = O.port_volume_grad(moving)
        sc = shard.SlabScorer(grid, oracle_evaluator(fixed, moving, mgrad))
        s, g, n = sc.score_mse(coeff)
        # a second call with other coefficients: the scorer is reusable
        s2, g2, n2 = sc.score_mse(coeff * 0.5)
        q.put((rank, s, g, n, s2, g2, n2))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,name", [(2, "blobs"), (3, "blobs"),
                                        (2, "mse_dcos"), (5, "mse_small")])
def test_slab_all_reduce_matches_whole_volume(world, name):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, name, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    if name == "blobs":
        fixed, moving, grid, coeff = _case()
    else:
        fixed, moving, grid, coeff, _ = load_golden(name)
    mgrad = O.port_volume_grad(moving)
    for c, idx in ((coeff, 1), (coeff * 0.5, 4)):
        ref = O.port_mse(grid, fixed, moving, c, moving_grad=mgrad,
                         precision="f64")
        for r in res:
            s, g, n = r[idx], r[idx + 1], r[idx + 2]
            assert n == ref.num_vox
            assert abs(s - ref.score) <= 1e-6 * abs(ref.score)
            assert rel_err(g, ref.grad) < 1e-6
    # every rank holds the same result
    for r in res[1:]:
        assert r[1] == res[0][1]
        np.testing.assert_array_equal(r[2], res[0][2])


class OracleMiEvaluator:
    """PVI-8 MI passes of a slab with the oracle (double precision)."""

    def __init__(self, fixed, moving, bins):
        self.fixed, self.moving, self.bins = fixed, moving, bins

    def hist_len(self):
        return 2 * self.bins + self.bins * self.bins + 1

    def hist(self, g, c):
        f, m, j, n = O.port_mi_pass1(g, self.fixed, self.moving, c, self.bins)
        return np.concatenate([f, m, j, [float(n)]])

    def grad(self, g, c, h):
        b = self.bins
        f, m, j, n = h[:b], h[b:2 * b], h[2 * b:-1], int(round(h[-1]))
        s, gr = O.port_mi_pass2(g, self.fixed, self.moving, c, f, m, j, n, b)
        return s, gr, n


def _mi_case():
    fixed = synth.gaussian_blobs((24, 22, 37), spacing=(1.0, 1.1, 0.9),
                                 seed=51)
    g0 = BsplineGrid.for_volume(fixed, 6)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.5, 52))
    # the reference's MI needs the ROI to be the whole image
    grid = BsplineGrid.for_volume(fixed, (5, 6, 4))
    coeff = synth.random_coeff(grid, 1.0, 53)
    return fixed, moving, grid, coeff


def _mi_thin_case():
    """Two tiles along z: a third rank gets an empty slab."""
    fixed = synth.gaussian_blobs((20, 18, 7), spacing=(1.0, 1.0, 1.2),
                                 seed=54)
    g0 = BsplineGrid.for_volume(fixed, 5)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 1.0, 55))
    grid = BsplineGrid.for_volume(fixed, (5, 4, 4))
    coeff = synth.random_coeff(grid, 0.8, 56)
    return fixed, moving, grid, coeff


def _mi_rank_main(rank, world, port, q, thin=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fixed, moving, grid, coeff = _mi_thin_case() if thin else _mi_case()
        sc = shard.SlabScorer(grid, None)
        s, g, n = sc.score_mi(coeff, OracleMiEvaluator(fixed, moving, 16))
        q.put((rank, s, g, n))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,thin", [(2, False), (3, False), (3, True)])
def test_slab_mi_matches_whole_volume(world, thin):
    """MI over z-slabs: histograms all-reduced between the passes, slab
    gradients all-reduced after; equal to the whole-volume oracle (score
    within 1e-6 relative, returned in float32; gradient 1e-6 L2).  The thin
    case leaves one rank an empty slab."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mi_rank_main, args=(r, world, port, q, thin))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fixed, moving, grid, coeff = _mi_thin_case() if thin else _mi_case()
    if thin:
        assert sum(s.empty for s in shard.plan_slabs(grid, world)) == 1
    ref = O.port_mi(grid, fixed, moving, coeff, bins=16, precision="f64")
    for _, s, g, n in res:
        assert n == ref.num_vox
        assert abs(s - ref.score) <= 1e-6 * abs(ref.score)
        assert rel_err(g, ref.grad) < 1e-6
    for r in res[1:]:
        assert r[1] == res[0][1]
        np.testing.assert_array_equal(r[2], res[0][2])
