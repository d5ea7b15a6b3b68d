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
