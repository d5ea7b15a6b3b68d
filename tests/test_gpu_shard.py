"""Z-slab sharding with the GPU kernels: two gloo ranks, each evaluating its
slab through a Context on the one visible GPU (the ranks never wait on each
other inside a kernel; the all-reduce runs on the host), against one
whole-volume Context.  MSE bars: voxel count within 2, score relative 1e-5,
gradient relative 1e-4 (both sides run the same tile kernel; slabs only
regroup the tiles and reorder sums).  MI: the slabs' integer histograms sum
to the whole volume's bit for bit, so the score is equal; gradient relative
1e-5 (double-precision slab parts, float32 whole-volume gradient)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _case():
    from plastimatch_b200 import synth
    from plastimatch_b200.geometry import BsplineGrid
    fixed = synth.gaussian_blobs((64, 60, 70), spacing=(1, 1, 1.5), seed=8)
    g0 = BsplineGrid.for_volume(fixed, 8)
    moving = synth.warp_trilinear(fixed, fixed, g0,
                                  synth.random_coeff(g0, 2.0, 9))
    grid = BsplineGrid.for_volume(fixed, (5, 6, 4))
    coeff = synth.random_coeff(grid, 1.5, 10)
    return fixed, moving, grid, coeff


def _rank(rank, world, port, form, q, metric="mse", window="pvi8"):
    import torch.distributed as dist
    from plastimatch_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fixed, moving, grid, coeff = _case()
        if metric == "mse":
            ev = shard.context_evaluator(fixed, moving, form=form)
            sc = shard.SlabScorer(grid, ev)
            q.put((rank,) + tuple(sc.score_mse(coeff)))
        else:
            ev = shard.ContextMiEvaluator(fixed, moving, form=form,
                                          mi_window=window)
            sc = shard.SlabScorer(grid, None)
            q.put((rank,) + tuple(sc.score_mi(coeff, ev)))
        for c in ev.contexts.values():
            c.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("form", ["tc", "fp32"])
def test_two_slabs_match_whole_volume(form):
    import plastimatch_b200 as P
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, form, q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fixed, moving, grid, coeff = _case()
    with P.Context(fixed, moving, grid, form=form) as c:
        c.set_images()
        s0, g0, n0 = c.score_mse(coeff)
    for _, s, g, n in res:
        assert abs(n - n0) <= 2
        assert abs(s - s0) <= 1e-5 * abs(s0)
        assert rel_err(g, g0) < 1e-4


@pytest.mark.parametrize("window", ["pvi8", "parzen"])
@pytest.mark.parametrize("form", ["tc", "fp32"])
def test_slab_mi_histograms_sum_exactly(form, window):
    """Two slab contexts in one process: their pass-1 histograms add up to
    the whole volume's exactly; pass 2 with the sum gives the whole
    volume's score and, scattered, its gradient."""
    import plastimatch_b200 as P
    from plastimatch_b200 import shard
    fixed, moving, grid, coeff = _case()
    with P.Context(fixed, moving, grid, form=form, mi_window=window) as c:
        c.set_images()
        s0, g0, n0 = c.score_mi(coeff)
        h0 = c.mi_hist(coeff)
    ev = shard.ContextMiEvaluator(fixed, moving, form=form, mi_window=window)
    slabs = [sl for sl in shard.plan_slabs(grid, 2) if not sl.empty]
    parts = [(shard.slab_grid(grid, sl), shard.slab_coeff(grid, sl, coeff))
             for sl in slabs]
    h = sum(ev.hist(g, cc) for g, cc in parts)
    np.testing.assert_array_equal(h, h0)
    acc = np.zeros(grid.num_coeff)
    for sl, (g, cc) in zip(slabs, parts):
        s, gr, n = ev.grad(g, cc, h)
        assert s == s0 and n == n0
        shard.scatter_grad(grid, sl, gr, acc)
    assert rel_err(acc, g0) < 1e-5
    for cx in ev.contexts.values():
        cx.close()


@pytest.mark.parametrize("window", ["pvi8", "parzen"])
def test_two_slab_ranks_mi(window):
    import plastimatch_b200 as P
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = [ctx.Process(target=_rank,
                         args=(r, 2, port, "tc", q, "mi", window))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fixed, moving, grid, coeff = _case()
    with P.Context(fixed, moving, grid, form="tc", mi_window=window) as c:
        c.set_images()
        s0, g0, n0 = c.score_mi(coeff)
    for _, s, g, n in res:
        assert n == n0 and s == s0
        assert rel_err(g, g0) < 1e-5
