"""Multi-rank host logic on CPU with gloo (world size 2): each rank renders
its own, disjoint set of views of the same size (weak scaling), and the job
time is the max over ranks."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from sv_raster_b200 import synthetic, workload


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        base = [synthetic.make_camera(320, 200, 50.0, (0.0, 0.0, -1.8)),
                synthetic.make_camera(320, 200, 50.0, (1.0, 0.2, -1.5))]
        cams = workload.rank_cameras(base, rank, world)
        # every rank sees every rank's camera positions: all distinct, same sizes
        pos = torch.tensor(np.stack([c.position for c in cams]), dtype=torch.float64)
        allpos = [torch.zeros_like(pos) for _ in range(world)]
        dist.all_gather(allpos, pos)
        flat = torch.cat(allpos)
        uniq = len({tuple(np.round(p.numpy(), 9)) for p in flat})
        sizes = {(c.width, c.height) for c in cams}
        t = workload.max_over_ranks(10.0 + rank)
        out[rank] = (len(cams), uniq, sizes == {(320, 200)}, t)
    finally:
        dist.destroy_process_group()


def test_view_sharding_and_max_over_ranks_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        n, uniq, same_size, t = out[r]
        assert n == 2 and same_size
        assert uniq == 4            # 2 ranks x 2 views, no view rendered twice
        assert t == 11.0            # max over ranks


def _exchange_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ex = workload.GradientExchange()
        # each rank's gradient of its own views' mean loss, laid out like the flat buffer
        g = torch.arange(12, dtype=torch.float32) * (rank + 1)
        loss = torch.tensor(float(rank + 1))
        ex(g, loss)
        out[rank] = (ex.world, g.tolist(), float(loss))
    finally:
        dist.destroy_process_group()


def test_gradient_exchange_averages_over_ranks_gloo():
    """View-parallel training: after the exchange every rank holds the mean
    of the ranks' gradients (the gradient of the mean loss over all views),
    so identical optimizer steps keep the parameters replicated."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_exchange_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    expect = [1.5 * i for i in range(12)]
    for r in range(world):
        w, g, loss = out[r]
        assert w == 2
        assert g == expect
        assert loss == 1.5


def test_gradient_exchange_is_identity_on_one_rank():
    ex = workload.GradientExchange()
    g = torch.ones(4)
    ex(g, torch.tensor(2.0))
    assert ex.world == 1 and g.tolist() == [1.0] * 4
