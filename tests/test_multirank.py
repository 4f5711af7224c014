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


def _view_grad(sc, cam, target):
    """Flat (densities, sh0, shs) gradient of one view's L2 loss (mean over
    its pixels), from the CPU oracle's fp32 forward, backward and SH backward."""
    import oracle as O
    idx = np.arange(sc.n_voxels)
    rgbs = O.sh_fwd(3, idx, sc.centers, cam.position, sc.sh0, sc.shs)
    o = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, sc.geos, rgbs)
    dC = (2.0 / o["color"].size * (o["color"] - target)).astype(np.float32)
    g = O.render_bwd(cam, o["ranges"], o["tile_last"], o["vals"], o["bbox"], sc.centers, sc.lengths, sc.geos, rgbs,
                     o["n_contrib"], o["T"], dC, np.zeros((cam.height, cam.width), np.float32))
    d0, ds = O.sh_bwd(3, 16, idx, sc.centers, cam.position, g["dL_drgbs"])
    return np.concatenate([g["dL_dgeos"].ravel(), d0.ravel(), ds.ravel()]).astype(np.float32)


def _split_scene():
    sc = synthetic.config_scene("c1", n_voxels=3000)
    sc.cameras = [synthetic.make_camera(96, 72, 50.0, (0.0, 0.0, -1.5)),
                  synthetic.make_camera(96, 72, 50.0, (1.0, -0.3, -1.1))]
    tg = [np.random.default_rng(40 + i).uniform(0, 1, (3, 72, 96)).astype(np.float32) for i in range(2)]
    return sc, tg


def _split_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sc, tg = _split_scene()
        flat = torch.from_numpy(_view_grad(sc, sc.cameras[rank], tg[rank]))  # this rank's view only
        workload.GradientExchange()(flat)
        out[rank] = flat.numpy().copy()
    finally:
        dist.destroy_process_group()


def test_view_split_reproduces_single_process_gradient_gloo():
    """Two ranks each back-propagate one view and exchange: every rank ends with
    the single-process gradient of the mean loss over both views (up to the
    order of the oracle's threaded per-tile additions)."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_split_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    sc, tg = _split_scene()
    g0, g1 = _view_grad(sc, sc.cameras[0], tg[0]), _view_grad(sc, sc.cameras[1], tg[1])
    want = (torch.from_numpy(g0) + torch.from_numpy(g1)) * 0.5
    assert float(want.abs().max()) > 0
    w = want.numpy().astype(np.float64)
    for r in range(world):
        assert np.linalg.norm(out[r] - w) <= 1e-6 * np.linalg.norm(w)
    assert np.array_equal(out[0], out[1])  # the ranks agree exactly: replicated parameters stay replicated


def test_rank_cameras_keep_the_configuration_distribution():
    """Every rank renders as many views as rank 0, at the configuration's sizes
    and camera distances, from distinct positions."""
    for name, radius in (("c4", (1.5, 2.0)), ("c3", (2.0, 4.0))):
        base = synthetic.config_cameras(name)
        r1 = workload.rank_cameras(base, 1, 4, config=name)
        r3 = workload.rank_cameras(base, 3, 4, config=name)
        assert workload.rank_cameras(base, 0, 4, config=name) == base
        for cams in (r1, r3):
            assert len(cams) == len(base)
            for c in cams:
                assert radius[0] - 1e-5 <= float(np.linalg.norm(c.position)) <= radius[1] + 1e-5
        if name == "c4":
            assert {(c.width, c.height) for c in r1} == {(1920, 1080)}
        else:
            assert all(640 <= c.width <= 1600 and 480 <= c.height <= 1200 for c in r1 + r3)
        pos = {tuple(np.round(c.position, 6)) for c in base + r1 + r3}
        assert len(pos) == 3 * len(base)


def _bucket_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ex = workload.GradientExchange()
        flat = torch.arange(20, dtype=torch.float32) * (rank + 1)
        loss = torch.tensor(float(rank + 3))
        dens, sh = flat[:8], flat[8:]  # views into the flat buffer, exchanged as two buckets
        w = ex.start(dens)
        sh.add_(1.0)  # work queued between the two starts (the SH backward in a training step)
        ex.finish([(w, dens), (ex.start(sh), sh), (ex.start(loss), loss)])
        out[rank] = (flat.tolist(), float(loss))
    finally:
        dist.destroy_process_group()


def test_bucketed_exchange_averages_each_bucket_gloo():
    """The training step's bucketed exchange: the density bucket is started
    before the SH gradients are final, the SH bucket after; every bucket of
    the flat buffer (a view into it) ends as the mean over ranks."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_bucket_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    want = [1.5 * i for i in range(8)] + [1.5 * i + 1.0 for i in range(8, 20)]
    for r in range(world):
        flat, loss = out[r]
        assert flat == want and loss == 3.5
