"""Benchmark workloads: a scene, its views and one timed step (every view
rendered and back-propagated), in the plain one-view-per-call form and the
batched multi-view form.  Used by bench.py; kept in the package so the step
is the same code a user would run.
"""
import ctypes
import math

import numpy as np
import torch

from . import _C
from ._native import Camera, check, lib

RECORD_BYTES = 68  # bbox 8 + centre 12 + length 4 + 8 densities 32 + rgb 12


def rank_cameras(cameras, rank, world, config=None, seed=0):
    """Views rendered by `rank` of `world` (weak scaling: every rank does the
    single-GPU workload's amount of work).  Rank 0 keeps the workload's own
    cameras; rank k > 0 gets view set k of the same configuration
    (synthetic.config_cameras): the same count, sizes and distance
    distribution, other seeded positions.  Without a configuration name,
    rank k gets seeded orbit cameras of the first camera's size."""
    if world <= 1 or rank == 0:
        return list(cameras)
    from . import synthetic
    n = len(cameras)
    if config is not None:
        return synthetic.config_cameras(config, seed, view_set=rank)[:n]
    extra = synthetic.orbit_cameras(n * world, 1007 + seed, radius=(1.5, 2.0),
                                    fixed_size=(cameras[0].width, cameras[0].height))
    return extra[rank * n:(rank + 1) * n]


def max_over_ranks(value, group=None, device=None):
    """Max of a per-rank float over the process group (the job's time is its
    slowest rank's)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def _t(a, dev, dt=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)


def tune_raster(raster, geos, sh0, shs):
    """Autotune a batched rasterizer on this scene (see autotune.py); returns
    the chosen launch parameters as a JSON-able dict."""
    from .autotune import tune_batched
    res = tune_batched(raster, geos, sh0, shs, 3)
    out = {k: (list(v) if isinstance(v, tuple) else v) for k, v in res["choice"].items()}
    out["timings_ms"] = res["timings"]
    out["cached"] = res["cached"]
    return out


class _Timer:
    """CUDA-event timing of one kernel stage on the launching stream."""

    def __init__(self, name):
        self.name = name
        self.pairs = []
        self.bytes = []

    def start(self, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        self.pairs.append((e0, e1))
        return e1

    def stats(self):
        ms = [a.elapsed_time(b) for a, b in self.pairs]
        return dict(name=self.name, launches=len(ms), ms=float(sum(ms)), bytes=float(sum(self.bytes)),
                    ms_per_launch=float(np.mean(ms)) if ms else 0.0,
                    bytes_per_launch=float(np.mean(self.bytes)) if self.bytes else 0.0)


class PlainWorkload:
    """The reference's call pattern: one view per call, fp32, a host read of
    the instance count per view (forward.cu:652-658)."""

    def __init__(self, scene, dev):
        self.sc = scene
        self.dev = dev
        self.octpath = _t(scene.octpath.reshape(-1, 1), dev, torch.int64)
        self.centers = _t(scene.centers, dev)
        self.lengths = _t(scene.lengths, dev)
        self.geos = _t(scene.geos, dev)
        self.sh0 = _t(scene.sh0, dev)
        self.shs = _t(scene.shs, dev)
        self.P = scene.n_voxels
        self.cams = []
        for c in scene.cameras:
            self.cams.append((c, _t(c.w2c, dev), _t(c.c2w, dev)))
        self.targets = [_t(t, dev) for t in scene.targets]
        self.timers = {}
        self._inst = []
        self.empty_idx = torch.empty(0, dtype=torch.int64, device=dev)
        self.n_passes = []

    def reset_kernel_timers(self):
        self.timers = {k: _Timer(k) for k in ("preprocess+scan", "binning", "render_fwd", "render_bwd", "sh")}
        self._inst = []

    def _stage(self, name, fn, nbytes=0.0):
        if name not in self.timers:
            return fn()
        st = torch.cuda.current_stream(self.dev)
        e1 = self.timers[name].start(st)
        r = fn()
        e1.record(st)
        self.timers[name].bytes.append(nbytes)
        return r

    def view_fwd_bwd(self, i):
        cam, w2c, c2w = self.cams[i]
        W, H = cam.width, cam.height
        L = lib()
        dev = self.dev
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        cam_pos = c2w[:3, 3].contiguous()
        ndup, geom = self._stage("preprocess+scan", lambda: _C.rasterize_preprocess(
            W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near, self.octpath, self.centers,
            self.lengths), 36.0 * self.P)
        vis = torch.where(ndup > 0)[0]  # host sync, as the reference's renderer.py:83
        V = int(vis.numel())
        rgbs = self._stage("sh", lambda: _C.sh_compute(3, vis, self.centers, cam_pos, self.sh0, self.shs),
                           V * (12 + 192 + 12.0))
        R = _C.geom_num_rendered(geom)
        self._inst.append(R)
        T_ = math.ceil(W / 16) * math.ceil(H / 16)
        binning = torch.empty(L.svr_binning_buffer_bytes(R, W, H), dtype=torch.uint8, device=dev)
        img = torch.empty(L.svr_image_buffer_bytes(W, H), dtype=torch.uint8, device=dev)
        color = torch.zeros(3, H, W, device=dev)
        Tm = torch.zeros(1, H, W, device=dev)
        ccam = Camera(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c.data_ptr(), c2w.data_ptr(), cam.near, 0.0)
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        self._stage("binning", lambda: check(L.svr_rasterize_binning(
            ctypes.byref(ccam), self.P, R, p(self.octpath), p(geom), p(binning), binning.numel(), p(img),
            img.numel(), 0, stream), "binning"), 28.0 * V + 12.0 * R + 24.0 * R + 8.0 * R + 8.0 * T_)
        self._stage("render_fwd", lambda: check(L.svr_rasterize_render(
            ctypes.byref(ccam), 1, 0, 0, 0, 0, self.P, R, p(self.centers), p(self.lengths), p(self.geos), p(rgbs),
            p(geom), p(binning), binning.numel(), p(img), img.numel(), p(color), None, None, p(Tm), None, 0,
            stream), "render"), R * (4.0 + RECORD_BYTES) + 20.0 * W * H + 12.0 * T_)
        tgt = self.targets[i % len(self.targets)]
        dC = (2.0 / color.numel()) * (color - tgt)
        dT = torch.zeros_like(Tm)
        dgeo = torch.zeros(self.P, 8, device=dev)
        drgb = torch.zeros(self.P, 3, device=dev)
        sub = torch.zeros(self.P, 1, device=dev)
        self._stage("render_bwd", lambda: check(L.svr_rasterize_backward(
            ctypes.byref(ccam), 1, self.P, R, p(self.centers), p(self.lengths), p(self.geos), p(rgbs), p(geom),
            p(binning), p(img), p(Tm), p(dC), None, None, p(dT), 0.0, None, 0.0, 0.0, 0, 0, None, None, p(dgeo),
            p(drgb), p(sub), 0, stream), "render_bwd"), R * (4.0 + RECORD_BYTES) + 24.0 * W * H + 48.0 * V)
        self._stage("sh", lambda: _C.sh_compute_bw(3, 16, vis, self.centers, cam_pos, rgbs, drgb),
                    V * (12 * 3 + 192.0))
        return dgeo

    def step(self):
        for i in range(len(self.cams)):
            self.view_fwd_bwd(i)

    def instances_per_view(self):
        return int(np.mean(self._inst)) if self._inst else None

    def launches_per_step(self):
        n = 0
        for cam, _, _ in self.cams:
            T_ = math.ceil(cam.width / 16) * math.ceil(cam.height / 16)
            passes = math.ceil(int(T_).bit_length() / 10)  # radix passes over the tile bits (8-10 bit digits)
            # preprocess 1 + scan 3 + duplicate 1 + sort 3/pass + ranges 1 + segment sort 4
            # + tile order (key kernel + one 3-kernel sort pass) 4 + fwd 1 + bwd 1 + sh 2
            n += 1 + 3 + 1 + 3 * passes + 1 + 4 + 4 + 1 + 1 + 2
        return n

    def kernel_stats(self):
        torch.cuda.synchronize()
        table = [t.stats() for t in self.timers.values()]
        dom = max(table, key=lambda s: s["ms"])
        fwd = [s for s in table if s["name"] in ("preprocess+scan", "binning", "render_fwd", "sh")]
        fwd_ms = sum(s["ms"] for s in fwd if s["name"] != "sh") + \
            sum(s["ms"] for s in table if s["name"] == "sh") / 2.0
        nviews = max(1, len(self.timers["render_fwd"].pairs))
        return dict(table=[{k: (round(v, 4) if isinstance(v, float) else v) for k, v in s.items()} for s in table],
                    dominant=dom, fwd_ms_per_view=fwd_ms / nviews)

    def e2e(self, steps, warmup):
        """Same step through the public autograd API; per step the targets and
        camera matrices are copied from pinned host memory and the loss is
        read back."""
        from . import renderer
        dev = self.dev
        host_t = [torch.from_numpy(np.ascontiguousarray(t)).pin_memory() for t in self.sc.targets]
        host_c = [(torch.from_numpy(c.w2c).pin_memory(), torch.from_numpy(c.c2w).pin_memory())
                  for c in self.sc.cameras]
        geos = self.geos.clone().requires_grad_(True)
        sh0 = self.sh0.clone().requires_grad_(True)
        shs = self.shs.clone().requires_grad_(True)
        h2d = sum(t.numel() * 4 for t in host_t[: len(self.cams)]) + 2 * 64 * len(self.cams)
        ones = torch.ones(self.P, 1, device=dev)

        def one_step():
            total = None
            for i, (cam, _, _) in enumerate(self.cams):
                tgt = host_t[i % len(host_t)].to(dev, non_blocking=True)
                w2c = host_c[i][0].to(dev, non_blocking=True)
                c2w = host_c[i][1].to(dev, non_blocking=True)
                s = renderer.RasterSettings(color_mode="sh", n_samp_per_vox=1, image_width=cam.width,
                                            image_height=cam.height, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy,
                                            cx=cam.cx, cy=cam.cy, w2c_matrix=w2c, c2w_matrix=c2w)

                def vox_fn(idx, cam_pos, color_mode):
                    rgbs = renderer.SH_eval.apply(3, idx, self.centers, cam_pos, None, sh0, shs)
                    return {"geos": geos, "rgbs": rgbs, "subdiv_p": ones}

                color, _, _, _, _ = renderer.rasterize_voxels(s, self.octpath, self.centers, self.lengths, vox_fn)
                loss = ((color - tgt) ** 2).mean()
                loss.backward()
                total = loss.detach() if total is None else total + loss.detach()
            return float(total.cpu())

        for _ in range(warmup):
            one_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream(dev)
        e0.record(st)
        for _ in range(steps):
            one_step()
        e1.record(st)
        torch.cuda.synchronize()
        return dict(ms_total=e0.elapsed_time(e1), h2d=h2d, d2h=4)


class _DevCam:
    def __init__(self, c, dev):
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = _t(c.w2c, dev)
        self.c2w = _t(c.c2w, dev)


class BatchedWorkload:
    """All views in one launch per stage, bf16 storage of densities and SH,
    fp32 compositing / gradients, no host sync inside a step (the step is
    also captured as a CUDA graph)."""

    def __init__(self, scene, dev, storage=torch.bfloat16, graph=True, tune=True, tile=None, exact=False,
                 bwd_walk=None):
        from .batched import BatchedRasterizer
        self.sc = scene
        self.dev = dev
        self.P = scene.n_voxels
        self.octpath = _t(scene.octpath.reshape(-1, 1), dev, torch.int64)
        self.centers = _t(scene.centers, dev)
        self.lengths = _t(scene.lengths, dev)
        self.geos = _t(scene.geos, dev).to(storage).contiguous()
        self.sh0 = _t(scene.sh0, dev).to(storage).contiguous()
        self.shs = _t(scene.shs, dev).to(storage).contiguous()
        self.cams = [_DevCam(c, dev) for c in scene.cameras]
        self.raster = BatchedRasterizer(self.cams, self.octpath, self.centers, self.lengths,
                                        max_level=scene.max_level, exact=exact)
        self.tuned = None
        if tile is not None:
            self.raster.set_tile_size(*tile[:2])
            if len(tile) > 2:
                self.raster.set_backward_staging(tile[2])
            self.tuned = {"tile": list(tile), "fixed": True}
        if bwd_walk is not None:
            # the backward's pixels per thread: one ("warp") or two ("pair")
            self.raster.set_backward_pixels_per_thread({"warp": 1, "pair": 2}[bwd_walk])
            if self.tuned is not None:
                self.tuned["bwd_walk"] = bwd_walk
        self.total = self.raster.fit_capacity(self.sh0, self.shs, 3)
        if tune:
            self.tuned = tune_raster(self.raster, self.geos, self.sh0, self.shs)
            self.total = self.raster.fit_capacity(self.sh0, self.shs, 3)
        r = self.raster
        tg = [_t(t, dev).reshape(-1) for t in scene.targets]
        self.target = torch.cat([tg[i % len(tg)] for i in range(len(self.cams))])
        scale = [torch.full((3 * h * w,), 2.0 / (3 * h * w), device=dev) for h, w in r.sizes]
        self.scale = torch.cat(scale)
        self.color = torch.zeros(3 * r.n_pixels, device=dev)
        self.T = torch.zeros(r.n_pixels, device=dev)
        self.dT = torch.zeros(r.n_pixels, device=dev)
        self.dC = torch.zeros_like(self.color)
        self.grads = (torch.zeros(self.P, 8, device=dev), torch.zeros(self.P, device=dev),
                      torch.zeros(self.P, 3, device=dev), torch.zeros(self.P, 15, 3, device=dev))
        self.timers = {}
        self.graph = None
        self.use_graph = graph

    def reset_kernel_timers(self):
        self.timers = {k: _Timer(k) for k in ("prepare", "render_fwd", "render_bwd", "sh_bwd")}

    def _stage(self, name, fn, nbytes=0.0):
        if name not in self.timers:
            return fn()
        st = torch.cuda.current_stream(self.dev)
        e1 = self.timers[name].start(st)
        r = fn()
        e1.record(st)
        self.timers[name].bytes.append(nbytes)
        return r

    def _bytes(self):
        I, V = self.total, self._visible()
        px, T_ = self.raster.n_pixels, self.raster.n_tiles
        geo_b = 2 * 8 if self.geos.dtype == torch.bfloat16 else 4 * 8
        rec = 8 + 12 + 4 + geo_b + 12
        sh_b = 48 * (2 if self.sh0.dtype == torch.bfloat16 else 4)
        return dict(
            prepare=36.0 * self.P * len(self.cams) + V * (sh_b + 12) + 8.0 * self.P * len(self.cams) +
            (28.0 * V + 12.0 * I) + 24.0 * I * 1 + 8.0 * I + 8.0 * T_,
            render_fwd=I * (4.0 + rec) + 20.0 * px + 12.0 * T_,
            render_bwd=I * (4.0 + rec) + 24.0 * px + 48.0 * V,
            sh_bwd=self.P * len(self.cams) * 12.0 + V * 12.0 + self.P * (12 + 192.0))

    def _visible(self):
        if not hasattr(self, "_V"):
            self._V = int((self.raster.arrays()["ndup"] > 0).sum())
        return self._V

    def _eager_step(self, timed):
        r = self.raster
        b = self._bytes() if timed else {}
        st = (lambda n, f: self._stage(n, f, b[n])) if timed else (lambda n, f: f())
        st("prepare", lambda: r.prepare(self.sh0, self.shs, 3))
        st("render_fwd", lambda: r.render(self.geos, self.color, self.T))
        torch.mul(self.scale, self.color - self.target, out=self.dC)
        g = self.grads
        st("render_bwd", lambda: self._bwd_render())
        st("sh_bwd", lambda: self._bwd_sh())
        return g

    def _bwd_render(self):
        r = self.raster
        L = lib()
        g = self.grads
        g[0].zero_()
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        s = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        check(L.svr_batch_backward(r.plan, p(r.ws), p(self.centers), p(self.lengths), p(self.geos),
                                   int(self.geos.dtype == torch.bfloat16), p(self.T), p(self.dC), p(self.dT),
                                   p(g[0]), s), "batch_backward")

    def _bwd_sh(self):
        r = self.raster
        g = self.grads
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        s = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        check(lib().svr_batch_sh_backward(r.plan, p(r.ws), p(self.centers), 3, 16, p(g[2]), p(g[3]), p(g[1]), s),
              "batch_sh_backward")

    def capture(self):
        """Capture one step as a CUDA graph (after warm-up launches)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self._eager_step(False)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._eager_step(False)
        self.graph = g

    def step(self):
        if self.timers:
            return self._eager_step(True)
        if self.use_graph:
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self._eager_step(False)

    def check_errors(self):
        total, err = self.raster.header()
        if err:
            raise RuntimeError(f"batched step reported device error word 0x{err:x} (instances {total}, "
                               f"capacity {self.raster.capacity})")
        return total

    def instances_per_view(self):
        return int(self.total / max(1, len(self.cams)))

    def launches_per_step(self):
        T_ = max(self.raster.n_tiles, 1)
        passes = math.ceil(int(T_).bit_length() / 10)  # radix passes over the tile bits (8-10 bit digits)
        g = self.raster.n_groups
        order = self.raster.schedule[0]
        # project 1 + scan 3 + segments 1 + grouping by tile + segment sort 4 (plan, small,
        # chunk, merge) + per ordered compositing stage a tile-order key kernel and one
        # 3-kernel sort pass + fwd 1 + bwd 1 + sh 1.  Grouping by tile: counting sort =
        # count 1 + tile scan 3 + ranges 1 + scatter 1; radix = duplicate 1 + (sort 3/pass
        # + ranges 1) per group.
        n_order = 4 * ((order & 1) + ((order >> 1) & 1))
        grouping = 6 if getattr(self.raster, "binning", 0) else 1 + g * (3 * passes + 1)
        return 1 + 3 + 1 + grouping + 4 + n_order + 1 + 1 + 1

    def kernel_stats(self):
        torch.cuda.synchronize()
        table = [t.stats() for t in self.timers.values()]
        dom = max(table, key=lambda s: s["ms"])
        nsteps = max(1, len(self.timers["render_fwd"].pairs))
        fwd_ms = sum(s["ms"] for s in table if s["name"] in ("prepare", "render_fwd")) / nsteps
        return dict(table=[{k: (round(v, 4) if isinstance(v, float) else v) for k, v in s.items()} for s in table],
                    dominant=dom, fwd_ms_per_view=fwd_ms / len(self.cams))

    def e2e(self, steps, warmup):
        """Public autograd API (BatchedRender) with the targets and camera
        matrices copied from pinned host memory each step and the loss read
        back; cameras are updated in place so the plan stays valid.  The next
        step's targets are uploaded on a copy stream while the current step
        computes (double-buffered), as a training loop would prefetch them."""
        from .batched import BatchedRender
        dev = self.dev
        host_t = self.target.cpu().pin_memory()
        host_w2c = [torch.from_numpy(c.w2c).pin_memory() for c in self.sc.cameras]
        host_c2w = [torch.from_numpy(c.c2w).pin_memory() for c in self.sc.cameras]
        tgt = [torch.empty_like(self.target), torch.empty_like(self.target)]
        geos = self.geos.clone().requires_grad_(True)
        sh0 = self.sh0.clone().requires_grad_(True)
        shs = self.shs.clone().requires_grad_(True)
        h2d = host_t.numel() * 4 + len(self.cams) * 2 * 64
        main = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(dev)
        ready = [torch.cuda.Event(), torch.cuda.Event()]  # target buffer uploaded
        free = [torch.cuda.Event(), torch.cuda.Event()]   # target buffer consumed by its step

        def upload(k):
            with torch.cuda.stream(copy):
                copy.wait_event(free[k % 2])
                tgt[k % 2].copy_(host_t, non_blocking=True)
                ready[k % 2].record(copy)

        # mean over views of each view's MSE: with equal view sizes one weight
        # for every pixel, so the fused sum-of-squares loss applies
        uniform = len({h * w for h, w in self.raster.sizes}) == 1
        w0 = float(self.scale[0]) * 0.5

        def one_step(k):
            upload(k + 1)  # prefetch the next step's inputs behind this step's compute
            main.wait_event(ready[k % 2])
            for c, a, b in zip(self.cams, host_w2c, host_c2w):
                c.w2c.copy_(a, non_blocking=True)
                c.c2w.copy_(b, non_blocking=True)
            for t in (geos, sh0, shs):
                t.grad = None  # as an optimizer's zero_grad(set_to_none=True) would
            color, T = BatchedRender.apply(self.raster, 3, geos, sh0, shs)
            if uniform:
                loss = torch.nn.functional.mse_loss(color, tgt[k % 2], reduction="sum") * w0
            else:
                loss = (self.scale * 0.5 * (color - tgt[k % 2]) ** 2).sum()
            free[k % 2].record(main)
            loss.backward()
            return float(loss.detach().cpu())

        for e in free:
            e.record(main)
        upload(0)
        for k in range(warmup):
            one_step(k)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for k in range(warmup, warmup + steps):
            one_step(k)
        main.wait_event(ready[(warmup + steps) % 2])  # every upload issued in the timed region has landed
        e1.record(main)
        torch.cuda.synchronize()
        return dict(ms_total=e0.elapsed_time(e1), h2d=h2d, d2h=4)


class DeviceAdam:
    """Fused unbiased Adam over several parameter tensors with the step count
    on the device, so one captured training step can be replayed."""

    def __init__(self, params, lrs, betas=(0.1, 0.99), eps=1e-15, sparse=False):
        self.params = list(params)
        dev = self.params[0].device
        self.m = [torch.zeros(p.shape, dtype=torch.float32, device=dev) for p in self.params]
        self.v = [torch.zeros(p.shape, dtype=torch.float32, device=dev) for p in self.params]
        self.d_step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.lrs, self.betas, self.eps, self.sparse = list(lrs), betas, eps, sparse
        n = len(self.params)
        self._P = (ctypes.c_void_p * n)(*[p.data_ptr() for p in self.params])
        self._B = (ctypes.c_int * n)(*[int(p.dtype == torch.bfloat16) for p in self.params])
        self._M = (ctypes.c_void_p * n)(*[t.data_ptr() for t in self.m])
        self._V = (ctypes.c_void_p * n)(*[t.data_ptr() for t in self.v])
        self._N = (ctypes.c_int64 * n)(*[p.numel() for p in self.params])
        self._LR = (ctypes.c_double * n)(*[float(x) for x in self.lrs])

    def step(self, grads):
        n = len(self.params)
        G = (ctypes.c_void_p * n)(*[g.data_ptr() for g in grads])
        check(lib().svr_fused_adam_step_device(
            n, int(self.sparse), self._P, self._B, G, self._M, self._V, self._N, self._LR, float(self.betas[0]),
            float(self.betas[1]), float(self.eps), ctypes.c_void_p(self.d_step.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream(self.params[0].device).cuda_stream)), "fused_adam_step_device")


class GradientExchange:
    """View-parallel training across ranks: every rank renders its own views
    of the replicated scene, then one sum all-reduce of its flat gradient
    buffer makes every rank's gradient the gradient of the mean loss over all
    ranks' views, so the identical Adam update keeps the parameters
    replicated.  The loss is averaged the same way (for reporting)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1

    def __call__(self, flat_grad, loss=None):
        if self.world == 1:
            return
        self.dist.all_reduce(flat_grad, group=self.group)
        flat_grad.mul_(1.0 / self.world)
        if loss is not None:
            self.dist.all_reduce(loss, group=self.group)
            loss.mul_(1.0 / self.world)

    def start(self, bucket):
        """Start the sum all-reduce of one bucket without waiting for it (with
        NCCL it runs on the collective stream once the work already queued on
        the current stream is done, overlapping what is queued after it)."""
        if self.world == 1:
            return None
        return self.dist.all_reduce(bucket, group=self.group, async_op=True)

    def finish(self, pending):
        """Wait for started buckets ([(work, bucket)], the current stream waits
        on the collective stream) and turn their sums into means."""
        for work, bucket in pending:
            if work is not None:
                work.wait()
                bucket.mul_(1.0 / self.world)


class BatchedTrainWorkload:
    """One training step over all views: batched projection + SH, binning,
    compositing, L2 loss, recompute backward, multi-view SH backward and a
    fused Adam update of densities and SH (bf16 storage, fp32 moments);
    capturable as one CUDA graph (the step count lives on the device).

    With ``grid`` (vox_key [P,8], grid values [M]) the trained densities are
    grid points: gathered into the [P,8] corner buffer at the start of the
    step, their gradient scattered back after the compositing backward (the
    reference's GatherGeoParams around its rasterizer, once per step for all
    views).

    With ``exchange`` (a GradientExchange over several ranks) each rank
    renders its own views and the step becomes: graph (forward + compositing
    backward) -> start the all-reduce of the density gradients -> graph (SH
    backward, overlapping that all-reduce) -> all-reduce of the SH gradients
    and the loss -> graph (Adam)."""

    def __init__(self, scene, dev, storage=torch.bfloat16, lr_geo=0.025, lr_sh=0.01, betas=(0.1, 0.99),
                 eps=1e-15, tune=True, exchange=None, grid=None):
        from .batched import BatchedRasterizer, gather_grid_geos
        self.sc, self.dev, self.P = scene, dev, scene.n_voxels
        self.octpath = _t(scene.octpath.reshape(-1, 1), dev, torch.int64)
        self.centers = _t(scene.centers, dev)
        self.lengths = _t(scene.lengths, dev)
        # densities: per-voxel corners, or (grid = (vox_key [P,8], grid values [M])) grid points
        # gathered into the [P,8] corner buffer every step, as the reference trains them
        self.grid = None
        if grid is not None:
            self.vox_key = grid[0].to(dev).contiguous()
            self.grid = _t(grid[1], dev).to(storage).contiguous()
            self.geos = torch.empty(self.P, 8, dtype=storage, device=dev)
            gather_grid_geos(self.vox_key, self.grid, self.geos)
        else:
            self.geos = _t(scene.geos, dev).to(storage).contiguous()
        self.sh0 = _t(scene.sh0, dev).to(storage).contiguous()
        self.shs = _t(scene.shs, dev).to(storage).contiguous()
        self.cams = [_DevCam(c, dev) for c in scene.cameras]
        self.raster = BatchedRasterizer(self.cams, self.octpath, self.centers, self.lengths,
                                        max_level=scene.max_level)
        self.total = self.raster.fit_capacity(self.sh0, self.shs, 3)
        self.tuned = None
        if tune:
            self.tuned = tune_raster(self.raster, self.geos, self.sh0, self.shs)
            self.total = self.raster.fit_capacity(self.sh0, self.shs, 3)
        r = self.raster
        tg = [_t(t, dev).reshape(-1) for t in scene.targets]
        self.target = torch.cat([tg[i % len(tg)] for i in range(len(self.cams))])
        nv = len(self.cams)
        self.scale = torch.cat([torch.full((3 * h * w,), 2.0 / (3 * h * w * nv), device=dev) for h, w in r.sizes])
        self.color = torch.zeros(3 * r.n_pixels, device=dev)
        self.T = torch.zeros(r.n_pixels, device=dev)
        self.dT = torch.zeros(r.n_pixels, device=dev)
        self.dC = torch.zeros_like(self.color)
        self.loss = torch.zeros((), device=dev)
        # one flat buffer for the exchanged gradients: densities (per-voxel corners or grid
        # points), sh0, shs; the subdivision priority is not exchanged
        # (each part starts 256-byte aligned: the fused Adam reads 16-byte vectors)
        P = self.P
        pad = lambda n: (n + 63) // 64 * 64
        nd = 8 * P if self.grid is None else self.grid.numel()
        self.n_dens = pad(nd)  # the density bucket, padding included
        o_shs = self.n_dens + pad(3 * P)
        self.flat_grad = torch.zeros(o_shs + 45 * P, device=dev)
        dgeo = self.flat_grad[:nd].view(P, 8) if self.grid is None else torch.zeros(P, 8, device=dev)
        self.grads = (dgeo, torch.zeros(P, device=dev), self.flat_grad[self.n_dens:self.n_dens + 3 * P].view(P, 3),
                      self.flat_grad[o_shs:].view(P, 15, 3))
        dens = self.geos if self.grid is None else self.grid
        self.adam_grads = [self.flat_grad[:nd].view(dens.shape), self.grads[2], self.grads[3]]
        self.adam = DeviceAdam([dens, self.sh0, self.shs], [lr_geo, lr_sh, lr_sh], betas, eps)
        self.exchange = exchange if (exchange is not None and exchange.world > 1) else None
        self.graph = None
        self.graph_sh = None
        self.graph_adam = None

    def _forward_backward_render(self):
        from .batched import gather_grid_geos, scatter_grid_grad
        r = self.raster
        if self.grid is not None:
            gather_grid_geos(self.vox_key, self.grid, self.geos)
        r.prepare(self.sh0, self.shs, 3)
        r.render(self.geos, self.color, self.T)
        diff = self.color - self.target
        torch.mul(self.scale, diff, out=self.dC)
        self.loss.copy_((self.dC * diff).sum() * 0.5)  # mean over views of MSE (scale = 2 / (N_v V))
        self.grads[0].zero_()
        r.backward_render(self.geos, self.T, self.dC, self.dT, self.grads[0])
        if self.grid is not None:
            dgrid = self.flat_grad[:self.grid.numel()]
            dgrid.zero_()
            scatter_grid_grad(self.vox_key, self.grads[0], dgrid)

    def _backward_sh(self):
        g = self.grads
        self.raster.backward_sh(3, 16, g[2], g[3], g[1])

    def _forward_backward(self):
        self._forward_backward_render()
        self._backward_sh()

    def _adam(self):
        self.adam.step(self.adam_grads)

    def _step(self):
        self._forward_backward()
        self._adam()

    def capture(self):
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):  # warm-up launches (sets kernel attributes, allocator pools)
            self._eager_probe()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        if self.exchange is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._step()
            self.graph = g
        else:
            # the collectives stay outside the graphs: forward + compositing
            # backward, SH backward, Adam
            g, gs, ga = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._forward_backward_render()
            with torch.cuda.graph(gs):
                self._backward_sh()
            with torch.cuda.graph(ga):
                self._adam()
            self.graph, self.graph_sh, self.graph_adam = g, gs, ga

    def replay(self):
        """One training step from the captured graph(s)."""
        self.graph.replay()
        if self.exchange is not None:
            dens, sh = self.flat_grad[:self.n_dens], self.flat_grad[self.n_dens:]
            w_dens = self.exchange.start(dens)       # densities are final: exchange them ...
            self.graph_sh.replay()                   # ... while the SH backward runs
            pending = [(w_dens, dens), (self.exchange.start(sh), sh), (self.exchange.start(self.loss), self.loss)]
            self.exchange.finish(pending)
            self.graph_adam.replay()

    def _eager_probe(self):
        # one forward/backward without the optimizer update, so parameters are untouched
        self._forward_backward()

    def release(self):
        """Drop the captured graphs (before the process group is destroyed)."""
        self.graph = self.graph_sh = self.graph_adam = None

    def run(self, steps):
        if self.graph is None:
            self.capture()
        losses = torch.zeros(steps, device=self.dev)
        st = torch.cuda.current_stream(self.dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for i in range(steps):
            self.replay()
            losses[i].copy_(self.loss)
        e1.record(st)
        torch.cuda.synchronize()
        total, err = self.raster.header()
        if err:
            raise RuntimeError(f"training step reported device error word 0x{err:x}")
        return e0.elapsed_time(e1) / steps, losses.cpu().tolist()


class PlainTrainWorkload:
    """The same training step in the reference's form: fp32 parameters, one
    view per call with its host syncs (visible-index and instance-count
    reads), gradients accumulated over the views, then SparseAdam's
    per-parameter launches with host-side bias correction.  With ``grid``
    (vox_key, grid values) the densities are grid points gathered per view
    through GatherGeoParams, as the reference's model does."""

    def __init__(self, scene, dev, lr_geo=0.025, lr_sh=0.01, betas=(0.1, 0.99), eps=1e-15, grid=None):
        from .sparse_adam import SparseAdam
        self.sc, self.dev, self.P = scene, dev, scene.n_voxels
        self.octpath = _t(scene.octpath.reshape(-1, 1), dev, torch.int64)
        self.centers = _t(scene.centers, dev)
        self.lengths = _t(scene.lengths, dev)
        self.grid = None
        if grid is not None:  # grid-point densities through GatherGeoParams (sparse_voxel_gears/renderer.py)
            self.vox_key = grid[0].to(dev).contiguous()
            self.care_idx = torch.arange(self.P, device=dev)
            self.grid = _t(grid[1], dev).reshape(-1, 1).requires_grad_(True)
            self.geos = None
        else:
            self.geos = _t(scene.geos, dev).requires_grad_(True)
        self.sh0 = _t(scene.sh0, dev).requires_grad_(True)
        self.shs = _t(scene.shs, dev).requires_grad_(True)
        self.cams = [(c, _t(c.w2c, dev), _t(c.c2w, dev)) for c in scene.cameras]
        self.targets = [_t(t, dev) for t in scene.targets]
        dens = self.geos if self.grid is None else self.grid
        self.opt = SparseAdam([{"params": [dens], "lr": lr_geo}, {"params": [self.sh0], "lr": lr_sh},
                               {"params": [self.shs], "lr": lr_sh}], betas=betas, eps=eps)

    def _step(self):
        from . import renderer
        for p in (self.geos, self.grid, self.sh0, self.shs):
            if p is not None:
                p.grad = None
        total = None
        nv = len(self.cams)
        ones = torch.ones(self.P, 1, device=self.dev)
        for i, (cam, w2c, c2w) in enumerate(self.cams):
            s = renderer.RasterSettings("sh", 1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy,
                                        w2c, c2w)

            def vox_fn(idx, cam_pos, mode):
                rg = renderer.SH_eval.apply(3, idx, self.centers, cam_pos, None, self.sh0, self.shs)
                geos = self.geos if self.grid is None else \
                    renderer.GatherGeoParams.apply(self.vox_key, self.care_idx, self.grid)
                return {"geos": geos, "rgbs": rg, "subdiv_p": ones}

            color, _, _, _, _ = renderer.rasterize_voxels(s, self.octpath, self.centers, self.lengths, vox_fn)
            loss = ((color - self.targets[i % len(self.targets)]) ** 2).mean() / nv
            loss.backward()
            total = loss.detach() if total is None else total + loss.detach()
        self.opt.step()
        return total

    def run(self, steps, warmup=2):
        """Runs `steps` training steps from the initial parameters and returns
        (ms per step, losses of all steps).  The first `warmup` steps (first
        kernel loads, allocator growth, optimizer state) are left out of the
        timing but not out of the losses, so the trajectories still compare
        step for step with the batched form's."""
        st = torch.cuda.current_stream(self.dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        warmup = min(warmup, max(steps - 1, 0))
        losses = []
        for k in range(steps):
            if k == warmup:
                torch.cuda.synchronize()
                e0.record(st)
            losses.append(self._step())
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / (steps - warmup), [float(x) for x in torch.stack(losses).cpu()]
